// Probability and Pauli-string expectation kernels (sm_100a), FP64
// accumulation for both precisions.
//
// The reference has no expectation result type (only StateVector is
// registered: src/braket/snuqs/result_types.py:149-151) and computes
// probabilities on the host from a full device-to-host copy
// (src/braket/snuqs/simulation.py:208-215).
//
// Expectation of a Pauli string P with X-or-Y mask x, Z-or-Y mask zy and ny
// Y factors (index bits):
//   <P> = (-i)^ny * sum_i (-1)^popc(i & zy) conj(psi_i) psi_(i^x).
// Terms are grouped by (x, ny mod 2).  For x != 0 the pair (i, i^x), i with
// the top bit of x clear, contributes (-1)^popc(i&zy) * q(i) with
// q = 2 Re(conj(psi_i) psi_j) (ny even) or 2 Im(...) (ny odd); the host folds
// the weight and the (-i)^ny phase into one real factor per term, so a group
// costs one read of the state and the kernel needs one FP64 accumulator.
#pragma once
#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stdint.h>

#include "sweep_kernels.cuh"
#endif

namespace sq {

constexpr int kMaxTerms = 1024;
constexpr int kMaxGroups = 256;
constexpr int kReduceThreads = 256;

struct PauliGroup {
  uint64_t x;        // flip mask (index bits)
  uint32_t odd;      // ny odd: q uses the imaginary part
  uint32_t t0, t1;   // term range
  uint32_t pad;
};

struct PauliParams {
  uint32_t n, ngroups;
  PauliGroup g[kMaxGroups];
  uint64_t zy[kMaxTerms];
  double f[kMaxTerms];
};

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = v;
  __syncthreads();
  v = 0;
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    v = lane < nw ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  __syncthreads();
  return v;  // valid in thread 0
}

// partial[blockIdx.x] (+)= this block's share of sum_groups sum_pairs q * W.
template <typename Real>
__global__ void __launch_bounds__(kReduceThreads)
    pauli_expect_kernel(const typename Vec2<Real>::T *__restrict__ psi,
                        const __grid_constant__ PauliParams P, double *__restrict__ partial,
                        int accumulate) {
  using C2 = typename Vec2<Real>::T;
  double acc = 0.0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint32_t gi = 0; gi < P.ngroups; ++gi) {
    const PauliGroup &G = P.g[gi];
    if (G.x == 0) {
      const uint64_t N = uint64_t(1) << P.n;
      for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += stride) {
        const C2 a = psi[i];
        const double q = double(a.x) * double(a.x) + double(a.y) * double(a.y);
        double w = 0.0;
        for (uint32_t t = G.t0; t < G.t1; ++t)
          w += (__popcll(i & P.zy[t]) & 1) ? -P.f[t] : P.f[t];
        acc = fma(q, w, acc);
      }
    } else {
      const uint32_t hb = 63 - __clzll(G.x);
      const uint64_t N = uint64_t(1) << (P.n - 1);
      for (uint64_t h = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; h < N; h += stride) {
        const uint64_t i = insert_zero(h, hb), j = i ^ G.x;
        const C2 a = psi[i], b = psi[j];
        // conj(a) * b
        const double zr = double(a.x) * double(b.x) + double(a.y) * double(b.y);
        const double zi = double(a.x) * double(b.y) - double(a.y) * double(b.x);
        const double q = 2.0 * (G.odd ? zi : zr);
        double w = 0.0;
        for (uint32_t t = G.t0; t < G.t1; ++t)
          w += (__popcll(i & P.zy[t]) & 1) ? -P.f[t] : P.f[t];
        acc = fma(q, w, acc);
      }
    }
  }
  const double s = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = accumulate ? partial[blockIdx.x] + s : s;
}

// out[0] = sum of partial[0..n) in a fixed order (deterministic).
static __global__ void __launch_bounds__(kReduceThreads)
    finalize_sum_kernel(const double *__restrict__ partial, uint32_t n, double *__restrict__ out) {
  double v = 0.0;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) v += partial[i];
  const double s = block_sum(v);
  if (threadIdx.x == 0) out[0] = s;
}

template <typename Real>
__global__ void __launch_bounds__(kReduceThreads)
    probabilities_kernel(const typename Vec2<Real>::T *__restrict__ psi, uint64_t N,
                         double *__restrict__ out) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const auto a = psi[i];
    out[i] = double(a.x) * double(a.x) + double(a.y) * double(a.y);
  }
}

template <typename Real>
__global__ void set_amplitude_kernel(typename Vec2<Real>::T *psi, uint64_t index, Real re, Real im) {
  typename Vec2<Real>::T v;
  v.x = re;
  v.y = im;
  psi[index] = v;
}

}  // namespace sq

// Adjoint-gradient kernels (sm_100a).
//
// adjoint_sweep_kernel: the two-state analogue of sweep_kernel.  Each thread
//   holds 8 amplitudes of phi and the same 8 amplitudes of lambda (3 register
//   bits per phase); every un-compute gate U^dagger is applied to both, and
//   every inner-product op accumulates <lambda| K |phi> over the tile into a
//   per-warp slot in shared memory.  phi and lambda are each read and written
//   once per sweep, however many gates and parameters the sweep carries.
// pauli_apply_kernel: lambda = H psi for a Pauli-string sum, with
//   E = Re <psi|lambda> accumulated in FP64 in the same pass.
// inner_reduce_kernel: fixed-order sum of the per-warp partials of each slot.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "reduce_kernels.cuh"
#include "sweep_kernels.cuh"

namespace sq {

struct PauliApplyGroup {
  uint64_t x;        // flip mask
  uint32_t t0, t1;   // term range
};

struct PauliApplyParams {
  uint32_t n, ngroups;
  PauliApplyGroup g[kMaxGroups];
  uint64_t zy[kMaxTerms];
  double wr[kMaxTerms], wi[kMaxTerms];  // w_t * (-i)^ny_t
  // Bit r of sgn[t]: parity of the two top index bits r (amplitude r of a
  // thread's four) under zy_t.  real[g / 32] bit g % 32: every wi of group g
  // is zero.
  uint8_t sgn[kMaxTerms];
  uint32_t real[kMaxGroups / 32];
};

// out[i] = sum_t w_t (-i)^ny_t (-1)^popc(i & zy_t) psi[i ^ x_t];
// partial[block] = this block's share of Re <psi|out> (FP64).  Each thread
// takes the four amplitudes j + r 2^(n-2) (r = 0..3; for each r the lanes
// read consecutive amplitudes): one popcount per term serves all four, and
// the imaginary weights are skipped for groups whose weights are real.  The
// per-amplitude sums add the signed weights in term order, as a direct
// evaluation would.
template <typename Real>
__global__ void __launch_bounds__(kReduceThreads)
    pauli_apply_kernel(const typename Vec2<Real>::T *__restrict__ psi,
                       typename Vec2<Real>::T *__restrict__ out,
                       const __grid_constant__ PauliApplyParams P, double *__restrict__ partial) {
  using C2 = typename Vec2<Real>::T;
  const uint32_t hs = P.n - 2;
  const uint64_t Q = uint64_t(1) << hs;
  double e = 0.0;
  for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < Q;
       j += uint64_t(gridDim.x) * blockDim.x) {
    double ar[4] = {0.0, 0.0, 0.0, 0.0}, ai[4] = {0.0, 0.0, 0.0, 0.0};
    for (uint32_t gi = 0; gi < P.ngroups; ++gi) {
      const PauliApplyGroup &G = P.g[gi];
      const bool real = (P.real[gi >> 5] >> (gi & 31)) & 1u;
      double cr[4] = {0.0, 0.0, 0.0, 0.0}, ci[4] = {0.0, 0.0, 0.0, 0.0};
      for (uint32_t t = G.t0; t < G.t1; ++t) {
        const uint32_t sg = P.sgn[t] ^ ((__popcll(j & P.zy[t]) & 1u) ? 0xfu : 0u);
        const double wr = P.wr[t];
#pragma unroll
        for (int r = 0; r < 4; ++r) cr[r] += ((sg >> r) & 1u) ? -wr : wr;
        if (!real) {
          const double wi = P.wi[t];
#pragma unroll
          for (int r = 0; r < 4; ++r) ci[r] += ((sg >> r) & 1u) ? -wi : wi;
        }
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const C2 b = psi[(j | (uint64_t(r) << hs)) ^ G.x];
        ar[r] += cr[r] * double(b.x) - ci[r] * double(b.y);
        ai[r] += cr[r] * double(b.y) + ci[r] * double(b.x);
      }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const uint64_t i = j | (uint64_t(r) << hs);
      C2 o;
      o.x = Real(ar[r]);
      o.y = Real(ai[r]);
      out[i] = o;
      const C2 a = psi[i];
      e += double(a.x) * ar[r] + double(a.y) * ai[r];  // Re(conj(a) * acc)
    }
  }
  const double s = block_sum(e);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

template <typename Real>
__device__ __forceinline__ void inner_op(const Amps<Real, kAdjAmps> &F, const Amps<Real, kAdjAmps> &G,
                                         const typename Vec2<Real>::T *coef, const SweepOp &op,
                                         uint64_t gbase, uint32_t jb, double &sr, double &si) {
  const auto *c = coef + op.coef;
  if (op.kind == kSwInnerDiag) {
    const uint32_t base = diag_base<Real>(op, gbase, jb);
    switch (op.vmask) {
#define SQ_CASE(V) \
  case V: inner_diag<Real, V>(F, G, c, base, sr, si); break;
      SQ_CASE(0) SQ_CASE(1) SQ_CASE(2) SQ_CASE(3) SQ_CASE(4) SQ_CASE(5) SQ_CASE(6) SQ_CASE(7)
#undef SQ_CASE
    }
  } else {
    switch (op.vmask) {
#define SQ_CASE(V) \
  case V: inner_dense<Real, V>(F, G, c, sr, si); break;
      SQ_CASE(1) SQ_CASE(2) SQ_CASE(3) SQ_CASE(4) SQ_CASE(5) SQ_CASE(6) SQ_CASE(7)
#undef SQ_CASE
    }
  }
}

// Two-state fused sweep over 2^M-amplitude tiles; 2^(M-3) threads.
// Dynamic shared memory: phi tiles (2 buffers) | lambda tiles (2 buffers) |
// coefficients | high-bit table | per-warp inner-product slots.
// partials[(block * warps + warp) * kMaxInner + slot] receives each warp's
// sums (complex, FP64) at the end.
template <typename Real, int M>
__global__ void __launch_bounds__(1 << (M - kAdjRegBits), 1)
    adjoint_sweep_kernel(typename Vec2<Real>::T *__restrict__ psi,
                         typename Vec2<Real>::T *__restrict__ lam,
                         const __grid_constant__ SweepParams<Real> P,
                         double2 *__restrict__ partials) {
  using C2 = typename Vec2<Real>::T;
  constexpr int NT = 1 << (M - kAdjRegBits);
  constexpr int NW = (NT + 31) / 32;
  constexpr int L = sweep_low_bits(M);
  constexpr uint32_t TS = 1u << M;
  constexpr uint32_t PER = TS / NT;
  constexpr uint32_t LOWMASK = (1u << L) - 1u;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SweepHeader &h = P.h;
  C2 *fbufs = reinterpret_cast<C2 *>(smem_raw);
  C2 *lbufs = fbufs + 2 * TS;
  C2 *coef = lbufs + 2 * TS;
  uint64_t *hitab = reinterpret_cast<uint64_t *>(coef + ((h.ncoef + 1) & ~1u));
  double2 *acc = reinterpret_cast<double2 *>(hitab + (1u << (M - L)));
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  for (uint32_t i = tid; i < h.ncoef; i += NT) {
    C2 v;
    v.x = P.coef[2 * i];
    v.y = P.coef[2 * i + 1];
    coef[i] = v;
  }
  for (uint32_t c = tid; c < (1u << (M - L)); c += NT) {
    uint64_t a = 0;
#pragma unroll
    for (int i = 0; i < M - L; ++i)
      if ((c >> i) & 1) a |= uint64_t(1) << h.hi[i];
    hitab[c] = a;
  }
  for (uint32_t i = tid; i < NW * kMaxInner; i += NT) acc[i] = make_double2(0.0, 0.0);
  __syncthreads();

  const uint32_t s_tid = swz<Real>(tid);
  auto prefetch = [&](uint64_t t, C2 *fdst, C2 *ldst) {
    const uint64_t gb = tile_base(t, h);
#pragma unroll
    for (uint32_t it = 0; it < PER; ++it) {
      const uint32_t j = it * NT + tid;
      const uint64_t g = gb | hitab[j >> L] | (j & LOWMASK);
      const uint32_t slot = s_tid ^ swz<Real>(it * NT);
      cp_async<sizeof(C2)>(fdst + slot, psi + g);
      cp_async<sizeof(C2)>(ldst + slot, lam + g);
    }
  };

  const uint32_t last = h.nphases - 1;
  uint32_t cur = 0;
  if (blockIdx.x < h.num_tiles) prefetch(blockIdx.x, fbufs, lbufs);
  cp_async_commit();
  for (uint64_t t = blockIdx.x; t < h.num_tiles; t += gridDim.x) {
    C2 *ftile = fbufs + cur * TS;
    C2 *ltile = lbufs + cur * TS;
    const uint64_t tn = t + gridDim.x;
    if (tn < h.num_tiles) prefetch(tn, fbufs + (cur ^ 1) * TS, lbufs + (cur ^ 1) * TS);
    cp_async_commit();
    cp_async_wait_prev();
    __syncthreads();
    const uint64_t gbase = tile_base(t, h);
    for (uint32_t p = 0; p <= last; ++p) {
      const SweepPhase &ph = P.ph[p];
      uint32_t jb = tid;
#pragma unroll
      for (int b = 0; b < kAdjRegBits; ++b) jb = uint32_t(insert_zero(jb, ph.reg[b]));
      const uint32_t sb = swz<Real>(jb);
      const uint32_t w0 = swz<Real>(1u << ph.reg[0]), w1 = swz<Real>(1u << ph.reg[1]);
      const uint32_t w2 = swz<Real>(1u << ph.reg[2]);
      Amps<Real, kAdjAmps> F, G;
#pragma unroll
      for (int ri = 0; ri < kAdjAmps; ++ri) {
        const uint32_t s = sb ^ ((ri & 1) ? w0 : 0) ^ ((ri & 2) ? w1 : 0) ^ ((ri & 4) ? w2 : 0);
        const C2 a = ftile[s], b = ltile[s];
        F.re[ri] = a.x;
        F.im[ri] = a.y;
        G.re[ri] = b.x;
        G.im[ri] = b.y;
      }
      for (uint32_t o = ph.op_begin; o < ph.op_end; ++o) {
        const SweepOp &op = P.op[o];
        if (op.kind == kSwInnerDiag || op.kind == kSwInnerDense) {
          double sr = 0.0, si = 0.0;
          inner_op<Real>(F, G, coef, op, gbase, jb, sr, si);
          // Warp sum (the warp is partial when the tile has < 32 threads).
          constexpr unsigned kMask = NT >= 32 ? 0xffffffffu : ((1u << NT) - 1u);
#pragma unroll
          for (int off = (NT >= 32 ? 16 : NT / 2); off > 0; off >>= 1) {
            sr += __shfl_xor_sync(kMask, sr, off);
            si += __shfl_xor_sync(kMask, si, off);
          }
          if (lane == 0) {
            double2 &a = acc[warp * kMaxInner + op.slot];
            a.x += sr;
            a.y += si;
          }
        } else {
          apply_op<Real, kAdjAmps>(F, coef, op, gbase, jb);
          apply_op<Real, kAdjAmps>(G, coef, op, gbase, jb);
        }
      }
#pragma unroll
      for (int ri = 0; ri < kAdjAmps; ++ri) {
        const uint32_t s = sb ^ ((ri & 1) ? w0 : 0) ^ ((ri & 2) ? w1 : 0) ^ ((ri & 4) ? w2 : 0);
        C2 a, b;
        a.x = F.re[ri];
        a.y = F.im[ri];
        b.x = G.re[ri];
        b.y = G.im[ri];
        ftile[s] = a;
        ltile[s] = b;
      }
      __syncthreads();
    }
#pragma unroll
    for (uint32_t it = 0; it < PER; ++it) {
      const uint32_t j = it * NT + tid;
      const uint64_t g = gbase | hitab[j >> L] | (j & LOWMASK);
      const uint32_t slot = s_tid ^ swz<Real>(it * NT);
      psi[g] = ftile[slot];
      lam[g] = ltile[slot];
    }
    __syncthreads();
    cur ^= 1;
  }
  cp_async_wait_prev();
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  for (uint32_t i = tid; i < NW * kMaxInner; i += NT)
    partials[size_t(blockIdx.x) * NW * kMaxInner + i] = acc[i];
}

struct InnerSlots {
  uint32_t nslots;
  uint32_t nrows;  // blocks x warps
  uint32_t global[kMaxInner];
};

// ipvals[global[s]] += sum over rows of partials[row * kMaxInner + s], in row
// order (deterministic).  One block per slot.
static __global__ void __launch_bounds__(kReduceThreads)
    inner_reduce_kernel(const double2 *__restrict__ partials, const __grid_constant__ InnerSlots S,
                        double2 *__restrict__ ipvals) {
  const uint32_t s = blockIdx.x;
  double r = 0.0, i = 0.0;
  for (uint32_t row = threadIdx.x; row < S.nrows; row += blockDim.x) {
    const double2 v = partials[size_t(row) * kMaxInner + s];
    r += v.x;
    i += v.y;
  }
  r = block_sum(r);
  i = block_sum(i);
  if (threadIdx.x == 0) {
    double2 &o = ipvals[S.global[s]];
    o.x += r;
    o.y += i;
  }
}

}  // namespace sq

// Result kernels beyond the expectation value: measurement sampling,
// amplitude lookup, marginal probabilities and Pauli-sum variance.
//
// The reference computes every result on the host after copying the whole
// state back: probabilities as |psi|^2 in numpy and shots with
// np.random.choice over them (src/braket/snuqs/simulation.py:208-220); its
// plugin registers no Expectation / Variance / Probability / Amplitude
// result types (src/braket/snuqs/result_types.py:149-151,
// src/braket/snuqs/simulator.py:578-580).  Here each is a device pass over
// the resident state and only the results cross PCIe.
//
// Sampling is an inverse CDF over |psi_i|^2 that is reproducible bit for bit:
// the probabilities are summed in one fixed binary tree (pairs of adjacent
// amplitudes, then pairs of pairs, ...), and a shot with uniform u walks that
// tree from the root with r = u * total: at a node with children sums (L, R)
// it goes left when r < L or R == 0, else subtracts L and goes right.  The
// tree is split at leaves of 2^12 amplitudes: the levels above the leaves
// stay in device memory, the levels inside a leaf are rebuilt in shared
// memory by the block that serves the leaf's shots.  Any restatement that
// sums in the same tree and walks it the same way returns the same indices.
#include <cuda_runtime.h>

#include <algorithm>
#include <complex>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "../../include/snuqs_b200.h"
#include "engine_internal.h"
#include "sweep_kernels.cuh"

namespace {

constexpr int kLeafBits = 12;
constexpr uint32_t kLeafAmps = 1u << kLeafBits;
constexpr int kLeafThreads = 256;
constexpr uint32_t kPerThread = kLeafAmps / kLeafThreads;  // 16 consecutive amplitudes

template <typename C2>
__device__ __forceinline__ double prob(const C2 *__restrict__ psi, uint64_t i, uint64_t N) {
  if (i >= N) return 0.0;  // states below 2^12 amplitudes are padded with zeros
  const C2 a = psi[i];
  const double re = double(a.x), im = double(a.y);
  return __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
}

// Sum of one leaf in the fixed tree (pairwise sums over consecutive
// amplitudes, level by level).  Warp w covers the 512 amplitudes from
// 512 w; lane l reads amplitude 32 k + l for k = 0..15 (coalesced), the five
// lowest levels of each group of 32 are lane pairs l, l^1, l^2, ... (shuffles;
// a commutative add gives both partners the same value), the next four are
// the groups k in registers, then the warps pairwise through shared memory.
template <typename C2>
__global__ void __launch_bounds__(kLeafThreads) leaf_sum_kernel(const C2 *__restrict__ psi, uint64_t N,
                                                                double *__restrict__ leaves) {
  __shared__ double ws[kLeafThreads / 32];
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t base = uint64_t(blockIdx.x) * kLeafAmps + uint64_t(threadIdx.x >> 5) * (32 * kPerThread) + lane;
  double v[kPerThread];
#pragma unroll
  for (uint32_t k = 0; k < kPerThread; ++k) v[k] = prob(psi, base + 32 * k, N);
#pragma unroll
  for (int o = 1; o < 32; o <<= 1)
#pragma unroll
    for (uint32_t k = 0; k < kPerThread; ++k) v[k] = __dadd_rn(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
#pragma unroll
  for (uint32_t w = kPerThread / 2; w >= 1; w >>= 1)
#pragma unroll
    for (uint32_t j = 0; j < w; ++j) v[j] = __dadd_rn(v[2 * j], v[2 * j + 1]);
  const double s = v[0];
  if (lane == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double w[kLeafThreads / 32];
#pragma unroll
    for (int j = 0; j < kLeafThreads / 32; ++j) w[j] = ws[j];
#pragma unroll
    for (int m = kLeafThreads / 64; m >= 1; m >>= 1)
#pragma unroll
      for (int j = 0; j < m; ++j) w[j] = __dadd_rn(w[2 * j], w[2 * j + 1]);
    leaves[blockIdx.x] = w[0];
  }
}

// Levels above the leaves: level d (2^d nodes) at tree + 2^d - 1, so the root
// is tree[0] and the leaves (depth D) start at tree + 2^D - 1.
__global__ void __launch_bounds__(1024) upper_tree_kernel(double *__restrict__ tree, uint32_t depth) {
  for (int d = int(depth) - 1; d >= 0; --d) {
    const uint64_t nodes = uint64_t(1) << d;
    double *lv = tree + (nodes - 1), *ch = tree + (2 * nodes - 1);
    for (uint64_t k = threadIdx.x; k < nodes; k += blockDim.x) lv[k] = __dadd_rn(ch[2 * k], ch[2 * k + 1]);
    __syncthreads();
  }
}

__device__ __forceinline__ bool go_left(double r, double l, double rr) { return r < l || rr == 0.0; }

// Per shot: r = u * total, walk down to a leaf; count the shots per leaf.
__global__ void shot_descend_kernel(const double *__restrict__ tree, uint32_t depth,
                                    const double *__restrict__ u, uint64_t shots, uint32_t *__restrict__ leaf,
                                    double *__restrict__ resid, uint32_t *__restrict__ count) {
  const uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= shots) return;
  double r = __dmul_rn(u[s], tree[0]);
  uint64_t k = 0;
  for (uint32_t d = 0; d < depth; ++d) {
    const double *ch = tree + ((uint64_t(2) << d) - 1);
    const double l = ch[2 * k], rr = ch[2 * k + 1];
    if (go_left(r, l, rr)) {
      k = 2 * k;
    } else {
      r = __dsub_rn(r, l);
      k = 2 * k + 1;
    }
  }
  leaf[s] = uint32_t(k);
  resid[s] = r;
  atomicAdd(&count[k], 1u);
}

// Exclusive scan of the per-leaf counts (one block; leaves <= 2^22): 1024
// counts per step, read coalesced, scanned with warp shuffles.
__global__ void __launch_bounds__(1024) count_scan_kernel(const uint32_t *__restrict__ count, uint32_t nleaves,
                                                          uint32_t *__restrict__ offset,
                                                          uint32_t *__restrict__ cursor) {
  __shared__ uint32_t wsum[32];
  __shared__ uint32_t total;
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  uint32_t base = 0;
  for (uint32_t t0 = 0; t0 < nleaves; t0 += 1024) {
    const uint32_t i = t0 + threadIdx.x;
    const uint32_t v = i < nleaves ? count[i] : 0u;
    uint32_t x = v;  // inclusive scan within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= uint32_t(o)) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      const uint32_t sw = wsum[lane];
      uint32_t y = sw;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t z = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= uint32_t(o)) y += z;
      }
      wsum[lane] = y - sw;  // exclusive over warps
      if (lane == 31) total = y;
    }
    __syncthreads();
    const uint32_t excl = base + wsum[w] + x - v;
    if (i < nleaves) {
      offset[i] = excl;
      cursor[i] = excl;
    }
    base += total;
    __syncthreads();
  }
}

__global__ void shot_bucket_kernel(const uint32_t *__restrict__ leaf, uint64_t shots, uint32_t *__restrict__ cursor,
                                   uint32_t *__restrict__ order) {
  const uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= shots) return;
  order[atomicAdd(&cursor[leaf[s]], 1u)] = uint32_t(s);
}

// One block per leaf with shots: the leaf's tree in shared memory (the same
// sums as leaf_sum_kernel), then each of its shots walks it to an amplitude.
template <typename C2>
__global__ void __launch_bounds__(kLeafThreads) leaf_sample_kernel(const C2 *__restrict__ psi, uint64_t N,
                                                                   uint32_t nleaves, const uint32_t *__restrict__ count,
                                                                   const uint32_t *__restrict__ offset,
                                                                   const uint32_t *__restrict__ order,
                                                                   const double *__restrict__ resid,
                                                                   uint64_t *__restrict__ out) {
  extern __shared__ double t[];  // level k (2^k nodes) at t + 2^k - 1; leaves' amplitudes at depth 12
  for (uint32_t lf = blockIdx.x; lf < nleaves; lf += gridDim.x) {
    const uint32_t c = count[lf];
    if (c == 0) continue;
    const uint64_t base = uint64_t(lf) * kLeafAmps;
    double *amps = t + (kLeafAmps - 1);
    for (uint32_t j = threadIdx.x; j < kLeafAmps; j += blockDim.x) amps[j] = prob(psi, base + j, N);
    __syncthreads();
    for (int d = kLeafBits - 1; d >= 0; --d) {
      const uint32_t nodes = 1u << d;
      double *lv = t + (nodes - 1), *ch = t + (2 * nodes - 1);
      for (uint32_t k = threadIdx.x; k < nodes; k += blockDim.x) lv[k] = __dadd_rn(ch[2 * k], ch[2 * k + 1]);
      __syncthreads();
    }
    const uint32_t o = offset[lf];
    for (uint32_t q = threadIdx.x; q < c; q += blockDim.x) {
      const uint32_t s = order[o + q];
      double r = resid[s];
      uint32_t k = 0;
      for (int d = 0; d < kLeafBits; ++d) {
        const double *ch = t + ((2u << d) - 1);
        const double l = ch[2 * k], rr = ch[2 * k + 1];
        if (go_left(r, l, rr)) {
          k = 2 * k;
        } else {
          r = __dsub_rn(r, l);
          k = 2 * k + 1;
        }
      }
      out[s] = base + k;
    }
    __syncthreads();
  }
}

template <typename C2>
__global__ void amplitude_kernel(const C2 *__restrict__ psi, uint64_t N, const uint64_t *__restrict__ idx,
                                 uint64_t count, double2 *__restrict__ out, uint32_t *__restrict__ bad) {
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint64_t j = idx[i];
  if (j >= N) {
    atomicOr(bad, 1u);
    out[i] = make_double2(0.0, 0.0);
    return;
  }
  const C2 a = psi[j];
  out[i] = make_double2(double(a.x), double(a.y));
}

// Marginal probabilities over k target bits: block (bin b, chunk c) sums
// |psi_i|^2 over the indices i whose target bits spell b and whose other
// bits fall in chunk c, in a fixed order; marginal_finalize adds a bin's
// chunks in order.
struct MarginalParams {
  uint32_t n, k;
  uint8_t tbit[64];  // index bit of target j (j = 0 is the most significant bit of b)
  uint64_t tmask;
};

__device__ __forceinline__ uint64_t deposit_rest(uint64_t r, uint64_t tmask, uint32_t n) {
  // Spread r over the index bits outside tmask, ascending.
  uint64_t x = 0;
  for (uint32_t p = 0, q = 0; p < n; ++p) {
    if ((tmask >> p) & 1) continue;
    x |= ((r >> q) & 1) << p;
    ++q;
  }
  return x;
}

template <typename C2>
__global__ void __launch_bounds__(256) marginal_kernel(const C2 *__restrict__ psi, const MarginalParams P,
                                                       uint32_t chunks, double *__restrict__ partial) {
  __shared__ double ws[8];
  const uint64_t bins = uint64_t(1) << P.k;
  const uint64_t rest = uint64_t(1) << (P.n - P.k);
  const uint64_t per = (rest + chunks - 1) / chunks;
  for (uint64_t item = blockIdx.x; item < bins * chunks; item += gridDim.x) {
    const uint64_t b = item / chunks, c = item % chunks;
    uint64_t tb = 0;
    for (uint32_t j = 0; j < P.k; ++j)
      if ((b >> (P.k - 1 - j)) & 1) tb |= uint64_t(1) << P.tbit[j];
    const uint64_t r0 = c * per, r1 = min(rest, r0 + per);
    double acc = 0.0;
    for (uint64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
      const C2 a = psi[deposit_rest(r, P.tmask, P.n) | tb];
      acc += double(a.x) * double(a.x) + double(a.y) * double(a.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int w = 0; w < 8; ++w) s += ws[w];
      partial[item] = s;
    }
    __syncthreads();
  }
}

__global__ void marginal_finalize_kernel(const double *__restrict__ partial, uint64_t bins, uint32_t chunks,
                                         double *__restrict__ out) {
  const uint64_t b = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= bins) return;
  double s = 0.0;
  for (uint32_t c = 0; c < chunks; ++c) s += partial[b * chunks + c];
  out[b] = s;
}

// Distance between two states of the same size, any precisions: per block
// max |a_i - b_i| and the FP64 sums <a|b> (re, im), <a|a>, <b|b>.
template <typename CA, typename CB>
__global__ void __launch_bounds__(256) distance_kernel(const CA *__restrict__ a, const CB *__restrict__ b, uint64_t N,
                                                       double *__restrict__ part) {
  __shared__ double sm[5][8];
  double mx = 0.0, re = 0.0, im = 0.0, na = 0.0, nb = 0.0;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < N; i += uint64_t(gridDim.x) * blockDim.x) {
    const double ar = double(a[i].x), ai = double(a[i].y), br = double(b[i].x), bi = double(b[i].y);
    mx = fmax(mx, hypot(ar - br, ai - bi));
    re += ar * br + ai * bi;  // conj(a) b
    im += ar * bi - ai * br;
    na += ar * ar + ai * ai;
    nb += br * br + bi * bi;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
    na += __shfl_xor_sync(0xffffffffu, na, o);
    nb += __shfl_xor_sync(0xffffffffu, nb, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sm[0][w] = mx;
    sm[1][w] = re;
    sm[2][w] = im;
    sm[3][w] = na;
    sm[4][w] = nb;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double v = threadIdx.x == 0 ? 0.0 : 0.0;
    for (int j = 0; j < 8; ++j) v = threadIdx.x == 0 ? fmax(v, sm[0][j]) : v + sm[threadIdx.x][j];
    part[uint64_t(blockIdx.x) * 5 + threadIdx.x] = v;
  }
}

int fail(int code, const std::string &msg) { return sq_detail_fail(code, msg.c_str()); }

#define RQ_CUDA(call)                                                                         \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(e_ == cudaErrorMemoryAllocation ? SQ_ERR_OOM : SQ_ERR_CUDA,                 \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                        \
  } while (0)

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Scratch bytes of sample_impl: the upper tree, per-leaf counts / offsets /
// cursors, per-shot leaf, residual and bucket order.
size_t sample_scratch_bytes(uint32_t n, uint64_t shots) {
  const uint32_t depth = n > uint32_t(kLeafBits) ? n - kLeafBits : 0;
  const uint64_t nleaves = uint64_t(1) << depth;
  return align256((2 * nleaves - 1) * sizeof(double)) + 3 * align256(nleaves * sizeof(uint32_t)) +
         2 * align256(shots * sizeof(uint32_t)) + align256(shots * sizeof(double));
}

// u_ready (optional): an event the shot phase waits for before reading the
// uniforms (they may still be in flight on another stream while the
// probability tree is built).
template <typename C2>
int sample_impl(const C2 *psi, uint32_t n, const double *u, uint64_t shots, uint64_t *out, void *scr,
                cudaStream_t st, cudaEvent_t u_ready = nullptr, const std::function<int()> &before_shots = {}) {
  const uint64_t N = uint64_t(1) << n;
  const uint32_t depth = n > uint32_t(kLeafBits) ? n - kLeafBits : 0;
  const uint64_t nleaves = uint64_t(1) << depth;
  const size_t b_tree = align256((2 * nleaves - 1) * sizeof(double));
  const size_t b_leafu = align256(nleaves * sizeof(uint32_t));
  const size_t b_shot32 = align256(shots * sizeof(uint32_t));
  char *p = static_cast<char *>(scr);
  double *tree = reinterpret_cast<double *>(p);
  p += b_tree;
  uint32_t *count = reinterpret_cast<uint32_t *>(p);
  p += b_leafu;
  uint32_t *offset = reinterpret_cast<uint32_t *>(p);
  p += b_leafu;
  uint32_t *cursor = reinterpret_cast<uint32_t *>(p);
  p += b_leafu;
  uint32_t *leaf = reinterpret_cast<uint32_t *>(p);
  p += b_shot32;
  uint32_t *order = reinterpret_cast<uint32_t *>(p);
  p += b_shot32;
  double *resid = reinterpret_cast<double *>(p);

  leaf_sum_kernel<C2><<<unsigned(nleaves), kLeafThreads, 0, st>>>(psi, N, tree + (nleaves - 1));
  RQ_CUDA(cudaGetLastError());
  if (depth) upper_tree_kernel<<<1, 1024, 0, st>>>(tree, depth);
  RQ_CUDA(cudaGetLastError());
  RQ_CUDA(cudaMemsetAsync(count, 0, nleaves * sizeof(uint32_t), st));
  if (before_shots) {
    const int rc = before_shots();
    if (rc != SQ_OK) return rc;
  }
  if (u_ready) RQ_CUDA(cudaStreamWaitEvent(st, u_ready, 0));
  const unsigned sb = unsigned((shots + 255) / 256);
  shot_descend_kernel<<<sb, 256, 0, st>>>(tree, depth, u, shots, leaf, resid, count);
  RQ_CUDA(cudaGetLastError());
  count_scan_kernel<<<1, 1024, 0, st>>>(count, uint32_t(nleaves), offset, cursor);
  RQ_CUDA(cudaGetLastError());
  shot_bucket_kernel<<<sb, 256, 0, st>>>(leaf, shots, cursor, order);
  RQ_CUDA(cudaGetLastError());
  const size_t smem = (2 * size_t(kLeafAmps) - 1) * sizeof(double);
  RQ_CUDA(cudaFuncSetAttribute(leaf_sample_kernel<C2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  int sms = 0, dev = 0, per_sm = 0;
  RQ_CUDA(cudaGetDevice(&dev));
  RQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  RQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, leaf_sample_kernel<C2>, kLeafThreads, smem));
  const unsigned grid = unsigned(std::min<uint64_t>(nleaves, uint64_t(sms) * uint64_t(std::max(per_sm, 1))));
  leaf_sample_kernel<C2><<<grid, kLeafThreads, smem, st>>>(psi, N, uint32_t(nleaves), count, offset, order,
                                                           resid, out);
  RQ_CUDA(cudaGetLastError());
  return SQ_OK;
}

}  // namespace

extern "C" {

int sq_sample(sq_state *s, const double *uniforms_device, uint64_t shots, uint64_t *out_device, void *stream) {
  if (!s || (shots && (!uniforms_device || !out_device))) return fail(SQ_ERR_INVALID, "sq_sample: null pointer");
  if (shots > (uint64_t(1) << 31)) return fail(SQ_ERR_UNSUPPORTED, "sq_sample: more than 2^31 shots per call");
  auto st = static_cast<cudaStream_t>(stream);
  const int rc = sq_flush(s, stream);
  if (rc != SQ_OK || shots == 0) return rc;
  const uint32_t n = sq_state_num_qubits(s);
  if (n > uint32_t(kLeafBits) + 22) return fail(SQ_ERR_UNSUPPORTED, "sq_sample: more than 34 qubits");
  void *scr = nullptr;
  const int sc = sq_detail_state_scratch(s, sample_scratch_bytes(n, shots), &scr);
  if (sc != SQ_OK) return sc;
  if (sq_state_dtype(s) == SQ_C64)
    return sample_impl(static_cast<const float2 *>(sq_state_data(s)), n, uniforms_device, shots, out_device, scr, st);
  return sample_impl(static_cast<const double2 *>(sq_state_data(s)), n, uniforms_device, shots, out_device, scr,
                     st);
}

int sq_sample_host(sq_state *s, const double *uniforms, uint64_t shots, uint64_t *out, void *stream) {
  if (!s || (shots && (!uniforms || !out))) return fail(SQ_ERR_INVALID, "sq_sample_host: null pointer");
  if (shots > (uint64_t(1) << 31)) return fail(SQ_ERR_UNSUPPORTED, "sq_sample_host: more than 2^31 shots per call");
  auto st = static_cast<cudaStream_t>(stream);
  int rc = sq_flush(s, stream);
  if (rc != SQ_OK || shots == 0) return rc;
  const uint32_t n = sq_state_num_qubits(s);
  if (n > uint32_t(kLeafBits) + 22) return fail(SQ_ERR_UNSUPPORTED, "sq_sample_host: more than 34 qubits");
  // The state's scratch holds the uniforms and the indices, then the sampler's own scratch.
  const size_t b_u = align256(shots * sizeof(double)), b_o = align256(shots * sizeof(uint64_t));
  void *scr = nullptr;
  rc = sq_detail_state_scratch(s, b_u + b_o + sample_scratch_bytes(n, shots), &scr);
  if (rc != SQ_OK) return rc;
  char *p = static_cast<char *>(scr);
  double *du = reinterpret_cast<double *>(p);
  uint64_t *dout = reinterpret_cast<uint64_t *>(p + b_u);
  // Pinned staging (the state's, reused): the uniforms are copied into it
  // and go up on a second stream while the probability tree is built; the
  // shot phase waits for them; the indices come back through it.
  void *hs = nullptr;
  rc = sq_detail_state_host_scratch(s, std::max(shots * sizeof(double), shots * sizeof(uint64_t)), &hs);
  if (rc != SQ_OK) return rc;
  cudaStream_t cs = nullptr;
  cudaEvent_t prior = nullptr, ready = nullptr;
  struct Release {
    cudaStream_t &cs;
    cudaEvent_t &a, &b;
    ~Release() {
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
      if (cs) cudaStreamDestroy(cs);
    }
  } release{cs, prior, ready};
  RQ_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  RQ_CUDA(cudaEventCreateWithFlags(&prior, cudaEventDisableTiming));
  RQ_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  RQ_CUDA(cudaEventRecord(prior, st));  // earlier work on the state's stream
  auto upload = [&]() -> int {
    std::memcpy(hs, uniforms, shots * sizeof(double));  // while the tree kernels run
    RQ_CUDA(cudaStreamWaitEvent(cs, prior, 0));
    RQ_CUDA(cudaMemcpyAsync(du, hs, shots * sizeof(double), cudaMemcpyHostToDevice, cs));
    RQ_CUDA(cudaEventRecord(ready, cs));
    return SQ_OK;
  };
  rc = sq_state_dtype(s) == SQ_C64
           ? sample_impl(static_cast<const float2 *>(sq_state_data(s)), n, du, shots, dout, p + b_u + b_o, st,
                         ready, upload)
           : sample_impl(static_cast<const double2 *>(sq_state_data(s)), n, du, shots, dout, p + b_u + b_o, st,
                         ready, upload);
  if (rc != SQ_OK) {
    cudaStreamSynchronize(cs);
    return rc;
  }
  RQ_CUDA(cudaMemcpyAsync(hs, dout, shots * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  RQ_CUDA(cudaStreamSynchronize(st));
  std::memcpy(out, hs, shots * sizeof(uint64_t));
  return SQ_OK;
}

int sq_amplitudes(sq_state *s, const uint64_t *indices_device, uint64_t count, double *out_device, void *stream) {
  if (!s || (count && (!indices_device || !out_device))) return fail(SQ_ERR_INVALID, "sq_amplitudes: null pointer");
  auto st = static_cast<cudaStream_t>(stream);
  int rc = sq_flush(s, stream);
  if (rc != SQ_OK || count == 0) return rc;
  void *scr = nullptr;
  rc = sq_detail_state_scratch(s, 256, &scr);
  if (rc != SQ_OK) return rc;
  uint32_t *bad = static_cast<uint32_t *>(scr);
  RQ_CUDA(cudaMemsetAsync(bad, 0, sizeof(uint32_t), st));
  const uint64_t N = uint64_t(1) << sq_state_num_qubits(s);
  const unsigned grid = unsigned((count + 255) / 256);
  auto *o = reinterpret_cast<double2 *>(out_device);
  if (sq_state_dtype(s) == SQ_C64)
    amplitude_kernel<float2><<<grid, 256, 0, st>>>(static_cast<const float2 *>(sq_state_data(s)), N,
                                                   indices_device, count, o, bad);
  else
    amplitude_kernel<double2><<<grid, 256, 0, st>>>(static_cast<const double2 *>(sq_state_data(s)), N,
                                                    indices_device, count, o, bad);
  RQ_CUDA(cudaGetLastError());
  uint32_t h = 0;
  RQ_CUDA(cudaMemcpyAsync(&h, bad, sizeof(h), cudaMemcpyDeviceToHost, st));
  RQ_CUDA(cudaStreamSynchronize(st));
  if (h) return fail(SQ_ERR_INVALID, "sq_amplitudes: an index is >= 2^num_qubits (its output is 0)");
  return SQ_OK;
}

int sq_marginal_probabilities(sq_state *s, const uint32_t *qubits, uint32_t k, double *out_device, void *stream) {
  if (!s || !out_device || (k && !qubits)) return fail(SQ_ERR_INVALID, "sq_marginal_probabilities: null pointer");
  const uint32_t n = sq_state_num_qubits(s);
  if (k > n) return fail(SQ_ERR_INVALID, "sq_marginal_probabilities: more targets than qubits");
  if (k > 30) return fail(SQ_ERR_UNSUPPORTED, "sq_marginal_probabilities: more than 30 target qubits");
  MarginalParams P;
  std::memset(&P, 0, sizeof(P));
  P.n = n;
  P.k = k;
  for (uint32_t j = 0; j < k; ++j) {
    if (qubits[j] >= n) return fail(SQ_ERR_INVALID, "sq_marginal_probabilities: qubit out of range");
    const uint64_t bit = uint64_t(1) << (n - 1 - qubits[j]);
    if (P.tmask & bit) return fail(SQ_ERR_INVALID, "sq_marginal_probabilities: repeated qubit");
    P.tmask |= bit;
    P.tbit[j] = uint8_t(n - 1 - qubits[j]);
  }
  auto st = static_cast<cudaStream_t>(stream);
  int rc = sq_flush(s, stream);
  if (rc != SQ_OK) return rc;
  int sms = 0, dev = 0;
  RQ_CUDA(cudaGetDevice(&dev));
  RQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const uint64_t bins = uint64_t(1) << k, rest = uint64_t(1) << (n - k);
  // Enough (bin, chunk) items to fill the GPU; chunks of at least 2^12
  // amplitudes where the state allows.
  const uint64_t want = uint64_t(sms) * 8;
  uint32_t chunks = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>((want + bins - 1) / bins,
                                                                        std::max<uint64_t>(1, rest >> 12))));
  void *scr = nullptr;
  rc = sq_detail_state_scratch(s, bins * chunks * sizeof(double), &scr);
  if (rc != SQ_OK) return rc;
  double *partial = static_cast<double *>(scr);
  const unsigned grid = unsigned(std::min<uint64_t>(bins * chunks, uint64_t(sms) * 16));
  if (sq_state_dtype(s) == SQ_C64)
    marginal_kernel<float2><<<grid, 256, 0, st>>>(static_cast<const float2 *>(sq_state_data(s)), P, chunks, partial);
  else
    marginal_kernel<double2><<<grid, 256, 0, st>>>(static_cast<const double2 *>(sq_state_data(s)), P, chunks,
                                                    partial);
  RQ_CUDA(cudaGetLastError());
  marginal_finalize_kernel<<<unsigned((bins + 255) / 256), 256, 0, st>>>(partial, bins, chunks, out_device);
  RQ_CUDA(cudaGetLastError());
  return SQ_OK;
}

int sq_state_distance(sq_state *a, sq_state *b, double *max_abs, double *one_minus_fidelity, void *stream) {
  if (!a || !b || !max_abs || !one_minus_fidelity) return fail(SQ_ERR_INVALID, "sq_state_distance: null pointer");
  const uint32_t n = sq_state_num_qubits(a);
  if (sq_state_num_qubits(b) != n) return fail(SQ_ERR_INVALID, "sq_state_distance: states of different size");
  auto st = static_cast<cudaStream_t>(stream);
  int rc = sq_flush(a, stream);
  if (rc == SQ_OK) rc = sq_flush(b, stream);
  if (rc != SQ_OK) return rc;
  int sms = 0, dev = 0;
  RQ_CUDA(cudaGetDevice(&dev));
  RQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const uint64_t N = uint64_t(1) << n;
  const unsigned blocks = unsigned(std::max<uint64_t>(1, std::min<uint64_t>((N + 255) / 256, uint64_t(sms) * 4)));
  void *scr = nullptr;
  rc = sq_detail_state_scratch(a, size_t(blocks) * 5 * sizeof(double), &scr);
  if (rc != SQ_OK) return rc;
  double *part = static_cast<double *>(scr);
  const bool a64 = sq_state_dtype(a) == SQ_C64, b64 = sq_state_dtype(b) == SQ_C64;
  const void *pa = sq_state_data(a), *pb = sq_state_data(b);
  if (!a64 && !b64)
    distance_kernel<<<blocks, 256, 0, st>>>(static_cast<const double2 *>(pa), static_cast<const double2 *>(pb), N, part);
  else if (!a64 && b64)
    distance_kernel<<<blocks, 256, 0, st>>>(static_cast<const double2 *>(pa), static_cast<const float2 *>(pb), N, part);
  else if (a64 && !b64)
    distance_kernel<<<blocks, 256, 0, st>>>(static_cast<const float2 *>(pa), static_cast<const double2 *>(pb), N, part);
  else
    distance_kernel<<<blocks, 256, 0, st>>>(static_cast<const float2 *>(pa), static_cast<const float2 *>(pb), N, part);
  RQ_CUDA(cudaGetLastError());
  std::vector<double> h(size_t(blocks) * 5);
  RQ_CUDA(cudaMemcpyAsync(h.data(), part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  RQ_CUDA(cudaStreamSynchronize(st));
  double mx = 0, re = 0, im = 0, na = 0, nb = 0;
  for (unsigned i = 0; i < blocks; ++i) {
    mx = std::max(mx, h[5 * i]);
    re += h[5 * i + 1];
    im += h[5 * i + 2];
    na += h[5 * i + 3];
    nb += h[5 * i + 4];
  }
  *max_abs = mx;
  *one_minus_fidelity = (na > 0 && nb > 0) ? 1.0 - (re * re + im * im) / (na * nb) : 1.0;
  return SQ_OK;
}

}  // extern "C"

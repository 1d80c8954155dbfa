// Batched circuits in one persistent launch (sm_100a).
//
// Thousands of small circuits of uneven qubit counts: each CTA takes the next
// circuit from an atomic work queue (circuits are sorted largest first), runs
// all of the circuit's planned sweeps itself and reduces the circuit's
// Pauli-sum energy.  A circuit that fits one tile (n <= M) lives in shared
// memory from |0...0> to its energy and never touches HBM (unless its state
// is asked for); a larger circuit sweeps its own state in HBM tile by tile.
// No CTA ever waits on another: the only cross-CTA interaction is one
// atomicAdd per circuit on the work counter.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "adjoint_kernels.cuh"
#include "jit_batch.cuh"
#include "reduce_kernels.cuh"
#include "sweep_kernels.cuh"

namespace sq {

// Phases of one packed sweep on one tile held in shared memory.  Threads
// with tid >= 2^(m-4) only take part in the barriers.
template <typename Real>
__device__ __forceinline__ void batch_tile_phases(typename Vec2<Real>::T *tile, const PackedSweep &ps,
                                                  const SweepPhase *ph, const SweepOp *ops,
                                                  const typename Vec2<Real>::T *coef,
                                                  uint64_t gbase) {
  using C2 = typename Vec2<Real>::T;
  const uint32_t tid = threadIdx.x;
  const uint32_t nthr = 1u << (ps.h.m - kRegBits);
  for (uint32_t p = 0; p < ps.h.nphases; ++p) {
    if (tid < nthr) {
      const SweepPhase P = ph[p];
      uint32_t jb = tid;
#pragma unroll
      for (int b = 0; b < kRegBits; ++b) jb = uint32_t(insert_zero(jb, P.reg[b]));
      const uint32_t sb = swz<Real>(jb);
      const uint32_t w0 = swz<Real>(1u << P.reg[0]), w1 = swz<Real>(1u << P.reg[1]);
      const uint32_t w2 = swz<Real>(1u << P.reg[2]), w3 = swz<Real>(1u << P.reg[3]);
      Amps<Real> A;
#pragma unroll
      for (int ri = 0; ri < kRegAmps; ++ri) {
        const C2 v = tile[sb ^ ((ri & 1) ? w0 : 0) ^ ((ri & 2) ? w1 : 0) ^ ((ri & 4) ? w2 : 0) ^
                          ((ri & 8) ? w3 : 0)];
        A.re[ri] = v.x;
        A.im[ri] = v.y;
      }
      for (uint32_t o = P.op_begin; o < P.op_end; ++o) apply_op<Real, kRegAmps>(A, coef, ops[o], gbase, jb);
#pragma unroll
      for (int ri = 0; ri < kRegAmps; ++ri) {
        C2 v;
        v.x = A.re[ri];
        v.y = A.im[ri];
        tile[sb ^ ((ri & 1) ? w0 : 0) ^ ((ri & 2) ? w1 : 0) ^ ((ri & 4) ? w2 : 0) ^
             ((ri & 8) ? w3 : 0)] = v;
      }
    }
    __syncthreads();
  }
}

// sum_groups sum_pairs of the Pauli expectation (reduce_kernels.cuh) over a
// state read through `amp(i)`; result valid in thread 0.  Each thread issues
// the loads of U pairs before using any of them, so a state streamed from
// HBM by one CTA keeps U times more reads in flight.
template <typename Real, class AmpFn>
__device__ __forceinline__ double batch_energy(const PauliParams &H, uint32_t n, AmpFn amp) {
  using C2 = typename Vec2<Real>::T;
  constexpr int U = 4;
  double acc = 0.0;
  const uint64_t step = uint64_t(blockDim.x) * U;
  for (uint32_t gi = 0; gi < H.ngroups; ++gi) {
    const PauliGroup &G = H.g[gi];
    if (G.x == 0) {
      const uint64_t N = uint64_t(1) << n;
      for (uint64_t i0 = threadIdx.x; i0 < N; i0 += step) {
        C2 a[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const uint64_t i = i0 + uint64_t(u) * blockDim.x;
          a[u] = amp(i < N ? i : 0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const uint64_t i = i0 + uint64_t(u) * blockDim.x;
          if (i >= N) continue;
          const double q = double(a[u].x) * double(a[u].x) + double(a[u].y) * double(a[u].y);
          double w = 0.0;
          for (uint32_t t = G.t0; t < G.t1; ++t) w += (__popcll(i & H.zy[t]) & 1) ? -H.f[t] : H.f[t];
          acc = fma(q, w, acc);
        }
      }
    } else {
      const uint32_t hb = 63 - __clzll(G.x);
      const uint64_t NP = uint64_t(1) << (n - 1);
      for (uint64_t h0 = threadIdx.x; h0 < NP; h0 += step) {
        C2 a[U], b[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const uint64_t hh = h0 + uint64_t(u) * blockDim.x;
          const uint64_t i = insert_zero(hh < NP ? hh : 0, hb);
          a[u] = amp(i);
          b[u] = amp(i ^ G.x);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const uint64_t hh = h0 + uint64_t(u) * blockDim.x;
          if (hh >= NP) continue;
          const uint64_t i = insert_zero(hh, hb);
          const double zr = double(a[u].x) * double(b[u].x) + double(a[u].y) * double(b[u].y);
          const double zi = double(a[u].x) * double(b[u].y) - double(a[u].y) * double(b[u].x);
          const double q = 2.0 * (G.odd ? zi : zr);
          double w = 0.0;
          for (uint32_t t = G.t0; t < G.t1; ++t) w += (__popcll(i & H.zy[t]) & 1) ? -H.f[t] : H.f[t];
          acc = fma(q, w, acc);
        }
      }
    }
  }
  return block_sum(acc);
}

// Dynamic shared memory: two tiles (2 x 2^M amplitudes) | coefficients
// (kMaxCoef) | high-bit table (2^(M-3) u64).  A state streamed through tiles
// double-buffers them: tile t+1 arrives by cp.async while tile t is worked.
template <typename Real, int M>
__global__ void __launch_bounds__(1 << (M - kRegBits), 1)
    batch_kernel(typename Vec2<Real>::T *__restrict__ pool, const __grid_constant__ BatchParams B) {
  using C2 = typename Vec2<Real>::T;
  constexpr uint32_t TS = 1u << M;
  constexpr int NT = 1 << (M - kRegBits);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *tile = reinterpret_cast<C2 *>(smem_raw);
  C2 *coef = tile + 2 * TS;
  uint64_t *hitab = reinterpret_cast<uint64_t *>(coef + kMaxCoef);
  __shared__ uint32_t s_next;
  const uint32_t tid = threadIdx.x;

  for (;;) {
    if (tid == 0) s_next = atomicAdd(B.counter, 1u);
    __syncthreads();
    const uint32_t c = s_next;
    __syncthreads();
    if (c >= B.ncircuits) break;
    const BatchCircuit C = B.circuits[c];
    const uint32_t n = C.n;
    C2 *psi = pool + C.state_off;
    const bool resident = n <= uint32_t(M);
    const uint64_t N = uint64_t(1) << n;
    // |0...0>
    if (resident) {
      for (uint32_t j = tid; j < uint32_t(N); j += NT) {
        C2 v;
        v.x = Real(j == 0 ? 1 : 0);
        v.y = Real(0);
        tile[swz<Real>(j)] = v;
      }
    } else {
      for (uint64_t j = tid; j < N; j += NT) {
        C2 v;
        v.x = Real(j == 0 ? 1 : 0);
        v.y = Real(0);
        psi[j] = v;
      }
    }
    __syncthreads();
    const unsigned char *rec = B.plans + C.plan_off;
    for (uint32_t s = 0; s < C.nsweeps; ++s) {
      const PackedSweep &ps = *reinterpret_cast<const PackedSweep *>(rec);
      const SweepPhase *ph = reinterpret_cast<const SweepPhase *>(rec + ps.phase_off);
      const SweepOp *ops = reinterpret_cast<const SweepOp *>(rec + ps.op_off);
      const C2 *gcoef = reinterpret_cast<const C2 *>(rec + ps.coef_off);
      for (uint32_t i = tid; i < ps.h.ncoef; i += NT) coef[i] = gcoef[i];
      const uint32_t m = ps.h.m, l = ps.h.l;
      if (!resident)
        for (uint32_t cc = tid; cc < (1u << (m - l)); cc += NT) {
          uint64_t a = 0;
          for (uint32_t i = 0; i < m - l; ++i)
            if ((cc >> i) & 1) a |= uint64_t(1) << ps.h.hi[i];
          hitab[cc] = a;
        }
      __syncthreads();
      if (resident) {
        // The tile is the whole state in index order: tile base 0.
        batch_tile_phases<Real>(tile, ps, ph, ops, coef, 0);
      } else {
        const uint32_t lowmask = (1u << l) - 1u, tsize = 1u << m;
        auto prefetch = [&](uint64_t t, C2 *dst) {
          const uint64_t gb = tile_base(t, ps.h);
          for (uint32_t j = tid; j < tsize; j += NT)
            cp_async<sizeof(C2)>(dst + swz<Real>(j), psi + (gb | hitab[j >> l] | (j & lowmask)));
        };
        prefetch(0, tile);
        cp_async_commit();
        for (uint64_t t = 0; t < ps.h.num_tiles; ++t) {
          C2 *cur = tile + (t & 1) * TS;
          // The other buffer's previous tile was written back before the
          // barrier that ended the last iteration.
          if (t + 1 < ps.h.num_tiles) prefetch(t + 1, tile + ((t + 1) & 1) * TS);
          cp_async_commit();
          cp_async_wait_prev();
          __syncthreads();
          const uint64_t gbase = tile_base(t, ps.h);
          batch_tile_phases<Real>(cur, ps, ph, ops, coef, gbase);
          for (uint32_t j = tid; j < tsize; j += NT)
            psi[gbase | hitab[j >> l] | (j & lowmask)] = cur[swz<Real>(j)];
          __syncthreads();
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
      }
      rec += ps.bytes;
    }
    const PauliParams &H = B.hams[C.ham];
    if (!C.defer) {
      double e;
      if (resident)
        e = batch_energy<Real>(H, n, [&](uint64_t i) { return tile[swz<Real>(uint32_t(i))]; });
      else
        e = batch_energy<Real>(H, n, [&](uint64_t i) { return psi[i]; });
      if (tid == 0) B.energies[c] = e;
    }
    if (resident && C.keep)
      for (uint32_t j = tid; j < uint32_t(N); j += NT) psi[j] = tile[swz<Real>(j)];
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Energies of the streamed (pool-resident) circuits of a batch, after
// batch_kernel.  Work item w covers deferred circuit item_k[w] and chunk
// item_j[w] of its index range (kEnergyChunk pairs of every Pauli group, or
// 2 kEnergyChunk amplitudes of a diagonal group), so a large state is shared
// by many blocks at once and stays in L2 across its groups, while a small
// one is one block's work.  partials[w] receives the block's sum;
// batch_energy_finalize adds a circuit's items in order.
// ---------------------------------------------------------------------------
// Chunks of 2^10 pairs: a circuit of n qubits has 2^(n-11) items, and the
// blocks running at any one time (items in index order) cover a few states
// at most, which then stay in L2 across all of their Pauli groups (with
// larger chunks the concurrent items spanned tens of 2^20-amplitude states,
// more than L2 holds, and every group re-read its state from HBM).
constexpr uint32_t kEnergyChunkBits = 10;

template <typename Real>
__global__ void __launch_bounds__(kReduceThreads)
    batch_energy_grid(const typename Vec2<Real>::T *__restrict__ pool, const __grid_constant__ BatchParams B,
                      const uint32_t *__restrict__ deferred, const uint32_t *__restrict__ item_off, uint32_t ndef,
                      uint32_t nitems, double *__restrict__ partials) {
  using C2 = typename Vec2<Real>::T;
  constexpr int U = 4;
  for (uint32_t w = blockIdx.x; w < nitems; w += gridDim.x) {
    // Deferred circuit k with item_off[k] <= w < item_off[k + 1].
    uint32_t lo_k = 0, hi_k = ndef;
    while (hi_k - lo_k > 1) {
      const uint32_t mid = (lo_k + hi_k) / 2;
      if (item_off[mid] <= w) lo_k = mid;
      else hi_k = mid;
    }
    const BatchCircuit &C = B.circuits[deferred[lo_k]];
    const PauliParams &H = B.hams[C.ham];
    const C2 *psi = pool + C.state_off;
    const uint32_t n = C.n;
    const uint64_t j = w - item_off[lo_k];
    double acc = 0.0;
    for (uint32_t gi = 0; gi < H.ngroups; ++gi) {
      const PauliGroup &G = H.g[gi];
      if (G.x == 0) {
        const uint64_t N = uint64_t(1) << n;
        const uint64_t lo = j << (kEnergyChunkBits + 1), hi = lo + (uint64_t(2) << kEnergyChunkBits);
        const uint64_t end = hi < N ? hi : N;
        for (uint64_t i0 = lo + threadIdx.x; i0 < end; i0 += uint64_t(blockDim.x) * U) {
          C2 a[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const uint64_t i = i0 + uint64_t(u) * blockDim.x;
            a[u] = psi[i < end ? i : lo];
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const uint64_t i = i0 + uint64_t(u) * blockDim.x;
            if (i >= end) continue;
            const double q = double(a[u].x) * double(a[u].x) + double(a[u].y) * double(a[u].y);
            double wt = 0.0;
            for (uint32_t t = G.t0; t < G.t1; ++t) wt += (__popcll(i & H.zy[t]) & 1) ? -H.f[t] : H.f[t];
            acc = fma(q, wt, acc);
          }
        }
      } else {
        const uint32_t hb = 63 - __clzll(G.x);
        const uint64_t NP = uint64_t(1) << (n - 1);
        const uint64_t lo = j << kEnergyChunkBits, hi = lo + (uint64_t(1) << kEnergyChunkBits);
        const uint64_t end = hi < NP ? hi : NP;
        for (uint64_t h0 = lo + threadIdx.x; h0 < end; h0 += uint64_t(blockDim.x) * U) {
          C2 a[U], b[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const uint64_t hh = h0 + uint64_t(u) * blockDim.x;
            const uint64_t i = insert_zero(hh < end ? hh : lo, hb);
            a[u] = psi[i];
            b[u] = psi[i ^ G.x];
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const uint64_t hh = h0 + uint64_t(u) * blockDim.x;
            if (hh >= end) continue;
            const uint64_t i = insert_zero(hh, hb);
            const double zr = double(a[u].x) * double(b[u].x) + double(a[u].y) * double(b[u].y);
            const double zi = double(a[u].x) * double(b[u].y) - double(a[u].y) * double(b[u].x);
            const double q = 2.0 * (G.odd ? zi : zr);
            double wt = 0.0;
            for (uint32_t t = G.t0; t < G.t1; ++t) wt += (__popcll(i & H.zy[t]) & 1) ? -H.f[t] : H.f[t];
            acc = fma(q, wt, acc);
          }
        }
      }
    }
    const double s = block_sum(acc);
    if (threadIdx.x == 0) partials[w] = s;
  }
}

// energies[deferred[k]] = sum of partials[item_off[k] .. item_off[k+1]), in
// order.  One block per deferred circuit.
static __global__ void __launch_bounds__(kReduceThreads)
    batch_energy_finalize(const double *__restrict__ partials, const uint32_t *__restrict__ item_off,
                          const uint32_t *__restrict__ deferred, double *__restrict__ energies) {
  const uint32_t k = blockIdx.x;
  double v = 0.0;
  for (uint32_t i = item_off[k] + threadIdx.x; i < item_off[k + 1]; i += blockDim.x) v += partials[i];
  v = block_sum(v);
  if (threadIdx.x == 0) energies[deferred[k]] = v;
}

// |0...0> in each of the K states of 2^n amplitudes that lie back to back
// from psi (a structure group of a batch, before its multi-state sweeps);
// total = K 2^n.
template <typename Real>
__global__ void batch_group_init(typename Vec2<Real>::T *__restrict__ psi, uint64_t total, uint32_t n) {
  const uint64_t mask = (uint64_t(1) << n) - 1;
  for (uint64_t j = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; j < total;
       j += uint64_t(gridDim.x) * blockDim.x) {
    typename Vec2<Real>::T v;
    v.x = Real((j & mask) == 0 ? 1 : 0);
    v.y = Real(0);
    psi[j] = v;
  }
}

// ---------------------------------------------------------------------------
// Batched adjoint gradients: one circuit per CTA (work queue as above).  For
// each circuit: forward sweeps on psi, lambda = H psi with E = Re <psi|lambda>,
// then the reverse two-state sweeps that un-compute both states and
// accumulate <lambda| K |phi> for every parametrised angle occurrence
// (adjoint_kernels.cuh).  A circuit of n <= M qubits keeps psi and lambda in
// shared memory throughout; a larger one keeps them in the state pool and
// streams tiles.  Inner products are summed per warp (shuffles), then over
// warps in a fixed order, into occ[occ_off + occurrence] (one CTA owns a
// circuit: no atomics).
// ---------------------------------------------------------------------------

// Two-state phases of one packed reverse sweep on a (phi, lambda) tile pair
// in shared memory.  2^(m-3) threads take part; the others only meet the
// barriers.
template <typename Real>
__device__ __forceinline__ void batch_adjoint_phases(typename Vec2<Real>::T *ft, typename Vec2<Real>::T *lt,
                                                     const PackedSweep &ps, const SweepPhase *ph,
                                                     const SweepOp *ops, const typename Vec2<Real>::T *coef,
                                                     uint64_t gbase, double2 *acc) {
  using C2 = typename Vec2<Real>::T;
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t nthr = 1u << (ps.h.m - kAdjRegBits);
  const unsigned mask = nthr >= 32 ? 0xffffffffu : ((1u << nthr) - 1u);
  for (uint32_t p = 0; p < ps.h.nphases; ++p) {
    if (tid < nthr) {
      const SweepPhase P = ph[p];
      uint32_t jb = tid;
#pragma unroll
      for (int b = 0; b < kAdjRegBits; ++b) jb = uint32_t(insert_zero(jb, P.reg[b]));
      const uint32_t sb = swz<Real>(jb);
      const uint32_t w0 = swz<Real>(1u << P.reg[0]), w1 = swz<Real>(1u << P.reg[1]);
      const uint32_t w2 = swz<Real>(1u << P.reg[2]);
      Amps<Real, kAdjAmps> F, G;
#pragma unroll
      for (int ri = 0; ri < kAdjAmps; ++ri) {
        const uint32_t s = sb ^ ((ri & 1) ? w0 : 0) ^ ((ri & 2) ? w1 : 0) ^ ((ri & 4) ? w2 : 0);
        const C2 a = ft[s], b = lt[s];
        F.re[ri] = a.x;
        F.im[ri] = a.y;
        G.re[ri] = b.x;
        G.im[ri] = b.y;
      }
      for (uint32_t o = P.op_begin; o < P.op_end; ++o) {
        const SweepOp &op = ops[o];
        if (op.kind == kSwInnerDiag || op.kind == kSwInnerDense) {
          double sr = 0.0, si = 0.0;
          inner_op<Real>(F, G, coef, op, gbase, jb, sr, si);
          for (uint32_t off = (nthr >= 32 ? 16u : nthr / 2); off > 0; off >>= 1) {
            sr += __shfl_xor_sync(mask, sr, off);
            si += __shfl_xor_sync(mask, si, off);
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
        ft[s] = a;
        lt[s] = b;
      }
    }
    __syncthreads();
  }
}

// Dynamic shared memory: two (phi tile | lambda tile) buffers (2^M amplitudes
// each) | coefficients (kMaxCoef) | high-bit table (2^(M-L) u64) |
// inner-product slots (warps x kMaxInner double2).  2^(M-3) threads.  States
// streamed from the pool double-buffer their tiles: tile t+1 arrives by
// cp.async while tile t is worked.
template <typename Real, int M>
__global__ void __launch_bounds__(1 << (M - kAdjRegBits), 1)
    batch_adjoint_kernel(typename Vec2<Real>::T *__restrict__ pool, const __grid_constant__ BatchParams B,
                         double2 *__restrict__ occ) {
  using C2 = typename Vec2<Real>::T;
  constexpr uint32_t TS = 1u << M;
  constexpr int NT = 1 << (M - kAdjRegBits);
  constexpr int NW = (NT + 31) / 32;
  constexpr int L = sweep_low_bits(M);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *ft = reinterpret_cast<C2 *>(smem_raw);  // buffer b: phi at ft + 2 b TS, lambda after it
  C2 *lt = ft + TS;
  C2 *coef = ft + 4 * TS;
  uint64_t *hitab = reinterpret_cast<uint64_t *>(coef + kMaxCoef);
  double2 *acc = reinterpret_cast<double2 *>(hitab + (1u << (M - L)));
  __shared__ uint32_t s_next;
  const uint32_t tid = threadIdx.x;

  for (;;) {
    if (tid == 0) s_next = atomicAdd(B.counter, 1u);
    __syncthreads();
    const uint32_t c = s_next;
    __syncthreads();
    if (c >= B.ncircuits) break;
    const BatchCircuit C = B.circuits[c];
    const uint32_t n = C.n;
    C2 *psi = pool + C.state_off;
    C2 *lam = pool + C.lam_off;
    const bool resident = n <= uint32_t(M);
    const uint64_t N = uint64_t(1) << n;
    // |0...0>
    for (uint64_t j = tid; j < N; j += NT) {
      C2 v;
      v.x = Real(j == 0 ? 1 : 0);
      v.y = Real(0);
      if (resident)
        ft[swz<Real>(uint32_t(j))] = v;
      else
        psi[j] = v;
    }
    __syncthreads();
    const unsigned char *rec = B.plans + C.plan_off;
    // Forward sweeps (one state).
    for (uint32_t s = 0; s < C.nsweeps; ++s) {
      const PackedSweep &ps = *reinterpret_cast<const PackedSweep *>(rec);
      const SweepPhase *ph = reinterpret_cast<const SweepPhase *>(rec + ps.phase_off);
      const SweepOp *ops = reinterpret_cast<const SweepOp *>(rec + ps.op_off);
      const C2 *gcoef = reinterpret_cast<const C2 *>(rec + ps.coef_off);
      for (uint32_t i = tid; i < ps.h.ncoef; i += NT) coef[i] = gcoef[i];
      const uint32_t m = ps.h.m, l = ps.h.l;
      if (!resident)
        for (uint32_t cc = tid; cc < (1u << (m - l)); cc += NT) {
          uint64_t a = 0;
          for (uint32_t i = 0; i < m - l; ++i)
            if ((cc >> i) & 1) a |= uint64_t(1) << ps.h.hi[i];
          hitab[cc] = a;
        }
      __syncthreads();
      // One call site per phase routine (a resident state is one tile at base 0).
      const uint32_t lowmask = (1u << l) - 1u, tsize = 1u << m;
      const uint64_t ntiles = resident ? 1 : ps.h.num_tiles;
      auto prefetch1 = [&](uint64_t t, C2 *dst) {
        const uint64_t gb = tile_base(t, ps.h);
        for (uint32_t j = tid; j < tsize; j += NT)
          cp_async<sizeof(C2)>(dst + swz<Real>(j), psi + (gb | hitab[j >> l] | (j & lowmask)));
      };
      if (!resident) {
        prefetch1(0, ft);
        cp_async_commit();
      }
      for (uint64_t t = 0; t < ntiles; ++t) {
        C2 *cur = ft + (t & 1) * 2 * TS;
        const uint64_t gbase = resident ? 0 : tile_base(t, ps.h);
        if (!resident) {
          if (t + 1 < ntiles) prefetch1(t + 1, ft + ((t + 1) & 1) * 2 * TS);
          cp_async_commit();
          cp_async_wait_prev();
          __syncthreads();
        }
        batch_tile_phases<Real>(cur, ps, ph, ops, coef, gbase);
        if (!resident) {
          for (uint32_t j = tid; j < tsize; j += NT) psi[gbase | hitab[j >> l] | (j & lowmask)] = cur[swz<Real>(j)];
          __syncthreads();
        }
      }
      if (!resident) asm volatile("cp.async.wait_all;\n" ::: "memory");
      rec += ps.bytes;
    }
    // lambda = H psi, E = Re <psi|lambda>.
    const PauliParams &H = B.hams[C.ham];
    double e;
    if (resident)
      e = batch_pauli_apply<Real>(
          H, n, [&](uint64_t i) { return ft[swz<Real>(uint32_t(i))]; },
          [&](uint64_t i, const C2 &v) { lt[swz<Real>(uint32_t(i))] = v; });
    else
      e = batch_pauli_apply<Real>(
          H, n, [&](uint64_t i) { return psi[i]; }, [&](uint64_t i, const C2 &v) { lam[i] = v; });
    e = block_sum(e);
    if (tid == 0) B.energies[c] = e;
    __syncthreads();
    // Reverse two-state sweeps.
    for (uint32_t s = 0; s < C.nrev; ++s) {
      const PackedSweep &ps = *reinterpret_cast<const PackedSweep *>(rec);
      const SweepPhase *ph = reinterpret_cast<const SweepPhase *>(rec + ps.phase_off);
      const SweepOp *ops = reinterpret_cast<const SweepOp *>(rec + ps.op_off);
      const C2 *gcoef = reinterpret_cast<const C2 *>(rec + ps.coef_off);
      const uint32_t *inner = ps.inner_off ? reinterpret_cast<const uint32_t *>(rec + ps.inner_off) : nullptr;
      for (uint32_t i = tid; i < ps.h.ncoef; i += NT) coef[i] = gcoef[i];
      for (uint32_t i = tid; i < NW * kMaxInner; i += NT) acc[i] = make_double2(0.0, 0.0);
      const uint32_t m = ps.h.m, l = ps.h.l;
      if (!resident)
        for (uint32_t cc = tid; cc < (1u << (m - l)); cc += NT) {
          uint64_t a = 0;
          for (uint32_t i = 0; i < m - l; ++i)
            if ((cc >> i) & 1) a |= uint64_t(1) << ps.h.hi[i];
          hitab[cc] = a;
        }
      __syncthreads();
      const uint32_t lowmask = (1u << l) - 1u, tsize = 1u << m;
      const uint64_t ntiles = resident ? 1 : ps.h.num_tiles;
      auto prefetch2 = [&](uint64_t t, C2 *dst) {
        const uint64_t gb = tile_base(t, ps.h);
        for (uint32_t j = tid; j < tsize; j += NT) {
          const uint64_t g = gb | hitab[j >> l] | (j & lowmask);
          cp_async<sizeof(C2)>(dst + swz<Real>(j), psi + g);
          cp_async<sizeof(C2)>(dst + TS + swz<Real>(j), lam + g);
        }
      };
      if (!resident) {
        prefetch2(0, ft);
        cp_async_commit();
      }
      for (uint64_t t = 0; t < ntiles; ++t) {
        C2 *cf = ft + (t & 1) * 2 * TS, *cl = cf + TS;
        const uint64_t gbase = resident ? 0 : tile_base(t, ps.h);
        if (!resident) {
          if (t + 1 < ntiles) prefetch2(t + 1, ft + ((t + 1) & 1) * 2 * TS);
          cp_async_commit();
          cp_async_wait_prev();
          __syncthreads();
        }
        batch_adjoint_phases<Real>(cf, cl, ps, ph, ops, coef, gbase, acc);
        if (!resident) {
          for (uint32_t j = tid; j < tsize; j += NT) {
            const uint64_t g = gbase | hitab[j >> l] | (j & lowmask);
            psi[g] = cf[swz<Real>(j)];
            lam[g] = cl[swz<Real>(j)];
          }
          __syncthreads();
        }
      }
      if (!resident) asm volatile("cp.async.wait_all;\n" ::: "memory");
      if (inner && tid < inner[0]) {
        double r = 0.0, i = 0.0;
        for (int w = 0; w < NW; ++w) {
          r += acc[w * kMaxInner + tid].x;
          i += acc[w * kMaxInner + tid].y;
        }
        double2 &o = occ[C.occ_off + inner[1 + tid]];
        o.x += r;
        o.y += i;
      }
      __syncthreads();
      rec += ps.bytes;
    }
  }
}

}  // namespace sq

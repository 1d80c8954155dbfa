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

#include "reduce_kernels.cuh"
#include "sweep_kernels.cuh"

namespace sq {

// Device table entry of one circuit.
struct BatchCircuit {
  uint32_t n;          // qubits (>= 4)
  uint32_t nsweeps;
  uint32_t ham;        // Hamiltonian index
  uint32_t keep;       // 1: leave the final state in the state pool
  uint64_t state_off;  // amplitude offset of its state in the pool
  uint64_t plan_off;   // byte offset of its first packed sweep in the plan pool
};

// A packed sweep: this header, then nphases SweepPhase, then nops SweepOp,
// then ncoef complex coefficients of the state's precision; `bytes` is the
// 16-byte-aligned size of the whole record.
struct PackedSweep {
  SweepHeader h;
  uint32_t nops;
  uint32_t bytes;
  uint32_t phase_off, op_off, coef_off;  // byte offsets from the record start
  uint32_t pad;
};

struct BatchParams {
  const BatchCircuit *circuits;
  const unsigned char *plans;
  const PauliParams *hams;
  uint32_t ncircuits;
  uint32_t pad;
  unsigned int *counter;  // work queue head (zeroed before the launch)
  double *energies;       // one per circuit
};

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
// state read through `amp(i)`; result valid in thread 0.
template <typename Real, class AmpFn>
__device__ __forceinline__ double batch_energy(const PauliParams &H, uint32_t n, AmpFn amp) {
  double acc = 0.0;
  for (uint32_t gi = 0; gi < H.ngroups; ++gi) {
    const PauliGroup &G = H.g[gi];
    if (G.x == 0) {
      for (uint64_t i = threadIdx.x; i < (uint64_t(1) << n); i += blockDim.x) {
        const auto a = amp(i);
        const double q = double(a.x) * double(a.x) + double(a.y) * double(a.y);
        double w = 0.0;
        for (uint32_t t = G.t0; t < G.t1; ++t) w += (__popcll(i & H.zy[t]) & 1) ? -H.f[t] : H.f[t];
        acc = fma(q, w, acc);
      }
    } else {
      const uint32_t hb = 63 - __clzll(G.x);
      for (uint64_t hh = threadIdx.x; hh < (uint64_t(1) << (n - 1)); hh += blockDim.x) {
        const uint64_t i = insert_zero(hh, hb), j = i ^ G.x;
        const auto a = amp(i), b = amp(j);
        const double zr = double(a.x) * double(b.x) + double(a.y) * double(b.y);
        const double zi = double(a.x) * double(b.y) - double(a.y) * double(b.x);
        const double q = 2.0 * (G.odd ? zi : zr);
        double w = 0.0;
        for (uint32_t t = G.t0; t < G.t1; ++t) w += (__popcll(i & H.zy[t]) & 1) ? -H.f[t] : H.f[t];
        acc = fma(q, w, acc);
      }
    }
  }
  return block_sum(acc);
}

// Dynamic shared memory: tile (2^M amplitudes) | coefficients (kMaxCoef) |
// high-bit table (2^(M-L) u64).
template <typename Real, int M>
__global__ void __launch_bounds__(1 << (M - kRegBits), 1)
    batch_kernel(typename Vec2<Real>::T *__restrict__ pool, const __grid_constant__ BatchParams B) {
  using C2 = typename Vec2<Real>::T;
  constexpr uint32_t TS = 1u << M;
  constexpr int NT = 1 << (M - kRegBits);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *tile = reinterpret_cast<C2 *>(smem_raw);
  C2 *coef = tile + TS;
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
        for (uint64_t t = 0; t < ps.h.num_tiles; ++t) {
          const uint64_t gbase = tile_base(t, ps.h);
          for (uint32_t j = tid; j < tsize; j += NT)
            tile[swz<Real>(j)] = psi[gbase | hitab[j >> l] | (j & lowmask)];
          __syncthreads();
          batch_tile_phases<Real>(tile, ps, ph, ops, coef, gbase);
          for (uint32_t j = tid; j < tsize; j += NT)
            psi[gbase | hitab[j >> l] | (j & lowmask)] = tile[swz<Real>(j)];
          __syncthreads();
        }
      }
      rec += ps.bytes;
    }
    const PauliParams &H = B.hams[C.ham];
    double e;
    if (resident)
      e = batch_energy<Real>(H, n, [&](uint64_t i) { return tile[swz<Real>(uint32_t(i))]; });
    else
      e = batch_energy<Real>(H, n, [&](uint64_t i) { return psi[i]; });
    if (tid == 0) B.energies[c] = e;
    if (resident && C.keep)
      for (uint32_t j = tid; j < uint32_t(N); j += NT) psi[j] = tile[swz<Real>(j)];
    __syncthreads();
  }
}

}  // namespace sq

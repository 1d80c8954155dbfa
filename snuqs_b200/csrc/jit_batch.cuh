// Batch types and the building blocks of the JIT-specialised batched-gradient
// kernel (snuqs_b200/csrc/jit.cu generates it for batches whose circuits all
// share one plan structure, e.g. many parameter sets of one circuit).  Also
// compiled into the library itself (batch_kernels.cuh includes it).
#pragma once
#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stdint.h>

#include "reduce_kernels.cuh"
#include "sweep_kernels.cuh"
#endif

namespace sq {

// Device table entry of one circuit.
struct BatchCircuit {
  uint32_t n;          // qubits (>= 4)
  uint32_t nsweeps;    // forward sweeps
  uint32_t ham;        // Hamiltonian index
  uint32_t keep;       // 1: leave the final state in the state pool
  uint64_t state_off;  // amplitude offset of its state in the pool
  uint64_t plan_off;   // byte offset of its first packed sweep in the plan pool
  // Gradient runs only: the reverse (two-state) sweeps follow the forward
  // ones in the plan pool; lambda's pool offset (n > tile bits); offset of the
  // circuit's parameter-occurrence inner products in the output array.
  uint32_t nrev;
  uint32_t defer;  // energy runs: 1 = the energy is left to batch_energy_grid (state in the pool)
  uint64_t lam_off;
  uint64_t occ_off;
};

// A packed sweep: this header, then nphases SweepPhase, then nops SweepOp,
// then ncoef complex coefficients of the state's precision; `bytes` is the
// 16-byte-aligned size of the whole record.
struct PackedSweep {
  SweepHeader h;
  uint32_t nops;
  uint32_t bytes;
  uint32_t phase_off, op_off, coef_off;  // byte offsets from the record start
  // Reverse sweeps of a gradient run: byte offset of a uint32 array
  // [nslots, occurrence of slot 0, ...] (0 when the sweep has no inner ops).
  uint32_t inner_off;
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

// lambda = H psi over a state read through psi_at(i) and written through
// lam_set(i, v); returns this thread's share of Re <psi|lambda>.  Group g
// contributes (sum_t f_t (-1)^popc(i & zy_t)) * (odd_g ? -i : 1) * psi[i ^ x_g]
// (PauliParams stores w_t (-1)^(ny_t / 2) in f and ny_t mod 2 in odd).
template <typename Real, class PsiAt, class LamSet>
__device__ __forceinline__ double batch_pauli_apply(const PauliParams &H, uint32_t n, PsiAt psi_at,
                                                    LamSet lam_set) {
  using C2 = typename Vec2<Real>::T;
  double e = 0.0;
  for (uint64_t i = threadIdx.x; i < (uint64_t(1) << n); i += blockDim.x) {
    double ar = 0.0, ai = 0.0;
    for (uint32_t gi = 0; gi < H.ngroups; ++gi) {
      const PauliGroup &G = H.g[gi];
      double c = 0.0;
      for (uint32_t t = G.t0; t < G.t1; ++t) c += (__popcll(i & H.zy[t]) & 1) ? -H.f[t] : H.f[t];
      const C2 b = psi_at(i ^ G.x);
      if (G.odd) {  // c * (-i) * b
        ar += c * double(b.y);
        ai -= c * double(b.x);
      } else {
        ar += c * double(b.x);
        ai += c * double(b.y);
      }
    }
    C2 o;
    o.x = Real(ar);
    o.y = Real(ai);
    lam_set(i, o);
    const C2 a = psi_at(i);
    e += double(a.x) * ar + double(a.y) * ai;
  }
  return e;
}

// --- JIT batched-gradient building blocks ---------------------------------
// The generated kernel runs one circuit per CTA (2^(M-3) threads), its psi
// and lambda streamed from the state pool through double-buffered tiles
// (buffer b: phi at bufs + 2 b TS, lambda after it); every sweep's phases are
// straight-line code with the sweep's tile bits as constants.

// |0...0> in a pool state of 2^n amplitudes.
template <typename Real>
__device__ __forceinline__ void jit_batch_init(typename Vec2<Real>::T *psi, uint32_t n) {
  for (uint64_t j = threadIdx.x; j < (uint64_t(1) << n); j += blockDim.x) {
    typename Vec2<Real>::T v;
    v.x = Real(j == 0 ? 1 : 0);
    v.y = Real(0);
    psi[j] = v;
  }
}

// The circuit's coefficients of one sweep (packed record) into shared memory.
template <typename Real>
__device__ __forceinline__ void jit_batch_coef(typename Vec2<Real>::T *coef, const unsigned char *rec,
                                               uint32_t coef_off, uint32_t ncoef) {
  const auto *g = reinterpret_cast<const typename Vec2<Real>::T *>(rec + coef_off);
  for (uint32_t i = threadIdx.x; i < ncoef; i += blockDim.x) coef[i] = g[i];
}

// One single-state sweep over a pool state: phases(tile, gbase) per tile.
template <typename Real, int M, class Tile, class Phases>
__device__ __forceinline__ void jit_batch_fwd(typename Vec2<Real>::T *psi, typename Vec2<Real>::T *bufs,
                                              uint64_t ntiles, Phases phases) {
  using C2 = typename Vec2<Real>::T;
  constexpr uint32_t TS = 1u << M;
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  auto prefetch = [&](uint64_t t, C2 *dst) {
    const uint64_t gb = Tile::base(t);
    for (uint32_t j = tid; j < TS; j += nt) cp_async<sizeof(C2)>(dst + swz<Real>(j), psi + (gb | Tile::off(j)));
  };
  prefetch(0, bufs);
  cp_async_commit();
  for (uint64_t t = 0; t < ntiles; ++t) {
    C2 *cur = bufs + (t & 1) * 2 * TS;
    if (t + 1 < ntiles) prefetch(t + 1, bufs + ((t + 1) & 1) * 2 * TS);
    cp_async_commit();
    cp_async_wait_prev();
    __syncthreads();
    const uint64_t gbase = Tile::base(t);
    phases(cur, gbase);
    for (uint32_t j = tid; j < TS; j += nt) psi[gbase | Tile::off(j)] = cur[swz<Real>(j)];
    __syncthreads();
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// One two-state (reverse) sweep over the pool states psi and lambda:
// phases(phi_tile, lambda_tile, gbase) per tile.
template <typename Real, int M, class Tile, class Phases>
__device__ __forceinline__ void jit_batch_rev(typename Vec2<Real>::T *psi, typename Vec2<Real>::T *lam,
                                              typename Vec2<Real>::T *bufs, uint64_t ntiles, Phases phases) {
  using C2 = typename Vec2<Real>::T;
  constexpr uint32_t TS = 1u << M;
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  auto prefetch = [&](uint64_t t, C2 *dst) {
    const uint64_t gb = Tile::base(t);
    for (uint32_t j = tid; j < TS; j += nt) {
      const uint64_t g = gb | Tile::off(j);
      cp_async<sizeof(C2)>(dst + swz<Real>(j), psi + g);
      cp_async<sizeof(C2)>(dst + TS + swz<Real>(j), lam + g);
    }
  };
  prefetch(0, bufs);
  cp_async_commit();
  for (uint64_t t = 0; t < ntiles; ++t) {
    C2 *cf = bufs + (t & 1) * 2 * TS, *cl = cf + TS;
    if (t + 1 < ntiles) prefetch(t + 1, bufs + ((t + 1) & 1) * 2 * TS);
    cp_async_commit();
    cp_async_wait_prev();
    __syncthreads();
    const uint64_t gbase = Tile::base(t);
    phases(cf, cl, gbase);
    for (uint32_t j = tid; j < TS; j += nt) {
      const uint64_t g = gbase | Tile::off(j);
      psi[g] = cf[swz<Real>(j)];
      lam[g] = cl[swz<Real>(j)];
    }
    __syncthreads();
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Zeroes the per-warp inner-product slots.
__device__ __forceinline__ void jit_batch_acc_zero(double2 *acc, int nw) {
  for (int i = threadIdx.x; i < nw * kMaxInner; i += blockDim.x) {
    double2 z;
    z.x = 0.0;
    z.y = 0.0;
    acc[i] = z;
  }
}

// Adds slot SLOT's sum over warps (fixed order) to one occurrence's output.
__device__ __forceinline__ void jit_batch_slot_add(const double2 *acc, int nw, int slot, double2 *out) {
  double r = 0.0, i = 0.0;
  for (int w = 0; w < nw; ++w) {
    r += acc[w * kMaxInner + slot].x;
    i += acc[w * kMaxInner + slot].y;
  }
  out->x += r;
  out->y += i;
}

}  // namespace sq

// Device building blocks of the JIT-specialised kernels (snuqs_b200/csrc/jit.cu
// generates one kernel per planned sweep from these and compiles it with
// NVRTC; jit.cu's host code uses the shared-memory size helpers).  Register
// positions, op kinds, masks and coefficient offsets become compile-time
// constants, so each phase compiles to straight-line code: no op dispatch,
// and no register shuffling back to fixed registers between gates.  Kept
// apart from sweep_kernels.cuh, which the precompiled kernels include.
#pragma once
#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stdint.h>

#include "sweep_kernels.cuh"
#endif

namespace sq {

// Coefficients read straight from the kernel's parameter block (constant
// bank) at compile-time offsets: no shared-memory load per coefficient, and
// one compiled kernel still serves every coefficient value.
template <typename Real, int OFF>
struct ParamCoef {
  const Real *p;  // SweepParams::coef
  __device__ __forceinline__ typename Vec2<Real>::T operator[](uint32_t i) const {
    typename Vec2<Real>::T v;
    v.x = p[2 * (OFF + i)];
    v.y = p[2 * (OFF + i) + 1];
    return v;
  }
};

// Complex products of the fused diagonal runs: o = a b, and a *= b.
template <typename Real>
__device__ __forceinline__ void jit_cmul(Real ar, Real ai, Real br, Real bi, Real &o_r, Real &o_i) {
  o_r = ar * br - ai * bi;
  o_i = ar * bi + ai * br;
}
template <typename Real>
__device__ __forceinline__ void jit_cmul_acc(Real &ar, Real &ai, Real br, Real bi) {
  const Real r = ar * br - ai * bi;
  ai = ar * bi + ai * br;
  ar = r;
}

// Tile geometry of one sweep with its high tile bits as constants: tile
// position L+i holds global index bit HI[i] (ascending); positions below L
// are the L lowest global bits.  Global addresses then need no lookup table.
template <int M, int L, int... HI>
struct JitTile {
  static_assert(sizeof...(HI) == M - L, "one global bit per high tile position");
  static constexpr int kLow = L;
  // Global offset of tile-local index j.  Bitwise: off(a | b) = off(a) | off(b)
  // for disjoint a, b.
  __host__ __device__ static constexpr uint64_t off(uint32_t j) {
    uint64_t x = j & ((1u << L) - 1u);
    int i = L;
    ((x |= uint64_t((j >> i++) & 1u) << HI), ...);
    return x;
  }
  // Global index of element 0 of tile t: the bits of t fill the non-tile
  // positions, ascending.
  __device__ __forceinline__ static uint64_t base(uint64_t t) {
    uint64_t x = t << L;
    ((x = ((x >> HI) << (HI + 1)) | (x & ((uint64_t(1) << HI) - 1))), ...);
    return x;
  }
  // Output order of the copy-out: tile positions are already ascending by
  // global bit, so output index o is tile element o.
  __host__ __device__ static constexpr uint32_t src(uint32_t o) { return o; }
  __host__ __device__ static constexpr uint64_t soff(uint32_t o) { return off(o); }
};

// Output geometry of a remapping sweep: tile position p is stored to global
// bit OUT[p] (a permutation of the tile's bits; the tile base is unchanged).
// off(j): global offset of tile element j on the way out.  For the copy-out,
// output index o numbers the outputs in ascending global-bit order (bit i of
// o <-> the i-th lowest output bit): src(o) is the tile element stored there
// and soff(o) its offset.  All three are linear over disjoint bits.
template <int M, int... OUT>
struct JitTileMap {
  static_assert(sizeof...(OUT) == M, "one output bit per tile position");
  __host__ __device__ static constexpr uint64_t off(uint32_t j) {
    uint64_t x = 0;
    int p = 0;
    ((x |= uint64_t((j >> p++) & 1u) << OUT), ...);
    return x;
  }
  // Tile position holding the i-th lowest output bit.
  __host__ __device__ static constexpr int sorted_pos(int i) {
    const int out[M] = {OUT...};
    for (int p = 0; p < M; ++p) {
      int below = 0;
      for (int q = 0; q < M; ++q) below += out[q] < out[p] ? 1 : 0;
      if (below == i) return p;
    }
    return 0;
  }
  __host__ __device__ static constexpr uint32_t src(uint32_t o) {
    uint32_t x = 0;
    for (int i = 0; i < M; ++i)
      if ((o >> i) & 1u) x |= 1u << sorted_pos(i);
    return x;
  }
  __host__ __device__ static constexpr uint64_t soff(uint32_t o) { return off(src(o)); }
};

// One phase: register bits R0..R3 (tile positions, ascending), thread bit i
// on tile position T[i].
template <typename Real, int M, class Tile, int R0, int R1, int R2, int R3, int... T>
struct JitPhase {
  using C2 = typename Vec2<Real>::T;
  static_assert(sizeof...(T) == M - kRegBits, "one tile position per thread bit");
  // The code generator places the lane bits that share a shared-memory
  // wavefront on positions whose swizzle images are independent
  // (conflict-free gathers and scatters), or, in a phase that moves data
  // straight between registers and HBM, on the lowest positions (coalesced).
  __device__ __forceinline__ static uint32_t jb(uint32_t tid) {
    uint32_t x = 0;
    int i = 0;
    ((x |= ((tid >> i++) & 1u) << T), ...);
    return x;
  }
  __device__ __forceinline__ static uint32_t slot(uint32_t sb, int ri) {
    constexpr uint32_t W0 = swz_c<Real>(1u << R0), W1 = swz_c<Real>(1u << R1);
    constexpr uint32_t W2 = swz_c<Real>(1u << R2), W3 = swz_c<Real>(1u << R3);
    return sb ^ ((ri & 1) ? W0 : 0u) ^ ((ri & 2) ? W1 : 0u) ^ ((ri & 4) ? W2 : 0u) ^ ((ri & 8) ? W3 : 0u);
  }
  // Global offset of register slot ri relative to the thread's base.
  __device__ __forceinline__ static constexpr uint64_t goff(int ri) {
    return ((ri & 1) ? Tile::off(1u << R0) : 0) + ((ri & 2) ? Tile::off(1u << R1) : 0) +
           ((ri & 4) ? Tile::off(1u << R2) : 0) + ((ri & 8) ? Tile::off(1u << R3) : 0);
  }
  __device__ __forceinline__ static void gather(Amps<Real> &A, const C2 *tile, uint32_t jbv) {
    const uint32_t sb = swz<Real>(jbv);
#pragma unroll
    for (int ri = 0; ri < kRegAmps; ++ri) {
      const C2 v = tile[slot(sb, ri)];
      A.re[ri] = v.x;
      A.im[ri] = v.y;
    }
  }
  __device__ __forceinline__ static void scatter(const Amps<Real> &A, C2 *tile, uint32_t jbv) {
    const uint32_t sb = swz<Real>(jbv);
#pragma unroll
    for (int ri = 0; ri < kRegAmps; ++ri) {
      C2 v;
      v.x = A.re[ri];
      v.y = A.im[ri];
      tile[slot(sb, ri)] = v;
    }
  }
  // From a row-major (unswizzled) copy of the tile: tile index j at j.
  __device__ __forceinline__ static constexpr uint32_t loff(int ri) {
    return ((ri & 1) ? 1u << R0 : 0u) | ((ri & 2) ? 1u << R1 : 0u) | ((ri & 4) ? 1u << R2 : 0u) |
           ((ri & 8) ? 1u << R3 : 0u);
  }
  __device__ __forceinline__ static void gather_lin(Amps<Real> &A, const C2 *stage, uint32_t jbv) {
    const C2 *p = stage + jbv;
#pragma unroll
    for (int ri = 0; ri < kRegAmps; ++ri) {
      const C2 v = p[loff(ri)];
      A.re[ri] = v.x;
      A.im[ri] = v.y;
    }
  }
  // Straight from HBM into registers (a first phase whose register bits
  // leave the low tile bits to the lanes).
  __device__ __forceinline__ static void load(Amps<Real> &A, const C2 *__restrict__ psi, uint64_t gbase,
                                              uint32_t jbv) {
    const C2 *p = psi + (gbase | Tile::off(jbv));
#pragma unroll
    for (int ri = 0; ri < kRegAmps; ++ri) {
      const C2 v = p[goff(ri)];
      A.re[ri] = v.x;
      A.im[ri] = v.y;
    }
  }
  // The first phase of a state that starts as |0...0>: amplitude 1 where the
  // global index has no bit of nmask set (state index bits), else 0; nothing
  // is read (multi-state sweeps: the first sweep of a structure group).
  __device__ __forceinline__ static void zero_state(Amps<Real> &A, uint64_t gbase, uint32_t jbv, uint64_t nmask) {
    const uint64_t base = gbase | Tile::off(jbv);
#pragma unroll
    for (int ri = 0; ri < kRegAmps; ++ri) {
      A.re[ri] = Real(((base | goff(ri)) & nmask) == 0 ? 1 : 0);
      A.im[ri] = Real(0);
    }
  }
  // Straight from registers to HBM (the mirror case for a last phase).
  __device__ __forceinline__ static void store(const Amps<Real> &A, C2 *psi, uint64_t gbase, uint32_t jbv) {
    C2 *p = psi + (gbase | Tile::off(jbv));
#pragma unroll
    for (int ri = 0; ri < kRegAmps; ++ri) {
      C2 v;
      v.x = A.re[ri];
      v.y = A.im[ri];
      p[goff(ri)] = v;
    }
  }
};

// Dynamic shared memory of a JIT sweep kernel: one tile buffer when the first
// phase loads from HBM (DLOAD), else two (the next tile streams into the
// second), then the coefficients when a phase reads them from shared memory.
__host__ __device__ constexpr size_t jit_smem_bytes(int m, size_t amp_bytes, bool dload, uint32_t smem_coef) {
  return (dload ? 1 : 2) * (size_t(1) << m) * amp_bytes + size_t(smem_coef) * amp_bytes;
}

// The tile loop with the phases supplied by the generated kernel:
// phases(tile, coef, gbase) runs every phase of one tile.
//  SMEM_COEF: the phases also read coefficients from shared memory (diagonal
//             ops indexed by tile bits that vary across the lanes);
//  DLOAD:     the first phase loads from HBM itself (no tile prefetch);
//  DSTORE:    the last phase stores to HBM itself (no copy-out).
// Early-load tile loop of a direct-load sweep: the registers of tile
// t + gridDim.x's first phase are loaded from HBM (load0) before tile t's
// phases run, so every CTA keeps one tile's loads in flight while it computes
// (at the price of a second register set).  phases(A0, tile, coef, gbase)
// runs every phase of one tile starting from the first phase's registers A0.
template <typename Real, int M, class Tile, bool SMEM_COEF, bool DSTORE, class Out, class Load0, class Phases>
__device__ __forceinline__ void jit_sweep_early(typename Vec2<Real>::T *__restrict__ psi,
                                                const SweepParams<Real> &P, Load0 load0, Phases phases) {
  using C2 = typename Vec2<Real>::T;
  constexpr int NT = 1 << (M - kRegBits);
  constexpr uint32_t TS = 1u << M;
  constexpr uint32_t PER = TS / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SweepHeader &h = P.h;
  C2 *tile = reinterpret_cast<C2 *>(smem_raw);
  C2 *coef = tile + TS;
  const uint32_t tid = threadIdx.x;
  if constexpr (SMEM_COEF) {
    for (uint32_t i = tid; i < h.ncoef; i += NT) {
      C2 v;
      v.x = P.coef[2 * i];
      v.y = P.coef[2 * i + 1];
      coef[i] = v;
    }
    __syncthreads();
  }
  const uint32_t s_tid = swz<Real>(tid);
  const uint32_t o_tid = swz<Real>(Out::src(tid));  // copy-out: output index tid
  const uint64_t ooff = Out::soff(tid);
  const uint64_t toff = Tile::off(tid);
  Amps<Real> next;
  if (blockIdx.x < h.num_tiles) load0(next, Tile::base(blockIdx.x));
  for (uint64_t t = blockIdx.x; t < h.num_tiles; t += gridDim.x) {
    const Amps<Real> cur = next;
    const uint64_t tn = t + gridDim.x;
    if (tn < h.num_tiles) load0(next, Tile::base(tn));
    const uint64_t gbase = Tile::base(t);
    phases(cur, tile, coef, gbase);
    if constexpr (!DSTORE) {
#pragma unroll
      for (uint32_t it = 0; it < PER; ++it)
        psi[gbase | ooff | Out::soff(it * NT)] = tile[o_tid ^ swz<Real>(Out::src(it * NT))];
    }
    __syncthreads();
  }
}

template <typename Real, int M, class Tile, bool SMEM_COEF, bool DLOAD, bool DSTORE, class Out, class Phases>
__device__ __forceinline__ void jit_sweep(typename Vec2<Real>::T *__restrict__ psi,
                                          const SweepParams<Real> &P, Phases phases) {
  using C2 = typename Vec2<Real>::T;
  constexpr int NT = 1 << (M - kRegBits);
  constexpr uint32_t TS = 1u << M;
  constexpr uint32_t PER = TS / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SweepHeader &h = P.h;
  C2 *bufs = reinterpret_cast<C2 *>(smem_raw);
  C2 *coef = bufs + (DLOAD ? 1 : 2) * TS;
  const uint32_t tid = threadIdx.x;
  if constexpr (SMEM_COEF) {
    for (uint32_t i = tid; i < h.ncoef; i += NT) {
      C2 v;
      v.x = P.coef[2 * i];
      v.y = P.coef[2 * i + 1];
      coef[i] = v;
    }
    __syncthreads();
  }
  // Element j = it * NT + tid of a tile: global offset off(it * NT) | off(tid).
  const uint32_t s_tid = swz<Real>(tid);
  const uint32_t o_tid = swz<Real>(Out::src(tid));  // copy-out: output index tid
  const uint64_t ooff = Out::soff(tid);
  const uint64_t toff = Tile::off(tid);
  if constexpr (DLOAD) {
    for (uint64_t t = blockIdx.x; t < h.num_tiles; t += gridDim.x) {
      const uint64_t gbase = Tile::base(t);
      phases(bufs, coef, gbase);
      if constexpr (!DSTORE) {
#pragma unroll
        for (uint32_t it = 0; it < PER; ++it)
          psi[gbase | ooff | Out::soff(it * NT)] = bufs[o_tid ^ swz<Real>(Out::src(it * NT))];
      }
      __syncthreads();
    }
  } else {
    auto prefetch = [&](uint64_t t, C2 *dst) {
      const C2 *src = psi + (Tile::base(t) | toff);
#pragma unroll
      for (uint32_t it = 0; it < PER; ++it)
        cp_async<sizeof(C2)>(dst + (s_tid ^ swz<Real>(it * NT)), src + Tile::off(it * NT));
    };
    uint32_t cur = 0;
    if (blockIdx.x < h.num_tiles) prefetch(blockIdx.x, bufs);
    cp_async_commit();
    for (uint64_t t = blockIdx.x; t < h.num_tiles; t += gridDim.x) {
      C2 *tile = bufs + cur * TS;
      const uint64_t tn = t + gridDim.x;
      if (tn < h.num_tiles) prefetch(tn, bufs + (cur ^ 1) * TS);
      cp_async_commit();
      cp_async_wait_prev();
      __syncthreads();
      const uint64_t gbase = Tile::base(t);
      phases(tile, coef, gbase);
      if constexpr (!DSTORE) {
#pragma unroll
        for (uint32_t it = 0; it < PER; ++it)
          psi[gbase | ooff | Out::soff(it * NT)] = tile[o_tid ^ swz<Real>(Out::src(it * NT))];
      }
      __syncthreads();
      cur ^= 1;
    }
    cp_async_wait_prev();
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  }
}

// ---------------------------------------------------------------------------
// Multi-state sweeps: one launch applies one sweep to K states of 2^n
// amplitudes that share the sweep's structure (the circuits of a batch with
// one plan structure and different angles).  The states lie back to back
// (state c at psi + c 2^n), so together they form one index space whose bits
// above n number the state: tile t of the launch is Tile::base(t), with
// t >> tile_shift the state (tile_shift = n - M), and the ops' conditions on
// global bits (all below n) hold per state.  State c's coefficients are the
// ncoef complex values at coefs + c stride (bytes), i.e. the coefficient
// block of this sweep's packed record in circuit c's plan.  Each CTA takes a
// contiguous range of tiles, so it reloads the shared-memory copy of the
// coefficients only when its range crosses into the next state.
struct MultiParams {
  const unsigned char *coefs;  // state 0's coefficients of this sweep
  uint64_t stride;             // bytes between consecutive states' coefficients
  uint64_t tiles;              // K << tile_shift
  uint32_t tile_shift;         // log2 tiles per state
  uint32_t ncoef;
};

template <typename Real>
__device__ __forceinline__ void jit_multi_coef(typename Vec2<Real>::T *coef, const MultiParams &Q, uint64_t c) {
  const auto *g = reinterpret_cast<const typename Vec2<Real>::T *>(Q.coefs + c * Q.stride);
  for (uint32_t i = threadIdx.x; i < Q.ncoef; i += blockDim.x) coef[i] = g[i];
}

// This CTA's tiles [t0, t1): an equal share of the launch's tiles.
__device__ __forceinline__ void jit_multi_range(const MultiParams &Q, uint64_t &t0, uint64_t &t1) {
  const uint64_t per = (Q.tiles + gridDim.x - 1) / gridDim.x;
  t0 = uint64_t(blockIdx.x) * per;
  t1 = t0 + per < Q.tiles ? t0 + per : Q.tiles;
}

// jit_sweep_early over the tiles of K states (coefficients always in shared
// memory).
template <typename Real, int M, class Tile, bool DSTORE, class Load0, class Phases>
__device__ __forceinline__ void jit_msweep_early(typename Vec2<Real>::T *__restrict__ psi, const MultiParams &Q,
                                                 Load0 load0, Phases phases) {
  using C2 = typename Vec2<Real>::T;
  constexpr int NT = 1 << (M - kRegBits);
  constexpr uint32_t TS = 1u << M;
  constexpr uint32_t PER = TS / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *tile = reinterpret_cast<C2 *>(smem_raw);
  C2 *coef = tile + TS;
  const uint32_t tid = threadIdx.x;
  const uint32_t s_tid = swz<Real>(tid);
  const uint64_t toff = Tile::off(tid);
  uint64_t t0, t1;
  jit_multi_range(Q, t0, t1);
  uint64_t cur_c = ~uint64_t(0);
  Amps<Real> next;
  if (t0 < t1) load0(next, Tile::base(t0));
  for (uint64_t t = t0; t < t1; ++t) {
    const Amps<Real> cur = next;
    if (t + 1 < t1) load0(next, Tile::base(t + 1));
    const uint64_t c = t >> Q.tile_shift;
    if (c != cur_c) {  // uniform: the previous tile ended with a barrier
      jit_multi_coef<Real>(coef, Q, c);
      cur_c = c;
      __syncthreads();
    }
    const uint64_t gbase = Tile::base(t);
    phases(cur, tile, coef, gbase);
    if constexpr (!DSTORE) {
#pragma unroll
      for (uint32_t it = 0; it < PER; ++it)
        psi[gbase | toff | Tile::off(it * NT)] = tile[s_tid ^ swz<Real>(it * NT)];
    }
    __syncthreads();
  }
}

// jit_sweep over the tiles of K states (coefficients always in shared
// memory; the first phase loads from HBM itself when DLOAD, else the next
// tile streams into a second buffer by cp.async).
template <typename Real, int M, class Tile, bool DLOAD, bool DSTORE, class Phases>
__device__ __forceinline__ void jit_msweep(typename Vec2<Real>::T *__restrict__ psi, const MultiParams &Q,
                                           Phases phases) {
  using C2 = typename Vec2<Real>::T;
  constexpr int NT = 1 << (M - kRegBits);
  constexpr uint32_t TS = 1u << M;
  constexpr uint32_t PER = TS / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *bufs = reinterpret_cast<C2 *>(smem_raw);
  C2 *coef = bufs + (DLOAD ? 1 : 2) * TS;
  const uint32_t tid = threadIdx.x;
  const uint32_t s_tid = swz<Real>(tid);
  const uint64_t toff = Tile::off(tid);
  uint64_t t0, t1;
  jit_multi_range(Q, t0, t1);
  uint64_t cur_c = ~uint64_t(0);
  auto prefetch = [&](uint64_t t, C2 *dst) {
    const C2 *src = psi + (Tile::base(t) | toff);
#pragma unroll
    for (uint32_t it = 0; it < PER; ++it)
      cp_async<sizeof(C2)>(dst + (s_tid ^ swz<Real>(it * NT)), src + Tile::off(it * NT));
  };
  uint32_t cur = 0;
  if constexpr (!DLOAD) {
    if (t0 < t1) prefetch(t0, bufs);
    cp_async_commit();
  }
  for (uint64_t t = t0; t < t1; ++t) {
    C2 *tile = bufs + (DLOAD ? 0 : cur * TS);
    if constexpr (!DLOAD) {
      if (t + 1 < t1) prefetch(t + 1, bufs + (cur ^ 1) * TS);
      cp_async_commit();
    }
    const uint64_t c = t >> Q.tile_shift;
    if (c != cur_c) {
      jit_multi_coef<Real>(coef, Q, c);
      cur_c = c;
    }
    if constexpr (!DLOAD) cp_async_wait_prev();
    __syncthreads();
    const uint64_t gbase = Tile::base(t);
    phases(tile, coef, gbase);
    if constexpr (!DSTORE) {
#pragma unroll
      for (uint32_t it = 0; it < PER; ++it)
        psi[gbase | toff | Tile::off(it * NT)] = tile[s_tid ^ swz<Real>(it * NT)];
    }
    __syncthreads();
    cur ^= 1;
  }
  if constexpr (!DLOAD) asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// Bulk-copy tile pipeline (cp.async.bulk with mbarrier transaction counts).
//
// A sweep whose first phase reads its amplitudes with the lanes on the low
// tile positions (the planner's direct-load sweeps) can take its tile from a
// plain row-major copy of the tile: the lanes that share a shared-memory
// wavefront then read consecutive amplitudes, conflict-free without a
// swizzle.  Such a copy is exactly what the bulk-copy engine produces: one
// cp.async.bulk per contiguous run of 2^L amplitudes (128 bytes), issued by
// one warp, completing on the stage's mbarrier.  The copies need no thread
// registers and no per-thread instructions, so a CTA keeps S tiles in flight
// while it computes: the loads of tile i + S are issued as soon as every
// thread has read tile i's stage (right after the first phase's gather), and
// overlap the remaining phases and stores of tile i.  Later phases pass the
// tile through a swizzled work buffer as in jit_sweep; the last phase of a
// direct-store sweep writes to HBM from registers.
// Every wait is bounded: a stage that has not arrived after kPipeWaitPolls
// polls sets the sweep's error word (read by the host) and the CTA stops
// waiting; the remaining tiles are then garbage, which the error reports.
// ---------------------------------------------------------------------------
constexpr uint32_t kPipeWaitPolls = 1u << 22;
constexpr uint32_t kKernelErrTimeout = 1u;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// One arrival that also announces `bytes` of bulk-copy transactions.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait for the phase of `bar` with the given parity.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  for (uint32_t i = 0; i < kPipeWaitPolls; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// Global -> shared bulk copy completing `bytes` transactions on `bar`
// (both addresses 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Orders this thread's earlier generic-proxy shared-memory accesses (made
// visible to it by a barrier) before its later bulk copies into the same
// memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Dynamic shared memory of a pipelined JIT sweep: S stages (row-major tiles),
// the swizzled work buffer when some phase passes the tile through shared
// memory, the coefficients when a phase reads them there, S mbarriers.
__host__ __device__ constexpr size_t jit_pipe_smem_bytes(int m, size_t amp_bytes, int stages, bool work,
                                                         uint32_t smem_coef) {
  return (size_t(stages) + (work ? 1 : 0)) * (size_t(1) << m) * amp_bytes + size_t(smem_coef) * amp_bytes +
         size_t(stages) * 8;
}

// Copy-engine side of the pipeline: warp 0 issues the bulk copies of local
// tile i (tile blockIdx.x + i * gridDim.x) into stage i % S; release() is
// called by every thread once it has read the current tile's stage.
template <typename Real, int M, class Tile, int S>
struct PipeCtl {
  using C2 = typename Vec2<Real>::T;
  static constexpr uint32_t TS = 1u << M;
  static constexpr int L = Tile::kLow;
  static constexpr uint32_t RUNS = 1u << (M - L);
  static constexpr uint32_t RUN_BYTES = (1u << L) * uint32_t(sizeof(C2));
  static_assert(RUN_BYTES % 16 == 0, "bulk copies move multiples of 16 bytes");
  const C2 *psi;
  C2 *stages;
  uint64_t *bar;
  uint64_t ntiles;  // tiles of this CTA
  uint64_t cur;     // local index of the tile being processed
  uint32_t lane, warp;

  __device__ __forceinline__ void issue(uint64_t i) const {
    const int s = int(i % S);
    if (lane == 0) mbar_arrive_expect_tx(&bar[s], TS * uint32_t(sizeof(C2)));
    __syncwarp();  // the transaction count is announced before any copy lands
    const C2 *src = psi + Tile::base(blockIdx.x + i * gridDim.x);
    C2 *dst = stages + s * TS;
    for (uint32_t r = lane; r < RUNS; r += 32)
      bulk_load(dst + (r << L), src + Tile::off(r << L), RUN_BYTES, &bar[s]);
  }
  // Every thread has read stage cur % S: hand it to tile cur + S.
  __device__ __forceinline__ void release() const {
    __syncthreads();
    if (warp == 0 && cur + S < ntiles) {
      fence_proxy_async_smem();
      issue(cur + S);
    }
  }
};

// The pipelined tile loop.  phases(stage, work, coef, gbase, ctl) runs every
// phase of one tile; its first phase gathers from `stage` (row-major) and
// then calls ctl.release(), which hands the stage back to the copy engine.
//  SMEM_COEF: some phase reads coefficients from shared memory;
//  WORK:      some phase passes the tile through the work buffer;
//  DSTORE:    the last phase stores to HBM itself (no copy-out);
//  S:         stages (tiles in flight per CTA).
template <typename Real, int M, class Tile, bool SMEM_COEF, bool WORK, bool DSTORE, int S, class Out,
          class Phases>
__device__ __forceinline__ void jit_sweep_pipe(typename Vec2<Real>::T *__restrict__ psi,
                                               const SweepParams<Real> &P, uint32_t *__restrict__ err,
                                               Phases phases) {
  using C2 = typename Vec2<Real>::T;
  constexpr int NT = 1 << (M - kRegBits);
  constexpr uint32_t TS = 1u << M;
  constexpr uint32_t PER = TS / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SweepHeader &h = P.h;
  PipeCtl<Real, M, Tile, S> ctl;
  ctl.psi = psi;
  ctl.stages = reinterpret_cast<C2 *>(smem_raw);
  C2 *work = ctl.stages + S * TS;
  C2 *coef = work + (WORK ? TS : 0);
  ctl.bar = reinterpret_cast<uint64_t *>(coef + (SMEM_COEF ? ((h.ncoef + 1) & ~1u) : 0u));
  const uint32_t tid = threadIdx.x;
  ctl.lane = tid & 31u;
  ctl.warp = tid >> 5;
  ctl.ntiles = h.num_tiles > blockIdx.x ? (h.num_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  ctl.cur = 0;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&ctl.bar[s], 1);
    fence_mbar_init();
  }
  if constexpr (SMEM_COEF) {
    for (uint32_t i = tid; i < h.ncoef; i += NT) {
      C2 v;
      v.x = P.coef[2 * i];
      v.y = P.coef[2 * i + 1];
      coef[i] = v;
    }
  }
  __syncthreads();
  if (ctl.warp == 0)
    for (uint64_t i = 0; i < uint64_t(S) && i < ctl.ntiles; ++i) ctl.issue(i);
  const uint32_t s_tid = swz<Real>(tid);
  const uint32_t o_tid = swz<Real>(Out::src(tid));  // copy-out: output index tid
  const uint64_t ooff = Out::soff(tid);
  const uint64_t toff = Tile::off(tid);
  bool alive = true;
  for (uint64_t i = 0; i < ctl.ntiles; ++i) {
    const int s = int(i % S);
    if (alive && !mbar_wait_bounded(&ctl.bar[s], uint32_t((i / S) & 1))) {
      alive = false;
      atomicOr(err, kKernelErrTimeout);
    }
    ctl.cur = i;
    const uint64_t gbase = Tile::base(blockIdx.x + i * gridDim.x);
    phases(ctl.stages + s * TS, work, coef, gbase, ctl);
    if constexpr (!DSTORE) {
#pragma unroll
      for (uint32_t it = 0; it < PER; ++it)
        psi[gbase | toff | Tile::off(it * NT)] = work[s_tid ^ swz<Real>(it * NT)];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// JIT-specialised two-state (adjoint reverse) sweeps: the generated kernel
// un-computes phi and lambda together and accumulates <lambda| K |phi> for
// each inner-product op, with the same plan, shared-memory layout and
// per-warp partial sums as adjoint_sweep_kernel (adjoint_kernels.cuh).
// ---------------------------------------------------------------------------
template <typename Real, int M, class Tile, int R0, int R1, int R2, int... T>
struct JitPhase2 {
  using C2 = typename Vec2<Real>::T;
  static_assert(sizeof...(T) == M - kAdjRegBits, "one tile position per thread bit");
  __device__ __forceinline__ static uint32_t jb(uint32_t tid) {
    uint32_t x = 0;
    int i = 0;
    ((x |= ((tid >> i++) & 1u) << T), ...);
    return x;
  }
  __device__ __forceinline__ static uint32_t slot(uint32_t sb, int ri) {
    constexpr uint32_t W0 = swz_c<Real>(1u << R0), W1 = swz_c<Real>(1u << R1);
    constexpr uint32_t W2 = swz_c<Real>(1u << R2);
    return sb ^ ((ri & 1) ? W0 : 0u) ^ ((ri & 2) ? W1 : 0u) ^ ((ri & 4) ? W2 : 0u);
  }
  __device__ __forceinline__ static void gather(Amps<Real, kAdjAmps> &F, Amps<Real, kAdjAmps> &G,
                                                const C2 *ft, const C2 *lt, uint32_t jbv) {
    const uint32_t sb = swz<Real>(jbv);
#pragma unroll
    for (int ri = 0; ri < kAdjAmps; ++ri) {
      const C2 a = ft[slot(sb, ri)], b = lt[slot(sb, ri)];
      F.re[ri] = a.x;
      F.im[ri] = a.y;
      G.re[ri] = b.x;
      G.im[ri] = b.y;
    }
  }
  __device__ __forceinline__ static void scatter(const Amps<Real, kAdjAmps> &F, const Amps<Real, kAdjAmps> &G,
                                                 C2 *ft, C2 *lt, uint32_t jbv) {
    const uint32_t sb = swz<Real>(jbv);
#pragma unroll
    for (int ri = 0; ri < kAdjAmps; ++ri) {
      C2 a, b;
      a.x = F.re[ri];
      a.y = F.im[ri];
      b.x = G.re[ri];
      b.y = G.im[ri];
      ft[slot(sb, ri)] = a;
      lt[slot(sb, ri)] = b;
    }
  }
};

// Adds one thread's inner-product share to its warp's slot (warp shuffle,
// then lane 0 adds to acc[warp * kMaxInner + SLOT]).
template <int NT, int SLOT>
__device__ __forceinline__ void jit_inner_acc(double2 *acc, double sr, double si) {
  constexpr unsigned kMask = NT >= 32 ? 0xffffffffu : ((1u << NT) - 1u);
#pragma unroll
  for (int off = (NT >= 32 ? 16 : NT / 2); off > 0; off >>= 1) {
    sr += __shfl_xor_sync(kMask, sr, off);
    si += __shfl_xor_sync(kMask, si, off);
  }
  if ((threadIdx.x & 31) == 0) {
    double2 &a = acc[(threadIdx.x >> 5) * kMaxInner + SLOT];
    a.x += sr;
    a.y += si;
  }
}

// Dynamic shared memory of a JIT adjoint sweep: phi tiles (2 buffers) |
// lambda tiles (2 buffers) | coefficients | per-warp inner-product slots.
__host__ __device__ constexpr size_t jit_adjoint_smem_bytes(int m, size_t amp_bytes, uint32_t ncoef) {
  return 4 * (size_t(1) << m) * amp_bytes + size_t((ncoef + 1) & ~1u) * amp_bytes +
         size_t(((1 << (m - kAdjRegBits)) + 31) / 32) * kMaxInner * 16;
}

// The two-state tile loop with the phases supplied by the generated kernel:
// phases(ft, lt, coef, gbase, acc) runs every phase of one tile pair.
// partials[(block * warps + warp) * kMaxInner + slot] receives each warp's
// sums at the end (as adjoint_sweep_kernel).
template <typename Real, int M, class Tile, class Phases>
__device__ __forceinline__ void jit_adjoint_sweep(typename Vec2<Real>::T *__restrict__ psi,
                                                  typename Vec2<Real>::T *__restrict__ lam,
                                                  const SweepParams<Real> &P, double2 *__restrict__ partials,
                                                  Phases phases) {
  using C2 = typename Vec2<Real>::T;
  constexpr int NT = 1 << (M - kAdjRegBits);
  constexpr int NW = (NT + 31) / 32;
  constexpr uint32_t TS = 1u << M;
  constexpr uint32_t PER = TS / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SweepHeader &h = P.h;
  C2 *fbufs = reinterpret_cast<C2 *>(smem_raw);
  C2 *lbufs = fbufs + 2 * TS;
  C2 *coef = lbufs + 2 * TS;
  double2 *acc = reinterpret_cast<double2 *>(coef + ((h.ncoef + 1) & ~1u));
  const uint32_t tid = threadIdx.x;
  for (uint32_t i = tid; i < h.ncoef; i += NT) {
    C2 v;
    v.x = P.coef[2 * i];
    v.y = P.coef[2 * i + 1];
    coef[i] = v;
  }
  for (uint32_t i = tid; i < NW * kMaxInner; i += NT) {
    double2 z;
    z.x = 0.0;
    z.y = 0.0;
    acc[i] = z;
  }
  __syncthreads();
  const uint32_t s_tid = swz<Real>(tid);
  const uint64_t toff = Tile::off(tid);
  auto prefetch = [&](uint64_t t, C2 *fdst, C2 *ldst) {
    const uint64_t g0 = Tile::base(t) | toff;
#pragma unroll
    for (uint32_t it = 0; it < PER; ++it) {
      const uint64_t g = g0 | Tile::off(it * NT);
      const uint32_t s = s_tid ^ swz<Real>(it * NT);
      cp_async<sizeof(C2)>(fdst + s, psi + g);
      cp_async<sizeof(C2)>(ldst + s, lam + g);
    }
  };
  uint32_t cur = 0;
  if (blockIdx.x < h.num_tiles) prefetch(blockIdx.x, fbufs, lbufs);
  cp_async_commit();
  for (uint64_t t = blockIdx.x; t < h.num_tiles; t += gridDim.x) {
    C2 *ft = fbufs + cur * TS, *lt = lbufs + cur * TS;
    const uint64_t tn = t + gridDim.x;
    if (tn < h.num_tiles) prefetch(tn, fbufs + (cur ^ 1) * TS, lbufs + (cur ^ 1) * TS);
    cp_async_commit();
    cp_async_wait_prev();
    __syncthreads();
    const uint64_t gbase = Tile::base(t);
    phases(ft, lt, coef, gbase, acc);
    const uint64_t g0 = gbase | toff;
#pragma unroll
    for (uint32_t it = 0; it < PER; ++it) {
      const uint64_t g = g0 | Tile::off(it * NT);
      const uint32_t s = s_tid ^ swz<Real>(it * NT);
      psi[g] = ft[s];
      lam[g] = lt[s];
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

}  // namespace sq

// Gate-application kernels for sm_100a.
//
// sweep_kernel: one fused HBM sweep that applies a whole run of gates to
//   2^m-amplitude tiles held in shared memory (see sq_plan.h).  Replaces the
//   reference's one-kernel-per-gate loop over 2^n threads
//   (src/braket/snuqs/csrc/operation/gate_operations_impl_cuda.cu:13-121):
//   64-bit indices throughout, every thread busy, each amplitude read and
//   written once per sweep however many gates the sweep carries.
// gate_kernel / gate_kernel_large: one unfused gate (any k <= 10), used when
//   fusion is off, for k > 4 dense matrices and for cu::applyGate's literal
//   replacement.
#pragma once
#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stdint.h>

#include "sq_plan.h"
#endif

namespace sq {

template <typename Real> struct Vec2;
template <> struct Vec2<double> { using T = double2; };
template <> struct Vec2<float> { using T = float2; };

// Shared-memory swizzle for the amplitude tile: slot(j) = j ^ S(j >> W),
// S linear over GF(2): tile position p >= W adds the W-bit image kSwzImage[p]
// to the low W bits.  W = log2 of the amplitudes one 128-byte shared-memory
// wavefront holds (3 for complex128, 4 for complex64), so the 2^W lanes that
// share a wavefront are conflict-free exactly when the images of the tile
// positions their lane bits sit on are linearly independent (position p < W
// has image e_p).  The images were chosen by exhaustive search so that
//  - for every choice of 4 register positions in tiles of 10..12 bits
//    (complex128) / 11..12 bits (complex64), the remaining positions span
//    GF(2)^W: the JIT kernels can always place the lane bits conflict-free;
//  - with the lane bits on the lowest non-register positions (the generic
//    kernels) 96 % (complex128) / 81 % (complex64) of those register choices
//    are conflict-free, against 48 % / 32 % for the plain fold of the
//    high bits.
// The map is a bijection that only changes the low W bits, and XOR-linear:
// slot(a ^ b) = slot(a) ^ slot(b).
template <typename Real> struct Swz;
template <> struct Swz<double> {
  static constexpr int W = 3;
  static constexpr uint8_t kImage[12] = {1, 2, 4, 7, 3, 5, 6, 4, 5, 7, 6, 6};
};
template <> struct Swz<float> {
  static constexpr int W = 4;
  static constexpr uint8_t kImage[12] = {1, 2, 4, 8, 14, 11, 7, 13, 10, 15, 6, 10};
};

// Positions p >= W whose image has bit i set.
template <typename Real>
__host__ __device__ constexpr uint32_t swz_mask(int i) {
  uint32_t m = 0;
  for (int p = Swz<Real>::W; p < kMaxTileBits; ++p)
    if ((Swz<Real>::kImage[p] >> i) & 1) m |= 1u << p;
  return m;
}

// Compile-time form (constant arguments).
template <typename Real>
__host__ __device__ constexpr uint32_t swz_c(uint32_t j) {
  uint32_t low = 0;
  for (int i = 0; i < Swz<Real>::W; ++i) {
    uint32_t x = j & swz_mask<Real>(i), par = 0;
    for (; x; x &= x - 1) par ^= 1u;
    low |= par << i;
  }
  return j ^ low;
}

template <typename Real>
__device__ __forceinline__ uint32_t swz(uint32_t j) {
  constexpr uint32_t m0 = swz_mask<Real>(0), m1 = swz_mask<Real>(1), m2 = swz_mask<Real>(2);
  constexpr uint32_t m3 = Swz<Real>::W > 3 ? swz_mask<Real>(3) : 0u;
  uint32_t low = (uint32_t(__popc(j & m0)) & 1u) | ((uint32_t(__popc(j & m1)) & 1u) << 1) |
                 ((uint32_t(__popc(j & m2)) & 1u) << 2);
  if constexpr (Swz<Real>::W > 3) low |= (uint32_t(__popc(j & m3)) & 1u) << 3;
  return j ^ low;
}

// Insert a zero bit at position p of x (shifts bits >= p up by one).
__device__ __forceinline__ uint64_t insert_zero(uint64_t x, uint32_t p) {
  const uint64_t lo = x & ((uint64_t(1) << p) - 1);
  return ((x >> p) << (p + 1)) | lo;
}

template <int V>
__device__ __forceinline__ constexpr int ct_popc() {
  return (V & 1) + ((V >> 1) & 1) + ((V >> 2) & 1) + ((V >> 3) & 1);
}

// Compile-time deposit of the low bits of x into the set bits of mask V.
template <int V>
__device__ __forceinline__ constexpr int ct_dep(int x) {
  int r = 0, b = 0;
  for (int p = 0; p < 4; ++p)
    if (V & (1 << p)) {
      if (x & (1 << b)) r |= 1 << p;
      ++b;
    }
  return r;
}

// Compile-time extract of the bits of x at the set bits of mask V.
template <int V>
__device__ __forceinline__ constexpr int ct_ext(int x) {
  int r = 0, b = 0;
  for (int p = 0; p < 4; ++p)
    if (V & (1 << p)) {
      if (x & (1 << p)) r |= 1 << b;
      ++b;
    }
  return r;
}

// Runs f(g) for every register group g (register index with the bits of V
// clear).  Without register controls the loop is branch-free; with them each
// group is predicated on its control bits.
template <int NA, int V, class F>
__device__ __forceinline__ void for_groups(int rmask, int rval, F &&f) {
  if (rmask == 0) {
#pragma unroll
    for (int g = 0; g < NA; ++g)
      if (!(g & V)) f(g);
  } else {
#pragma unroll
    for (int g = 0; g < NA; ++g)
      if (!(g & V) && ((g & rmask) == rval)) f(g);
  }
}

// NA register-resident amplitudes of one thread (16 in the sweep kernel, 8
// per state in the two-state adjoint kernel).
template <typename Real, int NA = kRegAmps>
struct Amps {
  Real re[NA], im[NA];
};

// out = p * a (complex)
template <typename Real>
__device__ __forceinline__ void cmul(Real pr, Real pi, Real ar, Real ai, Real &o_r, Real &o_i) {
  o_r = pr * ar - pi * ai;
  o_i = pr * ai + pi * ar;
}

// kSwDense on register positions V: row r accumulated left to right.
template <typename Real, int NA, int V, class CP>
__device__ __forceinline__ void op_dense(Amps<Real, NA> &A, CP c,
                                         int rmask, int rval) {
  constexpr int D = 1 << ct_popc<V>();
  for_groups<NA, V>(rmask, rval, [&](int g) {
    Real ar[D], ai[D];
#pragma unroll
    for (int x = 0; x < D; ++x) {
      ar[x] = A.re[g | ct_dep<V>(x)];
      ai[x] = A.im[g | ct_dep<V>(x)];
    }
#pragma unroll
    for (int r = 0; r < D; ++r) {
      const auto m0 = c[r * D];
      Real sr = m0.x * ar[0] - m0.y * ai[0];
      Real si = m0.x * ai[0] + m0.y * ar[0];
#pragma unroll
      for (int x = 1; x < D; ++x) {
        const auto m = c[r * D + x];
        sr = fma(m.x, ar[x], sr);
        sr = fma(-m.y, ai[x], sr);
        si = fma(m.x, ai[x], si);
        si = fma(m.y, ar[x], si);
      }
      A.re[g | ct_dep<V>(r)] = sr;
      A.im[g | ct_dep<V>(r)] = si;
    }
  });
}

// kSwAnti1 on register bit V: out0 = p0 a1, out1 = p1 a0 (a swap when pure).
template <typename Real, int NA, int V, bool PURE, class CP>
__device__ __forceinline__ void op_anti1(Amps<Real, NA> &A, CP c,
                                         int rmask, int rval) {
  if constexpr (PURE) {
    for_groups<NA, V>(rmask, rval, [&](int g) {
      const Real tr = A.re[g], ti = A.im[g];
      A.re[g] = A.re[g | V];
      A.im[g] = A.im[g | V];
      A.re[g | V] = tr;
      A.im[g | V] = ti;
    });
  } else {
    const auto p0 = c[0], p1 = c[1];
    for_groups<NA, V>(rmask, rval, [&](int g) {
      const Real a0r = A.re[g], a0i = A.im[g], a1r = A.re[g | V], a1i = A.im[g | V];
      cmul(p0.x, p0.y, a1r, a1i, A.re[g], A.im[g]);
      cmul(p1.x, p1.y, a0r, a0i, A.re[g | V], A.im[g | V]);
    });
  }
}

// kSwXRot on register positions V with partner mask X (canonical local bits):
// out_r = c_r a_r + f s_r a_(r^X).
template <typename Real, int NA, int V, int X, bool IMAG, class CP>
__device__ __forceinline__ void op_xrot(Amps<Real, NA> &A, CP c,
                                        int rmask, int rval) {
  constexpr int D = 1 << ct_popc<V>();
  Real cr[D], sr[D];
#pragma unroll
  for (int r = 0; r < D; ++r) {
    const auto v = c[r];
    cr[r] = v.x;
    sr[r] = v.y;
  }
  for_groups<NA, V>(rmask, rval, [&](int g) {
    Real ar[D], ai[D];
#pragma unroll
    for (int x = 0; x < D; ++x) {
      ar[x] = A.re[g | ct_dep<V>(x)];
      ai[x] = A.im[g | ct_dep<V>(x)];
    }
#pragma unroll
    for (int r = 0; r < D; ++r) {
      const int q = r ^ X;
      Real o_r, o_i;
      if constexpr (IMAG) {  // f = i: s (i a_q) = s (-a_q.im, a_q.re)
        o_r = fma(-sr[r], ai[q], cr[r] * ar[r]);
        o_i = fma(sr[r], ar[q], cr[r] * ai[r]);
      } else {
        o_r = fma(sr[r], ar[q], cr[r] * ar[r]);
        o_i = fma(sr[r], ai[q], cr[r] * ai[r]);
      }
      A.re[g | ct_dep<V>(r)] = o_r;
      A.im[g | ct_dep<V>(r)] = o_i;
    }
  });
}

// kSwSwap2 on register positions V (two bits): out1 = p12 a2, out2 = p21 a1.
template <typename Real, int NA, int V, bool PURE, class CP>
__device__ __forceinline__ void op_swap2(Amps<Real, NA> &A, CP c,
                                         int rmask, int rval) {
  constexpr int B1 = ct_dep<V>(1), B2 = ct_dep<V>(2);
  if constexpr (PURE) {
    for_groups<NA, V>(rmask, rval, [&](int g) {
      const Real tr = A.re[g | B1], ti = A.im[g | B1];
      A.re[g | B1] = A.re[g | B2];
      A.im[g | B1] = A.im[g | B2];
      A.re[g | B2] = tr;
      A.im[g | B2] = ti;
    });
  } else {
    const auto p12 = c[0], p21 = c[1];
    for_groups<NA, V>(rmask, rval, [&](int g) {
      const Real a1r = A.re[g | B1], a1i = A.im[g | B1], a2r = A.re[g | B2], a2i = A.im[g | B2];
      cmul(p12.x, p12.y, a2r, a2i, A.re[g | B1], A.im[g | B1]);
      cmul(p21.x, p21.y, a1r, a1i, A.re[g | B2], A.im[g | B2]);
    });
  }
}

// kSwDiag: coefficient index = thread part << popc(V) | register part.
template <typename Real, int NA, int V, class CP>
__device__ __forceinline__ void op_diag(Amps<Real, NA> &A, CP c,
                                        uint32_t base) {
  const uint32_t cb = base << ct_popc<V>();
#pragma unroll
  for (int ri = 0; ri < NA; ++ri) {
    const auto d = c[cb + ct_ext<V>(ri)];
    const Real r = A.re[ri], i = A.im[ri];
    cmul(d.x, d.y, r, i, A.re[ri], A.im[ri]);
  }
}

// kSwPhase: a *= p on the register slots whose bits match (rmask, rval).
template <typename Real, int NA, bool NEG, class CP>
__device__ __forceinline__ void op_phase(Amps<Real, NA> &A, CP c,
                                         int rmask, int rval) {
  if constexpr (NEG) {
#pragma unroll
    for (int ri = 0; ri < NA; ++ri)
      if ((ri & rmask) == rval) {
        A.re[ri] = -A.re[ri];
        A.im[ri] = -A.im[ri];
      }
  } else {
    const auto p = c[0];
#pragma unroll
    for (int ri = 0; ri < NA; ++ri)
      if ((ri & rmask) == rval) {
        const Real r = A.re[ri], i = A.im[ri];
        cmul(p.x, p.y, r, i, A.re[ri], A.im[ri]);
      }
  }
}

template <typename Real>
__device__ __forceinline__ uint32_t diag_base(const SweepOp &op, uint64_t gbase, uint32_t jb) {
  uint32_t base = 0;
  for (int t = 0; t < op.ndt; ++t) {
    const uint32_t bit = op.dsrc[t] == kSrcGlobal ? uint32_t(gbase >> op.dpos[t]) & 1u
                                                  : (jb >> op.dpos[t]) & 1u;
    base = (base << 1) | bit;
  }
  return base;
}

template <typename Real, int NA>
__device__ __forceinline__ void apply_op(Amps<Real, NA> &A, const typename Vec2<Real>::T *coef,
                                         const SweepOp &op, uint64_t gbase, uint32_t jb) {
  // Controls outside the registers are constant for this thread.
  if ((gbase & op.gmask) != op.gval || (jb & op.lmask) != op.lval) return;
  const auto *c = coef + op.coef;
  const int rm = op.rmask, rv = op.rval;
#define SQ_CODE(kind, v, aux) case sq_op_code(kind, v, aux):
  switch (op.code) {
    SQ_CODE(kSwPhase, 0, 0) op_phase<Real, NA, false>(A, c, rm, rv); break;
    SQ_CODE(kSwPhase, 0, kAuxPure) op_phase<Real, NA, true>(A, c, rm, rv); break;
    // Variants whose register mask V reaches past the NA registers are not
    // instantiated (the planner never emits them for that register count).
#define SQ_DIAG(V)                                                                      \
  SQ_CODE(kSwDiag, V, 0) if constexpr (V < NA) op_diag<Real, NA, V>(A, c, diag_base<Real>(op, gbase, jb)); \
  break;
    SQ_DIAG(0) SQ_DIAG(1) SQ_DIAG(2) SQ_DIAG(3) SQ_DIAG(4) SQ_DIAG(5) SQ_DIAG(6) SQ_DIAG(7)
    SQ_DIAG(8) SQ_DIAG(9) SQ_DIAG(10) SQ_DIAG(11) SQ_DIAG(12) SQ_DIAG(13) SQ_DIAG(14) SQ_DIAG(15)
#undef SQ_DIAG
#define SQ_ANTI(V)                                                                            \
  SQ_CODE(kSwAnti1, V, 0) if constexpr (V < NA) op_anti1<Real, NA, V, false>(A, c, rm, rv); break; \
  SQ_CODE(kSwAnti1, V, kAuxPure) if constexpr (V < NA) op_anti1<Real, NA, V, true>(A, c, rm, rv); break;
    SQ_ANTI(1) SQ_ANTI(2) SQ_ANTI(4) SQ_ANTI(8)
#undef SQ_ANTI
#define SQ_SWAP(V)                                                                            \
  SQ_CODE(kSwSwap2, V, 0) if constexpr (V < NA) op_swap2<Real, NA, V, false>(A, c, rm, rv); break; \
  SQ_CODE(kSwSwap2, V, kAuxPure) if constexpr (V < NA) op_swap2<Real, NA, V, true>(A, c, rm, rv); break;
    SQ_SWAP(3) SQ_SWAP(5) SQ_SWAP(6) SQ_SWAP(9) SQ_SWAP(10) SQ_SWAP(12)
#undef SQ_SWAP
#define SQ_XROT(V, X)                                                                            \
  SQ_CODE(kSwXRot, V, X) if constexpr (V < NA) op_xrot<Real, NA, V, X, false>(A, c, rm, rv); break; \
  SQ_CODE(kSwXRot, V, X | kAuxImag) if constexpr (V < NA) op_xrot<Real, NA, V, X, true>(A, c, rm, rv); break;
    SQ_XROT(1, 1) SQ_XROT(2, 1) SQ_XROT(4, 1) SQ_XROT(8, 1)
    SQ_XROT(3, 1) SQ_XROT(3, 2) SQ_XROT(3, 3) SQ_XROT(5, 1) SQ_XROT(5, 2) SQ_XROT(5, 3)
    SQ_XROT(6, 1) SQ_XROT(6, 2) SQ_XROT(6, 3) SQ_XROT(9, 1) SQ_XROT(9, 2) SQ_XROT(9, 3)
    SQ_XROT(10, 1) SQ_XROT(10, 2) SQ_XROT(10, 3) SQ_XROT(12, 1) SQ_XROT(12, 2) SQ_XROT(12, 3)
#undef SQ_XROT
#define SQ_DENSE(V) SQ_CODE(kSwDense, V, 0) if constexpr (V < NA) op_dense<Real, NA, V>(A, c, rm, rv); break;
    SQ_DENSE(1) SQ_DENSE(2) SQ_DENSE(3) SQ_DENSE(4) SQ_DENSE(5) SQ_DENSE(6) SQ_DENSE(7)
    SQ_DENSE(8) SQ_DENSE(9) SQ_DENSE(10) SQ_DENSE(11) SQ_DENSE(12) SQ_DENSE(13) SQ_DENSE(14)
#undef SQ_DENSE
    // A 4-qubit dense matrix needs a second copy of all 16 amplitudes; only
    // the complex64 registers have room (the planner keeps complex128
    // 4-qubit dense gates out of sweeps).
    SQ_CODE(kSwDense, 15, 0)
      if constexpr (sizeof(Real) == 4 && NA == 16) op_dense<Real, NA, 15>(A, c, rm, rv);
      break;
    default: break;
  }
#undef SQ_CODE
}

// Tile base: the tile index with zeros inserted at every tile bit position.
__device__ __forceinline__ uint64_t tile_base(uint64_t tile, const SweepHeader &h) {
  uint64_t x = tile << h.l;
  for (uint32_t i = 0; i < h.m - h.l; ++i) x = insert_zero(x, h.hi[i]);
  return x;
}

// Asynchronous global -> shared copy of one amplitude (Ampere-style
// cp.async: no register staging, so a CTA can have its next tile in flight
// while it computes on the current one).
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem) {
  const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// Fused sweep over 2^M-amplitude tiles; 2^(M-4) threads, 16 amplitudes each,
// at least MINB CTAs per SM.
// Persistent CTAs walk the tiles with a stride of gridDim.x and keep two tile
// buffers: while the phases of tile t run on one buffer, tile t + gridDim.x
// streams into the other.
// Dynamic shared memory: 2 tiles (2 x 2^M amplitudes) | coefficients |
// high-bit address table (2^(M-L) u64).  The swizzle is XOR-linear, so the
// slot of (a ^ b) is slot(a) ^ slot(b): a thread derives all 16 slots of a
// phase from five precomputed values.
template <typename Real, int M, int MINB>
__global__ void __launch_bounds__(1 << (M - kRegBits), MINB)
    sweep_kernel(typename Vec2<Real>::T *__restrict__ psi,
                 const __grid_constant__ SweepParams<Real> P) {
  using C2 = typename Vec2<Real>::T;
  constexpr int NT = 1 << (M - kRegBits);
  constexpr uint32_t TS = 1u << M;
  constexpr uint32_t PER = TS / NT;  // amplitudes each thread copies per tile
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SweepHeader &h = P.h;
  // Low contiguous bits: the plan's (every tile holds runs of 2^L amplitudes).
  const uint32_t L = h.l;
  const uint32_t LOWMASK = (1u << L) - 1u;
  C2 *bufs = reinterpret_cast<C2 *>(smem_raw);
  C2 *coef = bufs + 2 * TS;
  uint64_t *hitab = reinterpret_cast<uint64_t *>(coef + ((h.ncoef + 1) & ~1u));
  const uint32_t tid = threadIdx.x;

  for (uint32_t i = tid; i < h.ncoef; i += NT) {
    C2 v;
    v.x = P.coef[2 * i];
    v.y = P.coef[2 * i + 1];
    coef[i] = v;
  }
  for (uint32_t c = tid; c < (1u << (M - L)); c += NT) {
    uint64_t a = 0;
    for (uint32_t i = 0; i < M - L; ++i)
      if ((c >> i) & 1) a |= uint64_t(1) << h.hi[i];
    hitab[c] = a;
  }
  __syncthreads();

  // Element j = it * NT + tid of a tile; consecutive lanes cover runs of 2^L
  // contiguous amplitudes.
  const uint32_t s_tid = swz<Real>(tid);
  auto prefetch = [&](uint64_t t, C2 *dst) {
    const uint64_t gb = tile_base(t, h);
#pragma unroll
    for (uint32_t it = 0; it < PER; ++it) {
      const uint32_t j = it * NT + tid;
      cp_async<sizeof(C2)>(dst + (s_tid ^ swz<Real>(it * NT)), psi + (gb | hitab[j >> L] | (j & LOWMASK)));
    }
  };

  const uint32_t last = h.nphases - 1;
  uint32_t cur = 0;
  if (blockIdx.x < h.num_tiles) prefetch(blockIdx.x, bufs);
  cp_async_commit();
  for (uint64_t t = blockIdx.x; t < h.num_tiles; t += gridDim.x) {
    C2 *tile = bufs + cur * TS;
    const uint64_t tn = t + gridDim.x;
    if (tn < h.num_tiles) prefetch(tn, bufs + (cur ^ 1) * TS);
    cp_async_commit();
    cp_async_wait_prev();  // this thread's copies of tile t have landed
    __syncthreads();       // ... and everyone else's
    const uint64_t gbase = tile_base(t, h);
    for (uint32_t p = 0; p <= last; ++p) {
      const SweepPhase &ph = P.ph[p];
      // Thread bits fill the non-register tile positions, ascending.
      uint32_t jb = tid;
#pragma unroll
      for (int b = 0; b < kRegBits; ++b) jb = uint32_t(insert_zero(jb, ph.reg[b]));
      const bool gstore = (p == last) && (h.flags & kDirectStore);
      // Shared-memory slots: sb ^ (selected w_b).  Register-bit values are
      // disjoint bits.
      const uint32_t sb = swz<Real>(jb);
      const uint32_t w0 = swz<Real>(1u << ph.reg[0]), w1 = swz<Real>(1u << ph.reg[1]);
      const uint32_t w2 = swz<Real>(1u << ph.reg[2]), w3 = swz<Real>(1u << ph.reg[3]);
      Amps<Real> A;
#pragma unroll
      for (int ri = 0; ri < kRegAmps; ++ri) {
        const C2 v = tile[sb ^ ((ri & 1) ? w0 : 0) ^ ((ri & 2) ? w1 : 0) ^ ((ri & 4) ? w2 : 0) ^
                          ((ri & 8) ? w3 : 0)];
        A.re[ri] = v.x;
        A.im[ri] = v.y;
      }
      for (uint32_t o = ph.op_begin; o < ph.op_end; ++o)
        apply_op<Real, kRegAmps>(A, coef, P.op[o], gbase, jb);
      if (gstore) {
        // Global index of register slot ri = tbase | selected register-bit
        // weights (disjoint bits).
        auto gw = [&](uint32_t pos) -> uint64_t {
          return pos < L ? (uint64_t(1) << pos) : (uint64_t(1) << h.hi[pos - L]);
        };
        const uint64_t tbase = gbase | hitab[jb >> L] | (jb & LOWMASK);
        const uint64_t g0 = gw(ph.reg[0]), g1 = gw(ph.reg[1]), g2 = gw(ph.reg[2]), g3 = gw(ph.reg[3]);
#pragma unroll
        for (int ri = 0; ri < kRegAmps; ++ri) {
          C2 v;
          v.x = A.re[ri];
          v.y = A.im[ri];
          psi[tbase + ((ri & 1) ? g0 : 0) + ((ri & 2) ? g1 : 0) + ((ri & 4) ? g2 : 0) +
              ((ri & 8) ? g3 : 0)] = v;
        }
      } else {
#pragma unroll
        for (int ri = 0; ri < kRegAmps; ++ri) {
          C2 v;
          v.x = A.re[ri];
          v.y = A.im[ri];
          tile[sb ^ ((ri & 1) ? w0 : 0) ^ ((ri & 2) ? w1 : 0) ^ ((ri & 4) ? w2 : 0) ^
               ((ri & 8) ? w3 : 0)] = v;
        }
        __syncthreads();
      }
    }
    if (!(h.flags & kDirectStore)) {
#pragma unroll
      for (uint32_t it = 0; it < PER; ++it) {
        const uint32_t j = it * NT + tid;
        psi[gbase | hitab[j >> L] | (j & LOWMASK)] = tile[s_tid ^ swz<Real>(it * NT)];
      }
    }
    // Everyone is done with `tile` before the next iteration prefetches into it.
    __syncthreads();
    cur ^= 1;
  }
  cp_async_wait_prev();
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// ---------------------------------------------------------------------------
// Two-state (adjoint) building blocks shared by the generic adjoint kernel
// (adjoint_kernels.cuh) and the JIT-specialised one: 8 amplitudes of phi and
// the same 8 of lambda per thread (3 register bits).
// ---------------------------------------------------------------------------
constexpr int kAdjRegBits = 3;
constexpr int kAdjAmps = 1 << kAdjRegBits;

// Inner-product contribution of one thread for a kSwInnerDiag op.
template <typename Real, int V>
__device__ __forceinline__ void inner_diag(const Amps<Real, kAdjAmps> &F, const Amps<Real, kAdjAmps> &G,
                                           const typename Vec2<Real>::T *__restrict__ c,
                                           uint32_t base, double &sr, double &si) {
  const auto *cb = c + (base << ct_popc<V>());
#pragma unroll
  for (int ri = 0; ri < kAdjAmps; ++ri) {
    const auto d = cb[ct_ext<V>(ri)];
    // K phi
    const double kr = double(d.x) * double(F.re[ri]) - double(d.y) * double(F.im[ri]);
    const double ki = double(d.x) * double(F.im[ri]) + double(d.y) * double(F.re[ri]);
    // conj(lambda) * (K phi)
    sr += double(G.re[ri]) * kr + double(G.im[ri]) * ki;
    si += double(G.re[ri]) * ki - double(G.im[ri]) * kr;
  }
}

// Inner-product contribution of one thread for a kSwInnerDense op on
// register positions V (canonical coefficient order).
template <typename Real, int V>
__device__ __forceinline__ void inner_dense(const Amps<Real, kAdjAmps> &F, const Amps<Real, kAdjAmps> &G,
                                            const typename Vec2<Real>::T *__restrict__ c, double &sr,
                                            double &si) {
  constexpr int D = 1 << ct_popc<V>();
#pragma unroll
  for (int g = 0; g < kAdjAmps; ++g) {
    if (g & V) continue;
#pragma unroll
    for (int r = 0; r < D; ++r) {
      double kr = 0.0, ki = 0.0;
#pragma unroll
      for (int x = 0; x < D; ++x) {
        const auto m = c[r * D + x];
        const int ix = g | ct_dep<V>(x);
        kr += double(m.x) * double(F.re[ix]) - double(m.y) * double(F.im[ix]);
        ki += double(m.x) * double(F.im[ix]) + double(m.y) * double(F.re[ix]);
      }
      const int ir = g | ct_dep<V>(r);
      sr += double(G.re[ir]) * kr + double(G.im[ir]) * ki;
      si += double(G.re[ir]) * ki - double(G.im[ir]) * kr;
    }
  }
}

// Inner products of ops flagged kAuxPauli, K = alpha P with P a Pauli string
// over the op's canonical local bits (the generator of a rotation gate):
// (K phi)_r = alpha (-1)^popc(r & Z) phi_(r ^ X), alpha = c[X] (row 0).  Four
// FMAs per amplitude instead of a dense K phi.
//
// Diagonal form (X = 0): canonical index (b << popc(V)) | ext_V(ri) as for
// inner_diag; Z over those bits.
template <typename Real, int V, int Z>
__device__ __forceinline__ void inner_diag_pauli(const Amps<Real, kAdjAmps> &F, const Amps<Real, kAdjAmps> &G,
                                                 const typename Vec2<Real>::T *__restrict__ c, uint32_t b,
                                                 double &sr, double &si) {
  double pr = 0.0, pi = 0.0, mr = 0.0, mi = 0.0;
#pragma unroll
  for (int ri = 0; ri < kAdjAmps; ++ri) {
    const double gr = double(G.re[ri]), gi = double(G.im[ri]);
    const double fr = double(F.re[ri]), fi = double(F.im[ri]);
    if (__popc(uint32_t(ct_ext<V>(ri) & Z)) & 1) {
      mr = fma(gr, fr, fma(gi, fi, mr));
      mi = fma(gr, fi, fma(-gi, fr, mi));
    } else {
      pr = fma(gr, fr, fma(gi, fi, pr));
      pi = fma(gr, fi, fma(-gi, fr, pi));
    }
  }
  double qr = pr - mr, qi = pi - mi;
  if (__popc(b & uint32_t(Z >> ct_popc<V>())) & 1) {
    qr = -qr;
    qi = -qi;
  }
  const auto a = c[0];
  sr += double(a.x) * qr - double(a.y) * qi;
  si += double(a.x) * qi + double(a.y) * qr;
}

// Dense form: register targets V, canonical local index r, partner r ^ X.
template <typename Real, int V, int X, int Z>
__device__ __forceinline__ void inner_dense_pauli(const Amps<Real, kAdjAmps> &F, const Amps<Real, kAdjAmps> &G,
                                                  const typename Vec2<Real>::T *__restrict__ c, double &sr,
                                                  double &si) {
  constexpr int D = 1 << ct_popc<V>();
  double pr = 0.0, pi = 0.0, mr = 0.0, mi = 0.0;
#pragma unroll
  for (int g = 0; g < kAdjAmps; ++g) {
    if (g & V) continue;
#pragma unroll
    for (int r = 0; r < D; ++r) {
      const int ir = g | ct_dep<V>(r), ix = g | ct_dep<V>(r ^ X);
      const double gr = double(G.re[ir]), gi = double(G.im[ir]);
      const double fr = double(F.re[ix]), fi = double(F.im[ix]);
      if (__popc(uint32_t(r & Z)) & 1) {
        mr = fma(gr, fr, fma(gi, fi, mr));
        mi = fma(gr, fi, fma(-gi, fr, mi));
      } else {
        pr = fma(gr, fr, fma(gi, fi, pr));
        pi = fma(gr, fi, fma(-gi, fr, pi));
      }
    }
  }
  const double qr = pr - mr, qi = pi - mi;
  const auto a = c[X];
  sr += double(a.x) * qr - double(a.y) * qi;
  si += double(a.x) * qi + double(a.y) * qr;
}

// ---------------------------------------------------------------------------
// Unfused gate: one thread per group of 2^k amplitudes (k <= 4), 64-bit
// grid-stride loop.  Only groups whose target bits are zero are enumerated,
// so every thread does work (the reference launches 2^n threads and idles all
// but 1/2^k of them).  `mat` points at the row-major matrix: the params copy,
// or device memory for cu::applyGate's literal replacement.
// ---------------------------------------------------------------------------
template <typename Real, int K>
__global__ void __launch_bounds__(256)
    gate_kernel(typename Vec2<Real>::T *__restrict__ psi,
                const __grid_constant__ GateParams<Real> P,
                const typename Vec2<Real>::T *__restrict__ dmat) {
  using C2 = typename Vec2<Real>::T;
  constexpr int D = 1 << K;
  const uint64_t ngroups = (uint64_t(1) << P.n) >> K;
  uint64_t off[D];
#pragma unroll
  for (int x = 0; x < D; ++x) {
    uint64_t o = 0;
#pragma unroll
    for (int j = 0; j < K; ++j)
      if ((x >> (K - 1 - j)) & 1) o |= uint64_t(1) << P.tbit[j];
    off[x] = o;
  }
  for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < ngroups;
       g += uint64_t(gridDim.x) * blockDim.x) {
    uint64_t base = g;
#pragma unroll
    for (int j = 0; j < K; ++j) base = insert_zero(base, P.tsorted[j]);
    if ((base & P.cmask) != P.cval) continue;
    Real ar[D], ai[D];
#pragma unroll
    for (int x = 0; x < D; ++x) {
      const C2 v = psi[base | off[x]];
      ar[x] = v.x;
      ai[x] = v.y;
    }
#pragma unroll
    for (int r = 0; r < D; ++r) {
      Real mr, mi;
      if (dmat) { const C2 mm = dmat[r * D]; mr = mm.x; mi = mm.y; }
      else { mr = P.coef[2 * (r * D)]; mi = P.coef[2 * (r * D) + 1]; }
      Real sr = mr * ar[0] - mi * ai[0];
      Real si = mr * ai[0] + mi * ar[0];
#pragma unroll
      for (int x = 1; x < D; ++x) {
        if (dmat) { const C2 mm = dmat[r * D + x]; mr = mm.x; mi = mm.y; }
        else { mr = P.coef[2 * (r * D + x)]; mi = P.coef[2 * (r * D + x) + 1]; }
        sr = fma(mr, ar[x], sr);
        sr = fma(-mi, ai[x], sr);
        si = fma(mr, ai[x], si);
        si = fma(mi, ar[x], si);
      }
      C2 o;
      o.x = sr;
      o.y = si;
      psi[base | off[r]] = o;
    }
  }
}

// Unfused gate for 4 < k <= 10: one CTA of 2^k threads per group; the group
// is staged in shared memory and thread r computes output row r from the
// TRANSPOSED matrix (mat_t[c * 2^k + r] = M[r][c], so reads coalesce) in
// device memory.
struct LargeGateParams {
  uint32_t n, k;
  uint64_t cmask, cval;
  uint8_t tbit[16];     // index bit of target j (j = 0 is the MSB)
  uint8_t tsorted[16];  // target index bits, ascending
};

template <typename Real>
__global__ void gate_kernel_large(typename Vec2<Real>::T *__restrict__ psi,
                                  const __grid_constant__ LargeGateParams P,
                                  const typename Vec2<Real>::T *__restrict__ mat_t) {
  using C2 = typename Vec2<Real>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2 *a = reinterpret_cast<C2 *>(smem_raw);
  const uint32_t k = P.k, D = 1u << k, r = threadIdx.x;
  uint64_t offr = 0;
  for (uint32_t j = 0; j < k; ++j)
    if ((r >> (k - 1 - j)) & 1) offr |= uint64_t(1) << P.tbit[j];
  const uint64_t ngroups = (uint64_t(1) << P.n) >> k;
  for (uint64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
    uint64_t base = g;
    for (uint32_t j = 0; j < k; ++j) base = insert_zero(base, P.tsorted[j]);
    if ((base & P.cmask) != P.cval) continue;  // uniform across the CTA
    a[r] = psi[base | offr];
    __syncthreads();
    const C2 m0 = mat_t[r];
    Real sr = m0.x * a[0].x - m0.y * a[0].y;
    Real si = m0.x * a[0].y + m0.y * a[0].x;
    for (uint32_t x = 1; x < D; ++x) {
      const C2 m = mat_t[uint64_t(x) * D + r];
      sr = fma(m.x, a[x].x, sr);
      sr = fma(-m.y, a[x].y, sr);
      si = fma(m.x, a[x].y, si);
      si = fma(m.y, a[x].x, si);
    }
    __syncthreads();
    C2 o;
    o.x = sr;
    o.y = si;
    psi[base | offr] = o;
  }
}

}  // namespace sq

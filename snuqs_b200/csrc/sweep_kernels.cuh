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
#include <cuda_runtime.h>
#include <stdint.h>

#include "sq_plan.h"

namespace sq {

template <typename Real> struct Vec2;
template <> struct Vec2<double> { using T = double2; };
template <> struct Vec2<float> { using T = float2; };

// Shared-memory swizzle for the amplitude tile: XOR the low W bits of the
// tile index with the fold of its higher W-bit groups.  W = log2 of the
// number of amplitudes one 128-byte shared-memory wavefront holds, so the
// lanes of a warp that differ in any three (c128) / four (c64) tile bits of
// distinct residue land in distinct banks.
template <typename Real>
__device__ __forceinline__ uint32_t swz(uint32_t j) {
  constexpr int W = sizeof(Real) == 8 ? 3 : 4;
  uint32_t x = j >> W, f = 0;
#pragma unroll
  for (int s = 0; s < 16; s += W) f ^= x >> s;
  return j ^ (f & ((1u << W) - 1u));
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

// Dense op on register positions V (canonical order: coefficient-index bit b
// <-> the b-th set bit of V).  Row r of the output is accumulated left to
// right over the columns, as the reference does.
template <typename Real, int V>
__device__ __forceinline__ void dense_op(Real (&re)[kRegAmps], Real (&im)[kRegAmps],
                                         const typename Vec2<Real>::T *__restrict__ c,
                                         int rmask, int rval, bool tok) {
  constexpr int K = ct_popc<V>();
  constexpr int D = 1 << K;
#pragma unroll
  for (int g = 0; g < kRegAmps; ++g) {
    if (g & V) continue;
    if (!(tok && ((g & rmask) == rval))) continue;
    Real ar[D], ai[D];
#pragma unroll
    for (int x = 0; x < D; ++x) {
      ar[x] = re[g | ct_dep<V>(x)];
      ai[x] = im[g | ct_dep<V>(x)];
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
      re[g | ct_dep<V>(r)] = sr;
      im[g | ct_dep<V>(r)] = si;
    }
  }
}

template <typename Real>
__device__ __forceinline__ void dense_dispatch(int v, Real (&re)[kRegAmps], Real (&im)[kRegAmps],
                                               const typename Vec2<Real>::T *c, int rmask,
                                               int rval, bool tok) {
  switch (v) {
#define SQ_CASE(V) \
  case V: dense_op<Real, V>(re, im, c, rmask, rval, tok); break;
    SQ_CASE(1) SQ_CASE(2) SQ_CASE(3) SQ_CASE(4) SQ_CASE(5) SQ_CASE(6) SQ_CASE(7)
    SQ_CASE(8) SQ_CASE(9) SQ_CASE(10) SQ_CASE(11) SQ_CASE(12) SQ_CASE(13)
    SQ_CASE(14) SQ_CASE(15)
#undef SQ_CASE
    default: break;
  }
}

// Diagonal op: coefficient index = bits of the amplitude's global index at
// the op's targets.  Global and tile-local sources are constant per thread
// in a phase; register sources vary with the register slot.
template <typename Real>
__device__ __forceinline__ void diag_op(Real (&re)[kRegAmps], Real (&im)[kRegAmps],
                                        const typename Vec2<Real>::T *__restrict__ c,
                                        const SweepOp &op, uint64_t gbase, uint32_t jb) {
  uint32_t base = 0, w0 = 0, w1 = 0, w2 = 0, w3 = 0;
  const int k = op.k;
  for (int t = 0; t < k; ++t) {
    const uint32_t wt = 1u << (k - 1 - t);
    const int src = op.dsrc[t], pos = op.dpos[t];
    if (src == kSrcGlobal) {
      if ((gbase >> pos) & 1) base |= wt;
    } else if (src == kSrcLocal) {
      if ((jb >> pos) & 1) base |= wt;
    } else {
      w0 |= pos == 0 ? wt : 0;
      w1 |= pos == 1 ? wt : 0;
      w2 |= pos == 2 ? wt : 0;
      w3 |= pos == 3 ? wt : 0;
    }
  }
#pragma unroll
  for (int ri = 0; ri < kRegAmps; ++ri) {
    const uint32_t idx = base | ((ri & 1) ? w0 : 0) | ((ri & 2) ? w1 : 0) |
                         ((ri & 4) ? w2 : 0) | ((ri & 8) ? w3 : 0);
    const auto d = c[idx];
    const Real r = re[ri], i = im[ri];
    re[ri] = d.x * r - d.y * i;
    im[ri] = d.x * i + d.y * r;
  }
}

// Tile base: the tile index with zeros inserted at every tile bit position.
__device__ __forceinline__ uint64_t tile_base(uint64_t tile, const SweepHeader &h) {
  uint64_t x = tile << h.l;
  for (uint32_t i = 0; i < h.m - h.l; ++i) x = insert_zero(x, h.hi[i]);
  return x;
}

// Fused sweep.  blockDim.x = 2^(m-4).  Dynamic shared memory: tile
// (2^m amplitudes) | coefficients | high-bit address table (2^(m-l) u64).
template <typename Real>
__global__ void __launch_bounds__(256, 2)
    sweep_kernel(typename Vec2<Real>::T *__restrict__ psi,
                 const __grid_constant__ SweepParams<Real> P) {
  using C2 = typename Vec2<Real>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SweepHeader &h = P.h;
  const uint32_t m = h.m, l = h.l;
  const uint32_t tsize = 1u << m;
  C2 *tile = reinterpret_cast<C2 *>(smem_raw);
  C2 *coef = tile + tsize;
  uint64_t *hitab = reinterpret_cast<uint64_t *>(coef + ((h.ncoef + 1) & ~1u));
  const uint32_t tid = threadIdx.x, nthr = blockDim.x;
  const uint32_t lowmask = (1u << l) - 1u;

  for (uint32_t i = tid; i < h.ncoef; i += nthr) {
    C2 v;
    v.x = P.coef[2 * i];
    v.y = P.coef[2 * i + 1];
    coef[i] = v;
  }
  for (uint32_t c = tid; c < (1u << (m - l)); c += nthr) {
    uint64_t a = 0;
    for (uint32_t i = 0; i < m - l; ++i)
      if ((c >> i) & 1) a |= uint64_t(1) << h.hi[i];
    hitab[c] = a;
  }
  __syncthreads();

  const uint32_t last = h.nphases - 1;
  for (uint64_t t = blockIdx.x; t < h.num_tiles; t += gridDim.x) {
    const uint64_t gbase = tile_base(t, h);
    if (!(h.flags & kDirectLoad)) {
#pragma unroll 4
      for (uint32_t j = tid; j < tsize; j += nthr)
        tile[swz<Real>(j)] = psi[gbase | hitab[j >> l] | (j & lowmask)];
      __syncthreads();
    }
    for (uint32_t p = 0; p <= last; ++p) {
      const SweepPhase &ph = P.ph[p];
      // Thread bits fill the non-register tile positions, ascending.
      uint32_t jb = tid;
#pragma unroll
      for (int b = 0; b < kRegBits; ++b) jb = uint32_t(insert_zero(jb, ph.reg[b]));
      const uint32_t r0 = 1u << ph.reg[0], r1 = 1u << ph.reg[1];
      const uint32_t r2 = 1u << ph.reg[2], r3 = 1u << ph.reg[3];
      Real re[kRegAmps], im[kRegAmps];
      const bool gload = (p == 0) && (h.flags & kDirectLoad);
#pragma unroll
      for (int ri = 0; ri < kRegAmps; ++ri) {
        const uint32_t j = jb | ((ri & 1) ? r0 : 0) | ((ri & 2) ? r1 : 0) |
                           ((ri & 4) ? r2 : 0) | ((ri & 8) ? r3 : 0);
        C2 v;
        if (gload)
          v = psi[gbase | hitab[j >> l] | (j & lowmask)];
        else
          v = tile[swz<Real>(j)];
        re[ri] = v.x;
        im[ri] = v.y;
      }
      for (uint32_t o = ph.op_begin; o < ph.op_end; ++o) {
        const SweepOp &op = P.op[o];
        if (op.kind == kOpDiag) {
          diag_op<Real>(re, im, coef + op.coef, op, gbase, jb);
        } else {
          const bool tok = ((gbase & op.gmask) == op.gval) && ((jb & op.lmask) == op.lval);
          dense_dispatch<Real>(op.vmask, re, im, coef + op.coef, op.rmask, op.rval, tok);
        }
      }
      const bool gstore = (p == last) && (h.flags & kDirectStore);
#pragma unroll
      for (int ri = 0; ri < kRegAmps; ++ri) {
        const uint32_t j = jb | ((ri & 1) ? r0 : 0) | ((ri & 2) ? r1 : 0) |
                           ((ri & 4) ? r2 : 0) | ((ri & 8) ? r3 : 0);
        C2 v;
        v.x = re[ri];
        v.y = im[ri];
        if (gstore)
          psi[gbase | hitab[j >> l] | (j & lowmask)] = v;
        else
          tile[swz<Real>(j)] = v;
      }
      __syncthreads();
    }
    if (!(h.flags & kDirectStore)) {
#pragma unroll 4
      for (uint32_t j = tid; j < tsize; j += nthr)
        psi[gbase | hitab[j >> l] | (j & lowmask)] = tile[swz<Real>(j)];
      __syncthreads();
    }
  }
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

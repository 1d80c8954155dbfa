// Plan structures shared by the host planner and the sm_100a kernels.
//
// A "sweep" is one read + one write of the whole state.  The state is cut
// into tiles of 2^m amplitudes; a tile holds the amplitudes whose index bits
// outside the tile's bit set S are fixed.  S always contains the l lowest
// index bits (contiguous runs of 2^l amplitudes, so loads coalesce) plus
// m - l arbitrary higher bits.  Inside a tile the sweep runs phases: in each
// phase a thread holds 16 amplitudes in registers that differ in 4 tile bits
// R (the phase's register bits) and applies every queued gate whose targets
// lie in R.  Controls and diagonal gates may sit on any index bit, inside or
// outside the tile: a thread knows the full index of every amplitude it holds.
#pragma once
#ifndef __CUDACC_RTC__
#include <stdint.h>
#endif

namespace sq {

constexpr int kRegBits = 4;                 // register bits per phase
constexpr int kRegAmps = 1 << kRegBits;     // amplitudes per thread
constexpr int kMaxTileBits = 12;            // 2^12 amplitudes per tile
constexpr int kLowBits = 5;                 // contiguous low bits in every tile
constexpr int kMaxPhases = 24;
constexpr int kMaxOps = 64;
constexpr int kMaxCoef = 1024;              // complex coefficients per sweep
constexpr int kMaxDiagK = 8;                // targets of one diagonal op
constexpr int kMaxInner = 32;               // inner-product ops per adjoint sweep

// HostOp kinds (structure analysis) ...
enum OpKind : uint8_t { kOpDense = 1, kOpDiag = 2, kOpInner = 3 };
// ... and the specialised sweep-op kinds the planner encodes them as.  The
// coefficient layout of each kind:
//   kSwDense  4^k complex, canonical row-major (matrix bit b <-> b-th set bit
//             of vmask)
//   kSwDiag   2^k complex; index = (non-register target bits) << popc(vmask)
//             | (register target bits in canonical order)
//   kSwAnti1  p0, p1:            out0 = p0 a1, out1 = p1 a0
//   kSwXRot   2^k (c_r, s_r) pairs stored as (re, im):
//             out_r = c_r a_r + f s_r a_(r^x), f = i when aux & kAuxImag
//   kSwSwap2  p12, p21:          out1 = p12 a2, out2 = p21 a1
//   kSwPhase  p:                 a *= p where the op's condition holds
//   kSwInnerDiag / kSwInnerDense (adjoint sweeps only): accumulate
//             <lambda| K |phi> into inner-product slot `slot`, K laid out as
//             kSwDiag / kSwDense; the states are not modified.
enum SweepKind : uint8_t {
  kSwDense = 1, kSwDiag = 2, kSwAnti1 = 3, kSwXRot = 4, kSwSwap2 = 5, kSwPhase = 6,
  kSwInnerDiag = 7, kSwInnerDense = 8
};
enum SweepAux : uint8_t {
  kAuxXMask = 3,  // XRot: partner XOR mask over the op's canonical local bits
  kAuxImag = 4,   // XRot: f = i
  kAuxPure = 8,   // Anti1/Swap2: unit phases (pure permutation); Phase: p = -1
  // kSwInnerDiag / kSwInnerDense: K = alpha P for one Pauli string P = X^x Z^z
  // over the op's canonical local bits (up to a phase folded into alpha):
  // bits 0-2 x, bits 3-5 z (diagonal: bits 0-2 z).  The full K coefficients
  // stay in place (the generic kernels use them); alpha is K's row-0 entry in
  // column x.
  kAuxPauli = 128,
};
enum DiagSrc : uint8_t { kSrcGlobal = 0, kSrcLocal = 1, kSrcReg = 2 };

#ifdef __CUDACC__
#define SQ_HD __host__ __device__
#else
#define SQ_HD
#endif

// Contiguous low index bits of a 2^m tile: 5 (chunks of 32 amplitudes, one
// per warp) for m >= 9; smaller tiles keep 4 free bits for the registers.
SQ_HD constexpr int sweep_low_bits(int m) { return m >= kLowBits + kRegBits ? kLowBits : m - kRegBits; }

// Tile sizes with a compiled sweep kernel, per precision (ascending).
constexpr int kTileBitsC128[] = {4, 7, 10, 11, 12};
constexpr int kTileBitsC64[] = {4, 7, 10, 12};
constexpr int kDefaultTileBitsC128 = 11;
// Batched-circuit kernel tile sizes (a circuit of n <= this many qubits stays
// in shared memory).
constexpr int kBatchTileBitsC128 = 11;
constexpr int kBatchTileBitsC64 = 12;
// Two-state adjoint sweeps (twice the shared memory per tile).
constexpr int kAdjTileBitsC128[] = {4, 7, 10};
constexpr int kAdjTileBitsC64[] = {4, 7, 11};
constexpr int kDefaultTileBitsC64 = 12;

// Flat dispatch code of a sweep op: one switch in the kernel selects the
// fully specialised routine (kind, register positions, partner mask, flags).
SQ_HD constexpr int sq_log2_4(int v) { return v == 1 ? 0 : v == 2 ? 1 : v == 4 ? 2 : 3; }
SQ_HD constexpr int sq_pair_index(int v) {  // two-bit masks of 4 positions
  return v == 3 ? 0 : v == 5 ? 1 : v == 6 ? 2 : v == 9 ? 3 : v == 10 ? 4 : 5;
}
SQ_HD constexpr int sq_op_code(int kind, int v, int aux) {
  return kind == kSwPhase ? 1 + ((aux & kAuxPure) ? 1 : 0)
         : kind == kSwDiag ? 16 + v
         : kind == kSwAnti1 ? 32 + sq_log2_4(v) + ((aux & kAuxPure) ? 4 : 0)
         : kind == kSwSwap2 ? 40 + sq_pair_index(v) + ((aux & kAuxPure) ? 6 : 0)
         : kind == kSwXRot
             ? 52 + 2 * ((v & (v - 1)) == 0 ? sq_log2_4(v) : 4 + 3 * sq_pair_index(v) + (aux & 3) - 1) +
                   ((aux & kAuxImag) ? 1 : 0)
         : kind == kSwInnerDiag  ? 112 + v
         : kind == kSwInnerDense ? 128 + v
                                 : 96 + v;  // kSwDense
}
// kRemap: the sweep stores tile position p to global bit out[p] instead of
// the bit it was loaded from (a permutation of the tile's bits), so that the
// following sweeps find their most used qubits on the low, always-resident
// index bits.
enum SweepFlags : uint32_t { kDirectLoad = 1u, kDirectStore = 2u, kRemap = 4u };

struct SweepOp {
  uint8_t kind;    // SweepKind
  uint8_t k;       // number of targets
  uint8_t vmask;   // register positions of the targets (bit p = register bit p)
  uint8_t rmask;   // register positions that are controls / phase conditions
  uint8_t rval;    //        and their required values
  uint8_t aux;     // SweepAux flags
  uint8_t ndt;     // kSwDiag: number of non-register targets (dsrc/dpos)
  uint8_t code;    // sq_op_code(kind, vmask, aux)
  uint32_t coef;   // offset of the op's coefficients (complex units)
  uint32_t lmask;  // in-tile, non-register control bits (tile-local index)
  uint32_t lval;
  uint32_t slot;   // kSwInner*: inner-product slot within the sweep
  uint64_t gmask;  // control bits outside the tile (global index)
  uint64_t gval;
  // kSwDiag: the non-register targets, most significant first: each from a
  // global bit or a tile-local bit; `ndt` of them.
  uint8_t dsrc[kMaxDiagK];
  uint8_t dpos[kMaxDiagK];
};

struct SweepPhase {
  uint8_t reg[kRegBits];  // tile positions of the register bits, ascending
  uint16_t op_begin, op_end;
};

struct SweepHeader {
  uint32_t n;        // qubits of the state
  uint32_t m;        // tile bits (threads per tile = 2^(m-4))
  uint32_t l;        // low contiguous bits
  uint32_t nphases;
  uint32_t ncoef;    // complex coefficients used
  uint32_t flags;    // SweepFlags
  uint64_t num_tiles;
  uint8_t hi[kMaxTileBits];  // global bit of tile position l+i, ascending
  uint8_t out[kMaxTileBits]; // kRemap: global bit tile position p is stored to
  uint8_t pad[8];
};

template <typename Real>
struct SweepParams {
  SweepHeader h;
  SweepPhase ph[kMaxPhases];
  SweepOp op[kMaxOps];
  Real coef[2 * kMaxCoef];  // interleaved re/im
};

// Unfused single-gate kernel parameters (k <= 4 keeps the matrix here).
constexpr int kSmallK = 4;
template <typename Real>
struct GateParams {
  uint32_t n, k;
  uint64_t cmask, cval;                // control bits (global index)
  uint8_t tbit[16];                    // index bit of target j (j = 0 is the MSB)
  uint8_t tsorted[16];                 // target index bits, ascending
  Real coef[2 * (1 << (2 * kSmallK))];  // row-major matrix
};

}  // namespace sq

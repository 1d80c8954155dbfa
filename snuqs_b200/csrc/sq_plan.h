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
#include <stdint.h>

namespace sq {

constexpr int kRegBits = 4;                 // register bits per phase
constexpr int kRegAmps = 1 << kRegBits;     // amplitudes per thread
constexpr int kMaxTileBits = 12;            // 2^12 amplitudes per tile
constexpr int kLowBits = 5;                 // contiguous low bits in every tile
constexpr int kMaxPhases = 24;
constexpr int kMaxOps = 64;
constexpr int kMaxCoef = 1024;              // complex coefficients per sweep
constexpr int kMaxDiagK = 8;                // targets of one diagonal op

enum OpKind : uint8_t { kOpDense = 1, kOpDiag = 2 };
enum DiagSrc : uint8_t { kSrcGlobal = 0, kSrcLocal = 1, kSrcReg = 2 };
enum SweepFlags : uint32_t { kDirectLoad = 1u, kDirectStore = 2u };

struct SweepOp {
  uint8_t kind;    // kOpDense / kOpDiag
  uint8_t k;       // number of targets
  uint8_t vmask;   // dense: register positions of the targets (bit p = register bit p)
  uint8_t rmask;   // dense: register positions that are controls
  uint8_t rval;    //        and their required values
  uint8_t pad0[3];
  uint32_t coef;   // offset of the op's coefficients (complex units)
  uint32_t lmask;  // dense: in-tile, non-register control bits (tile-local index)
  uint32_t lval;
  uint32_t pad1;
  uint64_t gmask;  // dense: control bits outside the tile (global index)
  uint64_t gval;
  // diag: target t (t = 0 is the most significant bit of the coefficient
  // index) comes from a global bit, a tile-local bit or a register bit.
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
  uint8_t pad[4];
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

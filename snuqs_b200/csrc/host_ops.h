// Host-side gate representation, gate-matrix factory and fusion planner.
#pragma once
#include <complex>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "sq_plan.h"

namespace sq {

using cplx = std::complex<double>;

// Matrix of gate `gate` (sq_gate id) into m (4^k entries, row-major).
// Returns k, or -1 for an unknown gate / wrong angle count.
int gate_matrix(int gate, const double *angles, uint32_t nangles, std::vector<cplx> &m);
int gate_qubits(int gate);
int gate_num_angles(int gate);
// d/d angle[param] of gate_matrix(gate, angles) (analytic).  Returns k, or -1
// for a gate without that parameter.
int gate_matrix_derivative(int gate, const double *angles, uint32_t nangles, int param,
                           std::vector<cplx> &m);

// One queued gate after qubit -> index-bit translation.
//   kind kOpDense: m is 4^k row-major, tbits[0] is the MSB of its index.
//   kind kOpDiag:  m is the 2^k diagonal.
// Controls (cmask/cval, index bits) apply to dense ops; diagonal ops fold
// their controls into the diagonal.
struct HostOp {
  uint8_t kind = kOpDense;  // kOpDense / kOpDiag / kOpInner
  // kOpInner (adjoint): accumulate <lambda| K |phi> into inner-product slot
  // `slot`; K is m (dense 4^k, or the 2^k diagonal when inner_diag).
  bool inner_diag = false;
  uint32_t slot = 0;
  std::vector<int> tbits;
  uint64_t cmask = 0, cval = 0;
  std::vector<cplx> m;
  uint64_t target_mask() const;
  uint64_t touched_mask() const;  // targets + controls
  uint64_t nondiag_mask() const;  // bits acted on non-diagonally
};

// Structure analysis of a dense matrix on `tbits` with controls: peels off
// exact control qubits, detects exactly diagonal matrices and drops exact
// identities.  Entries are compared exactly (== 0, == 1), so the result
// applies the same products as the full matrix minus exact zeros.
// Returns false when the op is an exact identity (nothing to apply).
bool analyse_op(const std::vector<cplx> &m, const std::vector<int> &tbits, uint64_t cmask,
                uint64_t cval, HostOp &out);

// How a planned sweep was formed, so that the same gate sequence with other
// values (other angles) is re-emitted without planning (rebuild_plan): the
// tile bits, every phase's register bits and first op, and the position of
// each of the sweep's ops in the planner's input.  Empty `src`: not
// rebuildable (a sweep of a remapping plan).
struct SweepRecipe {
  uint64_t S = 0;
  std::vector<uint64_t> phase_regs;
  std::vector<uint32_t> phase_first;
  std::vector<uint32_t> src;
  uint32_t reg_bits = 0, max_dense_k = 0;
};

// A planned launch: a fused sweep, or one unfused gate.
struct PlannedSweep {
  SweepHeader h;
  std::vector<SweepPhase> ph;
  std::vector<SweepOp> op;
  std::vector<cplx> coef;
  uint32_t ngates = 0;  // queued ops it carries
  // Adjoint sweeps: global inner-product slot of each local slot 0, 1, ...
  std::vector<uint32_t> inner_global;
  SweepRecipe recipe;
};

struct PlannedLaunch {
  bool is_sweep = true;
  PlannedSweep sweep;
  HostOp gate;  // unfused gate (dense, any k; cmask/cval are its controls)
  uint32_t gate_src = 0;  // its position in the planner's input
};

struct PlanOptions {
  uint32_t tile_bits = kMaxTileBits;
  bool reorder = true;
  // Widest dense gate a sweep may carry in registers: 3 for complex128 (a
  // 4-qubit dense matrix needs a second copy of all 16 amplitudes), 4 for
  // complex64.  Wider dense gates run unfused.
  uint32_t max_dense_k = 3;
  // Register bits per phase: 4 (16 amplitudes per thread, the sweep kernel)
  // or 3 (8 amplitudes per state per thread, the two-state adjoint kernel).
  uint32_t reg_bits = kRegBits;
  // Low index bits every tile contains (contiguous runs of 2^low_bits
  // amplitudes per global access); 0: sweep_low_bits(tile bits).
  uint32_t low_bits = 0;
  // Most ops one sweep carries (fusion width in gates); 0: kMaxOps.
  uint32_t max_ops = 0;
  // Tile selection and phase scheduling (needs reorder): 1 = choose each
  // sweep's tile bits to absorb the most upcoming gates and order the gates
  // of a sweep into the fewest register phases; 0 = take gates first come
  // first served; -1 = 1 for states of >= kSelectMinQubits qubits.
  int select = -1;
  // Qubit remapping (needs select): a sweep may store its tile with the low
  // index bits exchanged for tile bits that the next sweep uses most, so the
  // low bits every tile must hold carry hot qubits; the plan ends with the
  // original bit order (a last restoring permutation, merged into the last
  // sweep when its tile holds every moved bit).  Only the JIT-specialised
  // sweep kernels implement the permuted store.
  bool remap = false;
};
constexpr uint32_t kSelectMinQubits = 18;

// Low bits the engine plans with by default: runs of 128 bytes (8 complex128
// / 16 complex64 amplitudes) when the state spans several tiles of m bits;
// 0 (the planner's own default) otherwise.
inline uint32_t auto_low_bits(bool c64, uint32_t n, uint32_t m) {
  const uint32_t lb = n > m ? (c64 ? 4u : 3u) : 0u;
  return lb && lb + uint32_t(kRegBits) <= m ? lb : 0u;
}

// The plan options a plan depends on, packed into one word (a cache key).
inline uint64_t plan_options_key(const PlanOptions &o) {
  return uint64_t(o.tile_bits) | (uint64_t(o.low_bits) << 8) | (uint64_t(o.max_dense_k) << 16) |
         (uint64_t(o.reg_bits) << 24) | (uint64_t(o.max_ops) << 32) | (uint64_t(o.reorder) << 48) |
         (uint64_t(o.remap) << 49) | (uint64_t(uint8_t(o.select)) << 50);
}

// Packs ops (in circuit order) into fused sweeps for an n-qubit state.
std::vector<PlannedLaunch> plan_sweeps(const std::vector<HostOp> &ops, uint32_t n,
                                       const PlanOptions &opt);

// The op structure a plan depends on: per op its kind, targets, controls and
// inner-product slot, not its values.  Two op lists with equal signatures
// can share one plan's recipes.
std::vector<uint64_t> op_signature(const std::vector<HostOp> &ops);
// Two independent 64-bit FNV-1a hashes of op_signature(ops).
std::pair<uint64_t, uint64_t> op_signature_hash(const std::vector<HostOp> &ops);

// Re-emits `plan` (made by plan_sweeps for ops of the same signature) for
// `ops`: every sweep rebuilt from its recipe with the new values.  False,
// leaving `plan` unusable, when a sweep has no recipe or when a rebuilt
// sweep's header, phases or ops differ from the old ones (a value that changes
// an op's form, e.g. an angle that makes a dense gate a permutation); the
// caller then plans anew.
bool rebuild_plan(std::vector<PlannedLaunch> &plan, const std::vector<HostOp> &ops, uint32_t n);
// One sweep of such a plan from its recipe (m, l: its tile and low bits);
// false when the recipe is empty or names an op past `ops`.
bool rebuild_sweep(const SweepRecipe &r, const std::vector<HostOp> &ops, uint32_t n, uint32_t m, uint32_t l,
                   PlannedSweep &out);

}  // namespace sq

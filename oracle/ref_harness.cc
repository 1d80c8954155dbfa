/*
 * TEST ORACLE ONLY.  A C-callable harness around the reference's own CPU gate
 * path, compiled from the reference sources where they lie (see
 * oracle/Makefile) into oracle/_ref/libsnuqs_ref.so.  Only tests/, the smoke
 * check and bench.py's CPU-baseline leg load it, always as the checker or the
 * timed CPU baseline, never as the product.
 *
 * Reference interfaces wrapped here:
 *   - gate constructors and matrices: src/braket/snuqs/csrc/operation/gate_operations.cc:9-734
 *   - GateOperation::ptr():           src/braket/snuqs/csrc/operation/operation.cc:118
 *   - cpu::applyGate:                 src/braket/snuqs/csrc/operation/gate_operations_impl_cpu.cc:131-148
 *   - cpu::initializeBasis_Z:         src/braket/snuqs/csrc/operation/initialization_impl_cpu.cc:15-22
 *   - functionals::apply (CPU branch) src/braket/snuqs/csrc/functionals/functionals.cc:15-21
 */
#include <omp.h>

#include <complex>
#include <cstring>
#include <memory>
#include <vector>

#include "operation/gate_operations.h"
#include "operation/gate_operations_impl_cpu.h"
#include "operation/initialization_impl_cpu.h"

namespace {

// Builds the reference gate object for GateOperationType `type`
// (operation.h:17-52 order), or nullptr for an unknown type.
std::unique_ptr<GateOperation> make_gate(int type,
                                         const std::vector<size_t> &t,
                                         const double *a) {
  const std::vector<size_t> c;  // ctrl_modifiers: unused by every kernel
  const size_t p = 1;           // power: unused by every kernel
  switch (static_cast<GateOperationType>(type)) {
    case GateOperationType::Identity: return std::make_unique<Identity>(t, c, p);
    case GateOperationType::Hadamard: return std::make_unique<Hadamard>(t, c, p);
    case GateOperationType::PauliX: return std::make_unique<PauliX>(t, c, p);
    case GateOperationType::PauliY: return std::make_unique<PauliY>(t, c, p);
    case GateOperationType::PauliZ: return std::make_unique<PauliZ>(t, c, p);
    case GateOperationType::CX: return std::make_unique<CX>(t, c, p);
    case GateOperationType::CY: return std::make_unique<CY>(t, c, p);
    case GateOperationType::CZ: return std::make_unique<CZ>(t, c, p);
    case GateOperationType::S: return std::make_unique<S>(t, c, p);
    case GateOperationType::Si: return std::make_unique<Si>(t, c, p);
    case GateOperationType::T: return std::make_unique<T>(t, c, p);
    case GateOperationType::Ti: return std::make_unique<Ti>(t, c, p);
    case GateOperationType::V: return std::make_unique<V>(t, c, p);
    case GateOperationType::Vi: return std::make_unique<Vi>(t, c, p);
    case GateOperationType::PhaseShift: return std::make_unique<PhaseShift>(t, a[0], c, p);
    case GateOperationType::CPhaseShift: return std::make_unique<CPhaseShift>(t, a[0], c, p);
    case GateOperationType::CPhaseShift00: return std::make_unique<CPhaseShift00>(t, a[0], c, p);
    case GateOperationType::CPhaseShift01: return std::make_unique<CPhaseShift01>(t, a[0], c, p);
    case GateOperationType::CPhaseShift10: return std::make_unique<CPhaseShift10>(t, a[0], c, p);
    case GateOperationType::RotX: return std::make_unique<RotX>(t, a[0], c, p);
    case GateOperationType::RotY: return std::make_unique<RotY>(t, a[0], c, p);
    case GateOperationType::RotZ: return std::make_unique<RotZ>(t, a[0], c, p);
    case GateOperationType::Swap: return std::make_unique<Swap>(t, c, p);
    case GateOperationType::ISwap: return std::make_unique<ISwap>(t, c, p);
    case GateOperationType::PSwap: return std::make_unique<PSwap>(t, a[0], c, p);
    case GateOperationType::XY: return std::make_unique<XY>(t, a[0], c, p);
    case GateOperationType::XX: return std::make_unique<XX>(t, a[0], c, p);
    case GateOperationType::YY: return std::make_unique<YY>(t, a[0], c, p);
    case GateOperationType::ZZ: return std::make_unique<ZZ>(t, a[0], c, p);
    case GateOperationType::CCNot: return std::make_unique<CCNot>(t, c, p);
    case GateOperationType::CSwap: return std::make_unique<CSwap>(t, c, p);
    case GateOperationType::U: return std::make_unique<U>(t, a[0], a[1], a[2], c, p);
    case GateOperationType::GPhase: return std::make_unique<GPhase>(t, a[0], c, p);
    case GateOperationType::SwapA2A: return std::make_unique<SwapA2A>(t, c, p);
  }
  return nullptr;
}

}  // namespace

extern "C" {

// Copies the reference matrix of gate `type` acting on `k` targets into
// `out` (row-major, interleaved re/im, 4^k complex).  Returns 0 on success.
int ref_gate_matrix(int type, const double *angles, size_t k, double *out) {
  std::vector<size_t> t(k);
  for (size_t i = 0; i < k; ++i) t[i] = i;
  auto g = make_gate(type, t, angles);
  if (!g) return -1;
  std::memcpy(out, g->ptr(), g->num_elems() * sizeof(std::complex<double>));
  return 0;
}

// functionals::apply, CPU branch: builds the gate and runs cpu::applyGate on
// a host state of 2^nqubits complex128 amplitudes.
int ref_apply_gate(double *state, size_t nqubits, int type,
                   const size_t *targets, size_t k, const double *angles) {
  std::vector<size_t> t(targets, targets + k);
  auto g = make_gate(type, t, angles);
  if (!g) return -1;
  cpu::applyGate(state, g->ptr(), t, nqubits, size_t(1) << nqubits);
  return 0;
}

// cpu::applyGate with a caller-supplied matrix (k in 0..3).
int ref_apply_matrix(double *state, size_t nqubits, const double *matrix,
                     const size_t *targets, size_t k) {
  if (k > 3) return -1;
  std::vector<size_t> t(targets, targets + k);
  cpu::applyGate(state, const_cast<double *>(matrix), t, nqubits,
                 size_t(1) << nqubits);
  return 0;
}

void ref_initialize_basis_z(double *state, size_t nqubits) {
  cpu::initializeBasis_Z(state, size_t(1) << nqubits);
}

int ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"

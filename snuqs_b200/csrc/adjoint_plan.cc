// Host side of the adjoint gradient: turns a parametrised circuit into the
// forward op list and the reverse (adjoint) op list the planner packs into
// two-state sweeps.
//
// Reverse pass, for gates l = L..1 with phi = psi_l and lambda_l =
// U_(l+1)^dagger ... U_L^dagger H psi:
//   for each parametrised angle a of gate l:
//     slot += <lambda_l| K |phi>,  K = (dU_l/da) U_l^dagger
//   phi <- U_l^dagger phi;  lambda <- U_l^dagger lambda
// and dE/da = 2 Re(slot).  (dE/da = 2 Re <lambda_l| dU_l/da |psi_(l-1)> and
// psi_(l-1) = U_l^dagger psi_l.)
#include "adjoint_plan.h"

#include <cstring>
#include <stdexcept>

namespace sq {

namespace {

std::vector<cplx> op_matrix(const sq_circuit_op &op) {
  std::vector<cplx> m;
  if (op.gate < 0) {
    const size_t d = size_t(1) << op.k;
    m.resize(d * d);
    std::memcpy(m.data(), op.matrix, d * d * sizeof(cplx));
    return m;
  }
  if (gate_matrix(op.gate, op.angles, op.nangles, m) < 0)
    throw std::invalid_argument("adjoint: bad gate or angle count");
  return m;
}

std::vector<cplx> dagger(const std::vector<cplx> &a, int d) {
  std::vector<cplx> c(size_t(d) * d);
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) c[size_t(j) * d + i] = std::conj(a[size_t(i) * d + j]);
  return c;
}

std::vector<cplx> matmul(const std::vector<cplx> &a, const std::vector<cplx> &b, int d) {
  std::vector<cplx> c(size_t(d) * d, cplx(0, 0));
  for (int i = 0; i < d; ++i)
    for (int k = 0; k < d; ++k) {
      const cplx x = a[size_t(i) * d + k];
      if (x == cplx(0, 0)) continue;
      for (int j = 0; j < d; ++j) c[size_t(i) * d + j] += x * b[size_t(k) * d + j];
    }
  return c;
}

std::vector<int> index_bits(const sq_circuit_op &op, uint32_t n) {
  std::vector<int> tb;
  for (uint32_t j = 0; j < op.k; ++j) tb.push_back(int(n - 1 - op.qubits[j]));
  return tb;
}

}  // namespace

void build_adjoint(const sq_circuit_op *ops, uint32_t nops, uint32_t n, AdjointPlan &out) {
  out = AdjointPlan();
  for (uint32_t i = 0; i < nops; ++i) {
    const sq_circuit_op &op = ops[i];
    if (op.k > 3) throw std::invalid_argument("adjoint: gates act on at most 3 qubits");
    if (op.gate < 0 && !op.matrix) throw std::invalid_argument("adjoint: null matrix");
    uint64_t seen = 0;
    for (uint32_t j = 0; j < op.k; ++j) {
      if (op.qubits[j] >= n || ((seen >> op.qubits[j]) & 1))
        throw std::invalid_argument("adjoint: bad or repeated qubit");
      seen |= uint64_t(1) << op.qubits[j];
    }
    if (op.gate >= 0 && gate_qubits(op.gate) != int(op.k))
      throw std::invalid_argument("adjoint: qubit count does not match the gate");
    const std::vector<cplx> m = op_matrix(op);
    HostOp h;
    if (analyse_op(m, index_bits(op, n), 0, 0, h)) out.forward.push_back(h);
  }
  for (uint32_t i = nops; i-- > 0;) {
    const sq_circuit_op &op = ops[i];
    const int d = 1 << op.k;
    const std::vector<cplx> m = op_matrix(op);
    const std::vector<cplx> md = dagger(m, d);
    if (op.gate >= 0) {
      const uint32_t na = uint32_t(gate_num_angles(op.gate));
      for (uint32_t a = 0; a < na && a < 3; ++a) {
        if (op.param[a] < 0) continue;
        std::vector<cplx> dm;
        if (gate_matrix_derivative(op.gate, op.angles, op.nangles, int(a), dm) < 0)
          throw std::invalid_argument("adjoint: gate has no derivative for that angle");
        std::vector<cplx> K = matmul(dm, md, d);
        HostOp ip;
        ip.kind = kOpInner;
        ip.tbits = index_bits(op, n);
        bool diag = true;
        for (int r = 0; r < d; ++r)
          for (int c = 0; c < d; ++c)
            if (r != c && K[size_t(r) * d + c] != cplx(0, 0)) diag = false;
        ip.inner_diag = diag;
        if (diag) {
          ip.m.resize(d);
          for (int r = 0; r < d; ++r) ip.m[r] = K[size_t(r) * d + r];
        } else {
          ip.m = K;
        }
        ip.slot = uint32_t(out.occurrences.size());
        out.occurrences.push_back({op.param[a], op.scale[a]});
        out.reverse.push_back(ip);
      }
    }
    HostOp h;
    if (analyse_op(md, index_bits(op, n), 0, 0, h)) out.reverse.push_back(h);
  }
}

}  // namespace sq

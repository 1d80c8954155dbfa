// Adjoint-gradient op lists (see adjoint_plan.cc).
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

#include "../../include/snuqs_b200.h"
#include "host_ops.h"

namespace sq {

struct AdjointPlan {
  std::vector<HostOp> forward;  // U_1 .. U_L
  std::vector<HostOp> reverse;  // inner products and U_l^dagger, l = L .. 1
  // Inner-product slot s feeds parameter occurrences[s].first with chain
  // factor occurrences[s].second.
  std::vector<std::pair<int32_t, double>> occurrences;
};

// Throws std::invalid_argument on a malformed circuit.
void build_adjoint(const sq_circuit_op *ops, uint32_t nops, uint32_t n, AdjointPlan &out);

}  // namespace sq

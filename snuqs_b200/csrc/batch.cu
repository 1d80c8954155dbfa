// Batched circuits: host side of sq_batch_* (include/snuqs_b200.h).
//
// sq_batch_run plans every circuit (in parallel on the host), packs the plans
// into one pinned buffer, and replays a CUDA graph that uploads the plans and
// the circuit table, resets the work counter, runs the persistent
// batch_kernel once and downloads the energies.  The graph is re-captured
// only when a buffer size changes, so a VQE loop that only changes angles
// replays the same graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/snuqs_b200.h"
#include "adjoint_plan.h"
#include "batch_kernels.cuh"
#include "host_ops.h"
#include "jit.h"
#include "jit_kernels.cuh"
#include "sweep_registry.h"

int sq_detail_fail(int code, const char *msg);

using sq::cplx;

namespace {

int fail(int code, const std::string &m) { return sq_detail_fail(code, m.c_str()); }

#define SQB_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return fail(e_ == cudaErrorMemoryAllocation ? SQ_ERR_OOM : SQ_ERR_CUDA,                   \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                          \
  } while (0)

struct Circ {
  uint32_t n = 0, ham = 0;
  std::vector<sq_circuit_op> ops;
  std::vector<std::vector<cplx>> fixed;  // copies of fixed matrices
};

// Device buffer that grows.
struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return SQ_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    SQB_CUDA(cudaMalloc(&p, bytes));
    cap = bytes;
    return SQ_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

struct HostBuf {
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return SQ_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    SQB_CUDA(cudaHostAlloc(&p, bytes, cudaHostAllocDefault));
    cap = bytes;
    return SQ_OK;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// One sweep of a structure group: its multi-state JIT kernel, dynamic shared
// memory, resident CTAs per SM, coefficient count, and the byte offset of its
// coefficients within a circuit's packed plan.
struct MultiSweep {
  const void *fn = nullptr;
  size_t smem = 0;
  int per_sm = 1;
  uint32_t ncoef = 0;
  uint64_t coef_at = 0;
};

// Streamed circuits whose plans differ only in coefficient values: their
// states lie back to back in the pool and their packed plans back to back in
// the plan buffer (table positions first .. first + count - 1), and each
// sweep runs as one multi-state launch over all of them.
struct MultiGroup {
  uint32_t n = 0, count = 0, first = 0;
  uint64_t pool_off = 0, plan_off = 0, rec_bytes = 0;
  std::vector<MultiSweep> sweeps;
  // The first sweep starts every state from |0...0> itself (no init pass,
  // no first read).
  bool zero_first = false;
};

}  // namespace

struct sq_batch {
  int dtype = SQ_C128;
  int device = 0;
  int keep = 0;
  std::vector<sq::PauliParams> hams;
  std::vector<uint32_t> ham_n;
  std::vector<Circ> circs;
  DevBuf d_pool, d_plans, d_table, d_hams, d_energy, d_counter, d_occ, d_def, d_part;
  HostBuf h_plans, h_table, h_energy, h_occ, h_def;
  std::vector<uint32_t> deferred;  // table positions whose energy the grid-wide pass computes
  uint32_t nitems = 0;              // work items of that pass
  size_t def_words = 0;             // staged words: deferred circuits, item offsets
  size_t hams_uploaded = 0;
  std::vector<uint64_t> state_off;  // per circuit id; ~0 when not kept
  std::vector<uint32_t> order;      // sorted position -> circuit id
  cudaGraphExec_t graph = nullptr;
  size_t graph_plan_bytes = 0, graph_ncirc = 0;
  void *graph_stream = nullptr;
  uint32_t graph_grid = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  uint32_t last_ctas = 0;
  const void *graph_fn = nullptr;
  bool last_jit = false;  // the last gradient run used the JIT kernel
  // Launch configuration (0 = default): tile bits, low bits of a streamed
  // tile, ops per sweep, CTAs per SM.
  uint32_t tile_bits = 0, low_bits = 0, max_ops = 0, ctas_per_sm = 0;
  // Energy-run plan cache: valid while the circuits and the plan settings
  // are those it was made for.
  uint64_t version = 0, planned_version = ~uint64_t(0);
  uint32_t planned_m = 0, planned_l = 0, planned_ops = 0;
  size_t planned_bytes = 0;
  // Plan statistics of the streamed circuits (n > tile bits) of the last
  // energy plan: count, fused sweeps, and their algorithmic HBM bytes (each
  // sweep reads and writes the state, the energy pass reads it once).
  uint64_t stat_streamed = 0, stat_sweeps = 0, stat_bytes = 0;
  // Structure groups of the last energy plan (run by multi-state JIT sweeps)
  // and the table positions [0, n_interp) that batch_kernel runs.
  std::vector<MultiGroup> groups;
  uint32_t n_interp = 0;
  // Angle changes (sq_batch_set_angles) bump values_version only: the next
  // energy run re-emits each circuit's plan from its sweep recipes with the
  // new coefficients (no planning) when the ops keep their signature.
  uint64_t values_version = 0, planned_values = 0;
  std::vector<std::vector<sq::SweepRecipe>> recipes;    // per circuit id
  std::vector<std::pair<uint64_t, uint64_t>> sigs;      // per circuit id
  std::vector<uint64_t> plan_at, plan_size;             // packed plan in h_plans, per circuit id
};

namespace {

// Pauli-string sum -> grouped expectation parameters (as sq_expect_pauli).
int build_pauli(uint32_t n, const char *paulis, const double *w, uint32_t nt, sq::PauliParams &P) {
  if (nt > uint32_t(sq::kMaxTerms)) return fail(SQ_ERR_UNSUPPORTED, "batch: > 1024 Pauli terms");
  std::vector<uint64_t> xm(nt), zym(nt);
  std::vector<int> ny(nt);
  for (uint32_t t = 0; t < nt; ++t)
    for (uint32_t q = 0; q < n; ++q) {
      const uint64_t bit = uint64_t(1) << (n - 1 - q);
      switch (paulis[size_t(t) * n + q]) {
        case 'I': case 'i': break;
        case 'X': case 'x': xm[t] |= bit; break;
        case 'Y': case 'y': xm[t] |= bit; zym[t] |= bit; ny[t]++; break;
        case 'Z': case 'z': zym[t] |= bit; break;
        default: return fail(SQ_ERR_INVALID, "batch: bad Pauli character");
      }
    }
  std::vector<uint32_t> idx(nt);
  for (uint32_t i = 0; i < nt; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
    if (xm[a] != xm[b]) return xm[a] < xm[b];
    return (ny[a] & 1) < (ny[b] & 1);
  });
  std::memset(&P, 0, sizeof(P));
  P.n = n;
  uint32_t k = 0;
  for (uint32_t pos = 0; pos < nt;) {
    uint32_t end = pos;
    while (end < nt && xm[idx[end]] == xm[idx[pos]] && (ny[idx[end]] & 1) == (ny[idx[pos]] & 1)) ++end;
    if (P.ngroups >= uint32_t(sq::kMaxGroups))
      return fail(SQ_ERR_UNSUPPORTED, "batch: > 256 Pauli groups");
    sq::PauliGroup &g = P.g[P.ngroups++];
    g.x = xm[idx[pos]];
    g.odd = ny[idx[pos]] & 1;
    g.t0 = k;
    for (uint32_t e = pos; e < end; ++e) {
      const uint32_t t = idx[e];
      P.zy[k] = zym[t];
      P.f[k] = w[t] * (((ny[t] / 2) & 1) ? -1.0 : 1.0);
      ++k;
    }
    g.t1 = k;
    pos = end;
  }
  return SQ_OK;
}

template <typename Real>
void pack_sweep(const sq::PlannedSweep &ps, std::vector<unsigned char> &out) {
  using C2 = typename sq::Vec2<Real>::T;
  sq::PackedSweep hdr;
  std::memset(&hdr, 0, sizeof(hdr));
  hdr.h = ps.h;
  hdr.nops = uint32_t(ps.op.size());
  hdr.phase_off = uint32_t(align16(sizeof(hdr)));
  hdr.op_off = uint32_t(align16(hdr.phase_off + ps.ph.size() * sizeof(sq::SweepPhase)));
  hdr.coef_off = uint32_t(align16(hdr.op_off + ps.op.size() * sizeof(sq::SweepOp)));
  hdr.bytes = uint32_t(align16(hdr.coef_off + ps.coef.size() * sizeof(C2)));
  if (!ps.inner_global.empty()) {
    hdr.inner_off = hdr.bytes;
    hdr.bytes = uint32_t(align16(hdr.inner_off + (1 + ps.inner_global.size()) * sizeof(uint32_t)));
  }
  const size_t base = out.size();
  out.resize(base + hdr.bytes, 0);
  unsigned char *r = out.data() + base;
  std::memcpy(r, &hdr, sizeof(hdr));
  std::memcpy(r + hdr.phase_off, ps.ph.data(), ps.ph.size() * sizeof(sq::SweepPhase));
  std::memcpy(r + hdr.op_off, ps.op.data(), ps.op.size() * sizeof(sq::SweepOp));
  C2 *c = reinterpret_cast<C2 *>(r + hdr.coef_off);
  for (size_t i = 0; i < ps.coef.size(); ++i) {
    c[i].x = Real(ps.coef[i].real());
    c[i].y = Real(ps.coef[i].imag());
  }
  if (hdr.inner_off) {
    uint32_t *g = reinterpret_cast<uint32_t *>(r + hdr.inner_off);
    g[0] = uint32_t(ps.inner_global.size());
    for (size_t i = 0; i < ps.inner_global.size(); ++i) g[1 + i] = ps.inner_global[i];
  }
}

// Plans one circuit into packed sweeps; returns the sweep count or < 0.
// Plans shared between the circuits of one structure within one planning
// pass (many parameter sets of one ansatz): the first circuit of a structure
// (op signature, qubits, plan options) is planned, the others re-emit its
// plan with their own values (sq::rebuild_plan), and fall back to planning
// when that fails.
struct PlanShare {
  using Key = std::tuple<uint64_t, uint64_t, uint64_t, uint32_t>;
  std::mutex mu;
  std::map<Key, std::shared_ptr<const std::vector<sq::PlannedLaunch>>> plans;

  std::vector<sq::PlannedLaunch> plan(const std::vector<sq::HostOp> &ops, uint32_t n, const sq::PlanOptions &opt) {
    const auto sig = sq::op_signature_hash(ops);
    const Key key{sig.first, sig.second, sq::plan_options_key(opt), n};
    std::shared_ptr<const std::vector<sq::PlannedLaunch>> have;
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = plans.find(key);
      if (it != plans.end()) have = it->second;
    }
    if (have) {
      std::vector<sq::PlannedLaunch> p = *have;
      if (sq::rebuild_plan(p, ops, n)) return p;
    }
    std::vector<sq::PlannedLaunch> p = sq::plan_sweeps(ops, n, opt);
    std::lock_guard<std::mutex> lk(mu);
    plans.emplace(key, std::make_shared<const std::vector<sq::PlannedLaunch>>(p));
    return p;
  }
};

// A circuit's gates as planner ops (identities dropped).  False with `err`.
bool circuit_host_ops(const Circ &c, std::vector<sq::HostOp> &ops, std::string &err) {
  ops.clear();
  for (const auto &op : c.ops) {
    std::vector<cplx> mat;
    if (op.gate < 0) {
      const size_t d = size_t(1) << op.k;
      mat.resize(d * d);
      std::memcpy(mat.data(), op.matrix, d * d * sizeof(cplx));
    } else if (sq::gate_matrix(op.gate, op.angles, op.nangles, mat) < 0) {
      err = "batch: bad gate or angle count";
      return false;
    }
    std::vector<int> tb;
    for (uint32_t j = 0; j < op.k; ++j) tb.push_back(int(c.n - 1 - op.qubits[j]));
    sq::HostOp h;
    if (sq::analyse_op(mat, tb, 0, 0, h)) ops.push_back(h);
  }
  return true;
}

std::pair<uint64_t, uint64_t> signature_hash(const std::vector<sq::HostOp> &ops) {
  return sq::op_signature_hash(ops);
}

// Plans one circuit of an energy run into packed sweeps.  recipes / sig (when
// given): the sweeps' recipes and the ops' signature hash, for re-emitting the
// plan when only angles change.
template <typename Real>
int plan_circuit(const Circ &c, uint32_t m, uint32_t low_bits, uint32_t max_ops,
                 std::vector<unsigned char> &out, std::string &err, int select = -1,
                 std::vector<sq::SweepRecipe> *recipes = nullptr, std::pair<uint64_t, uint64_t> *sig = nullptr,
                 PlanShare *share = nullptr) {
  try {
    std::vector<sq::HostOp> ops;
    if (!circuit_host_ops(c, ops, err)) return -1;
    if (sig) *sig = signature_hash(ops);
    if (recipes) recipes->clear();
    sq::PlanOptions opt;
    opt.tile_bits = m;
    opt.max_dense_k = sizeof(Real) == 4 ? 4 : 3;
    opt.max_ops = max_ops;
    opt.select = select;
    // Low bits matter only for a state streamed through tiles (n > m).
    if (low_bits && c.n > m && low_bits + uint32_t(sq::kRegBits) <= m) opt.low_bits = low_bits;
    const auto plan = share ? share->plan(ops, c.n, opt) : sq::plan_sweeps(ops, c.n, opt);
    int sweeps = 0;
    for (const auto &pl : plan) {
      if (!pl.is_sweep) {
        err = "batch: a gate wider than a sweep's registers (use the single-state API)";
        return -1;
      }
      pack_sweep<Real>(pl.sweep, out);
      if (recipes) recipes->push_back(pl.sweep.recipe);
      ++sweeps;
    }
    return sweeps;
  } catch (const std::exception &e) {
    err = std::string("batch planner: ") + e.what();
    return -1;
  }
}

// Byte ranges of the coefficient values in a packed plan.
template <typename Real>
std::vector<std::pair<size_t, size_t>> coef_ranges(const std::vector<unsigned char> &p) {
  using C2 = typename sq::Vec2<Real>::T;
  std::vector<std::pair<size_t, size_t>> holes;
  for (size_t off = 0; off < p.size();) {
    const auto &ps = *reinterpret_cast<const sq::PackedSweep *>(p.data() + off);
    holes.emplace_back(off + ps.coef_off, off + ps.coef_off + size_t(ps.h.ncoef) * sizeof(C2));
    off += ps.bytes;
  }
  return holes;
}

// Packed plans a and b are equal except for coefficient values (`holes`:
// a's coefficient ranges).
bool same_structure(const std::vector<unsigned char> &a, const std::vector<unsigned char> &b,
                    const std::vector<std::pair<size_t, size_t>> &holes) {
  if (a.size() != b.size()) return false;
  size_t pos = 0;
  for (const auto &h : holes) {
    if (std::memcmp(a.data() + pos, b.data() + pos, h.first - pos) != 0) return false;
    pos = h.second;
  }
  return std::memcmp(a.data() + pos, b.data() + pos, a.size() - pos) == 0;
}

// Hash of a packed plan's bytes outside its coefficient ranges, and of n.
std::pair<uint64_t, uint64_t> structure_key(const std::vector<unsigned char> &p,
                                            const std::vector<std::pair<size_t, size_t>> &holes, uint32_t n) {
  uint64_t a = 1469598103934665603ull ^ n, b = 0x9ae16a3b2f90404full + n;
  auto mix = [&](size_t from, size_t to) {
    for (size_t i = from; i < to; ++i) {
      a = (a ^ p[i]) * 1099511628211ull;
      b = (b ^ p[i]) * 0x100000001b3ull + 0x9e3779b97f4a7c15ull;
    }
  };
  size_t pos = 0;
  for (const auto &h : holes) {
    mix(pos, h.first);
    pos = h.second;
  }
  mix(pos, p.size());
  return {a, b ^ p.size()};
}

// The sweeps of a packed plan (structure only: coefficients are left zero)
// and the byte offset of each sweep's coefficients.
std::vector<sq::PlannedSweep> unpack_sweeps(const std::vector<unsigned char> &p, std::vector<uint64_t> &coef_at) {
  std::vector<sq::PlannedSweep> out;
  coef_at.clear();
  for (size_t off = 0; off < p.size();) {
    const auto &rec = *reinterpret_cast<const sq::PackedSweep *>(p.data() + off);
    sq::PlannedSweep ps;
    ps.h = rec.h;
    const auto *ph = reinterpret_cast<const sq::SweepPhase *>(p.data() + off + rec.phase_off);
    const auto *op = reinterpret_cast<const sq::SweepOp *>(p.data() + off + rec.op_off);
    ps.ph.assign(ph, ph + rec.h.nphases);
    ps.op.assign(op, op + rec.nops);
    ps.coef.assign(rec.h.ncoef, cplx(0.0, 0.0));
    out.push_back(std::move(ps));
    coef_at.push_back(off + rec.coef_off);
    off += rec.bytes;
  }
  return out;
}

// Tile selection for the circuits of structure groups (PlanOptions::select):
// on at every size (a group streams K states, so its sweeps behave as those
// of one large state): fewer sweeps (VQE ansatz, 15-17 qubits, complex128:
// 8/9/11 -> 6/8/8) and first and last phases that move data straight between
// HBM and registers.  SQ_BATCH_SELECT=-1 leaves it to the planner's size rule.
int multi_select() {
  const char *e = std::getenv("SQ_BATCH_SELECT");
  return e && *e ? std::atoi(e) : 1;
}

// Multi-state JIT sweeps for the energy runs: on unless SQ_JIT=0 or
// SQ_BATCH_MULTI=0, and only with NVRTC present.
bool multi_enabled() {
  const char *j = std::getenv("SQ_JIT");
  const char *m = std::getenv("SQ_BATCH_MULTI");
  if ((j && j[0] == '0') || (m && m[0] == '0')) return false;
  return sq::jit_available();
}

// Energy kernel of (precision, tile bits); nullptr when not compiled.
template <typename Real>
const void *batch_fn(uint32_t m) {
  if constexpr (sizeof(Real) == 8) {
    switch (m) {
      case 10: return SQ_BATCH_PTR_NAME(double, 10)();
      case 11: return SQ_BATCH_PTR_NAME(double, 11)();
      case 12: return SQ_BATCH_PTR_NAME(double, 12)();
    }
  } else {
    switch (m) {
      case 10: return SQ_BATCH_PTR_NAME(float, 10)();
      case 11: return SQ_BATCH_PTR_NAME(float, 11)();
      case 12: return SQ_BATCH_PTR_NAME(float, 12)();
    }
  }
  return nullptr;
}

// Gradient kernel of (precision, tile bits); nullptr when not compiled.
template <typename Real>
const void *batch_adj_fn(uint32_t m) {
  if constexpr (sizeof(Real) == 8) {
    switch (m) {
      case 10: return SQ_BATCH_ADJ_PTR_NAME(double, 10)();
      case 11: return SQ_BATCH_ADJ_PTR_NAME(double, 11)();
    }
  } else {
    switch (m) {
      case 11: return SQ_BATCH_ADJ_PTR_NAME(float, 11)();
      case 12: return SQ_BATCH_ADJ_PTR_NAME(float, 12)();
    }
  }
  return nullptr;
}

template <typename Real>
uint32_t batch_default_bits() {
  return uint32_t(sizeof(Real) == 4 ? sq::kBatchTileBitsC64 : sq::kBatchTileBitsC128);
}

template <typename Real>
uint32_t batch_tile_bits(const sq_batch *b) {
  return b->tile_bits ? b->tile_bits : uint32_t(sizeof(Real) == 4 ? sq::kBatchTileBitsC64 : sq::kBatchTileBitsC128);
}

// Threads, dynamic shared memory and resident CTAs per SM of the energy
// kernel for tile bits m.
template <typename Real>
int batch_shape(uint32_t m, const void *&fn, int &threads, size_t &smem, int &per_sm) {
  using C2 = typename sq::Vec2<Real>::T;
  fn = batch_fn<Real>(m);
  if (!fn) return fail(SQ_ERR_INVALID, "batch: no kernel for " + std::to_string(m) + " tile bits");
  const uint32_t L = uint32_t(sq::sweep_low_bits(int(m)));
  // The high-bit table is sized for the smallest low-bit count a plan may use (3).
  smem = 2 * (size_t(1) << m) * sizeof(C2) + size_t(sq::kMaxCoef) * sizeof(C2) +
         (size_t(1) << (m - std::min<uint32_t>(L, 3))) * sizeof(uint64_t);
  threads = 1 << (m - sq::kRegBits);
  SQB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  SQB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
  per_sm = std::max(per_sm, 1);
  return SQ_OK;
}

// Re-emits every circuit's packed plan (in the pinned staging buffer) for
// its current angles from the sweep recipes of the last planning.  False
// when a circuit's ops changed signature or a rebuilt sweep changed form (the
// caller then plans every circuit anew).
template <typename Real>
bool refresh_values(sq_batch *b) {
  const size_t nc = b->circs.size();
  if (b->recipes.size() != nc || b->sigs.size() != nc || b->plan_at.size() != nc || !b->h_plans.p) return false;
  unsigned char *hp = static_cast<unsigned char *>(b->h_plans.p);
  std::atomic<size_t> next{0};
  std::atomic<bool> ok{true};
  auto work = [&] {
    std::vector<sq::HostOp> ops;
    std::vector<unsigned char> packed, old;
    std::string err;
    for (size_t i = next++; i < nc && ok; i = next++) {
      const Circ &c = b->circs[i];
      if (!circuit_host_ops(c, ops, err) || signature_hash(ops) != b->sigs[i]) {
        ok = false;
        break;
      }
      old.assign(hp + b->plan_at[i], hp + b->plan_at[i] + b->plan_size[i]);
      packed.clear();
      size_t off = 0;
      bool good = true;
      for (const sq::SweepRecipe &r : b->recipes[i]) {
        if (off + sizeof(sq::PackedSweep) > old.size()) {
          good = false;
          break;
        }
        const auto &rec = *reinterpret_cast<const sq::PackedSweep *>(old.data() + off);
        sq::PlannedSweep ps;
        if (!sq::rebuild_sweep(r, ops, c.n, rec.h.m, rec.h.l, ps)) {
          good = false;
          break;
        }
        pack_sweep<Real>(ps, packed);
        off += rec.bytes;
      }
      if (!good || packed.size() != old.size() || !same_structure(old, packed, coef_ranges<Real>(old))) {
        ok = false;
        break;
      }
      std::memcpy(hp + b->plan_at[i], packed.data(), packed.size());
    }
  };
  const unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < nth; ++t) pool.emplace_back(work);
  for (auto &th : pool) th.join();
  return ok;
}

template <typename Real>
int run_impl(sq_batch *b, double *energies, cudaStream_t st) {
  using C2 = typename sq::Vec2<Real>::T;
  const uint32_t M = batch_tile_bits<Real>(b);
  const size_t nc = b->circs.size();
  if (nc == 0) return SQ_OK;
  const void *fn = nullptr;
  int threads = 0, per_sm = 0;
  size_t smem = 0;
  if (int s = batch_shape<Real>(M, fn, threads, smem, per_sm)) return s;
  bool replan = b->planned_version != b->version || b->planned_m != M || b->planned_l != b->low_bits ||
                b->planned_ops != b->max_ops;
  // Only angles changed: new coefficients into the same plans, else plan anew.
  if (!replan && b->planned_values != b->values_version) {
    if (refresh_values<Real>(b)) b->planned_values = b->values_version;
    else replan = true;
  }
  size_t plan_bytes = b->planned_bytes;
  if (replan) {
  b->planned_values = b->values_version;
  b->deferred.clear();
  int sms = 0;
  SQB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  // Candidates for multi-state JIT sweeps: streamed circuits, planned with
  // the default tile, low-bit and fusion settings (so the autotuner's trials
  // reuse the same compiled kernels); the rest with the batch's settings.
  const uint32_t MJ = batch_default_bits<Real>();
  const bool multi = multi_enabled();
  std::vector<char> cand(nc, 0);
  for (size_t i = 0; i < nc; ++i) cand[i] = multi && b->circs[i].n > std::max(M, MJ);
  // Plan all circuits in parallel.
  std::vector<std::vector<unsigned char>> packed(nc);
  std::vector<int> nsweeps(nc, 0);
  std::vector<std::string> errs(nc);
  std::atomic<size_t> next{0};
  const unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  PlanShare share;
  auto plan_all = [&](const std::vector<uint32_t> &ids) {
    next = 0;
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < std::min<size_t>(nth, ids.size()); ++t)
      pool.emplace_back([&]() {
        for (size_t k = next++; k < ids.size(); k = next++) {
          const uint32_t i = ids[k];
          packed[i].clear();
          nsweeps[i] = cand[i] ? plan_circuit<Real>(b->circs[i], MJ, 0, 0, packed[i], errs[i], multi_select(),
                                                    &b->recipes[i], &b->sigs[i], &share)
                               : plan_circuit<Real>(b->circs[i], M, b->low_bits, b->max_ops, packed[i], errs[i], -1,
                                                    &b->recipes[i], &b->sigs[i], &share);
        }
      });
    for (auto &th : pool) th.join();
  };
  b->recipes.assign(nc, {});
  b->sigs.assign(nc, {0, 0});
  {
    std::vector<uint32_t> all(nc);
    for (size_t i = 0; i < nc; ++i) all[i] = uint32_t(i);
    plan_all(all);
  }
  for (size_t i = 0; i < nc; ++i)
    if (nsweeps[i] < 0) return fail(SQ_ERR_UNSUPPORTED, errs[i]);
  // Structure groups among the candidates.  A group needs at least two
  // tiles per SM in total and a compiled kernel for every sweep; candidates
  // left out are planned again with the batch's settings.
  b->groups.clear();
  std::vector<int> group_of(nc, -1);
  {
    std::map<std::pair<uint64_t, uint64_t>, std::vector<uint32_t>> by_key;
    for (size_t i = 0; i < nc; ++i)
      if (cand[i] && nsweeps[i] > 0)
        by_key[structure_key(packed[i], coef_ranges<Real>(packed[i]), b->circs[i].n)].push_back(uint32_t(i));
    std::vector<std::vector<uint32_t>> members;
    std::vector<std::vector<sq::PlannedSweep>> gsweeps;
    std::vector<std::vector<uint64_t>> gcoef;
    for (auto &kv : by_key) {
      const auto &ids = kv.second;
      const auto holes = coef_ranges<Real>(packed[ids[0]]);
      std::vector<uint32_t> same;
      for (uint32_t i : ids)
        if (b->circs[i].n == b->circs[ids[0]].n && same_structure(packed[ids[0]], packed[i], holes))
          same.push_back(i);
      const uint32_t n = b->circs[ids[0]].n;
      if ((uint64_t(same.size()) << (n - MJ)) < 2 * uint64_t(sms)) continue;
      members.push_back(same);
      gcoef.emplace_back();
      gsweeps.push_back(unpack_sweeps(packed[ids[0]], gcoef.back()));
    }
    // The first sweep of a group in its from-|0...0> form where it has one.
    std::vector<const sq::PlannedSweep *> todo, zero;
    std::vector<char> zero_ok(gsweeps.size(), 0);
    for (size_t g = 0; g < gsweeps.size(); ++g)
      for (size_t k = 0; k < gsweeps[g].size(); ++k) {
        const sq::PlannedSweep &ps = gsweeps[g][k];
        if (k == 0 && !sq::jit_body(ps, sizeof(Real) == 4, sq::jit_minb(sizeof(Real) == 4, ps.h.m), true, true)
                           .empty()) {
          zero_ok[g] = 1;
          zero.push_back(&ps);
        } else {
          todo.push_back(&ps);
        }
      }
    sq::jit_prepare_multi(todo, sizeof(Real) == 4, zero);
    for (size_t g = 0; g < members.size(); ++g) {
      MultiGroup G;
      G.n = b->circs[members[g][0]].n;
      G.count = uint32_t(members[g].size());
      G.rec_bytes = packed[members[g][0]].size();
      bool ok = true;
      for (size_t k = 0; k < gsweeps[g].size() && ok; ++k) {
        const sq::PlannedSweep &ps = gsweeps[g][k];
        MultiSweep w;
        std::string err;
        if (k == 0 && zero_ok[g]) {
          w.fn = sq::jit_msweep_kernel(ps, sizeof(Real) == 4, err, true);
          G.zero_first = w.fn != nullptr;
        }
        if (!w.fn) w.fn = sq::jit_msweep_kernel(ps, sizeof(Real) == 4, err);
        w.smem = sq::jit_msweep_smem(ps, sizeof(Real) == 4);
        w.ncoef = ps.h.ncoef;
        w.coef_at = gcoef[g][k];
        ok = w.fn != nullptr &&
             cudaFuncSetAttribute(w.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(w.smem)) == cudaSuccess &&
             cudaOccupancyMaxActiveBlocksPerMultiprocessor(&w.per_sm, w.fn, 1 << (MJ - sq::kRegBits), w.smem) ==
                 cudaSuccess;
        if (!ok) cudaGetLastError();
        w.per_sm = std::max(w.per_sm, 1);
        G.sweeps.push_back(w);
      }
      if (!ok) continue;
      for (uint32_t i : members[g]) group_of[i] = int(b->groups.size());
      b->groups.push_back(std::move(G));
    }
    std::vector<uint32_t> again;
    for (size_t i = 0; i < nc; ++i)
      if (cand[i] && group_of[i] < 0) {
        cand[i] = 0;
        again.push_back(uint32_t(i));
      }
    if (!again.empty()) {
      plan_all(again);
      for (uint32_t i : again)
        if (nsweeps[i] < 0) return fail(SQ_ERR_UNSUPPORTED, errs[i]);
    }
  }
  b->stat_streamed = b->stat_sweeps = b->stat_bytes = 0;
  for (size_t i = 0; i < nc; ++i)
    if (b->circs[i].n > M || group_of[i] >= 0) {
      b->stat_streamed++;
      b->stat_sweeps += uint64_t(nsweeps[i]);
      // A group whose first sweep starts from |0...0> does not read the state there.
      const bool zf = group_of[i] >= 0 && b->groups[size_t(group_of[i])].zero_first;
      b->stat_bytes += (2 * uint64_t(nsweeps[i]) + 1 - (zf ? 1 : 0)) * (uint64_t(1) << b->circs[i].n) * sizeof(C2);
    }
  // Table order: the circuits batch_kernel runs, largest first (its dynamic
  // work queue), then each structure group's circuits together.
  b->order.clear();
  for (size_t i = 0; i < nc; ++i)
    if (group_of[i] < 0) b->order.push_back(uint32_t(i));
  std::stable_sort(b->order.begin(), b->order.end(), [&](uint32_t x, uint32_t y) {
    const uint64_t cx = (uint64_t(1) << b->circs[x].n) * (uint64_t(nsweeps[x]) + 1);
    const uint64_t cy = (uint64_t(1) << b->circs[y].n) * (uint64_t(nsweeps[y]) + 1);
    return cx > cy;
  });
  b->n_interp = uint32_t(b->order.size());
  for (size_t g = 0; g < b->groups.size(); ++g) {
    b->groups[g].first = uint32_t(b->order.size());
    for (size_t i = 0; i < nc; ++i)
      if (group_of[i] == int(g)) b->order.push_back(uint32_t(i));
  }
  // State pool: circuits that do not fit one tile, or whose state is kept
  // (in table order, so a group's states lie back to back).
  b->state_off.assign(nc, ~uint64_t(0));
  uint64_t pool_amps = 0;
  for (uint32_t id : b->order) {
    const Circ &c = b->circs[id];
    if (c.n > M || b->keep || group_of[id] >= 0) {
      b->state_off[id] = pool_amps;
      pool_amps += uint64_t(1) << c.n;
    }
  }
  plan_bytes = 0;
  for (size_t i = 0; i < nc; ++i) plan_bytes += packed[i].size();
  SQB_CUDA(cudaSetDevice(b->device));
  if (int s = b->d_pool.ensure(std::max<uint64_t>(pool_amps, 1) * sizeof(C2))) return s;
  if (int s = b->d_plans.ensure(plan_bytes + 16)) return s;
  if (int s = b->h_plans.ensure(plan_bytes + 16)) return s;
  if (int s = b->d_table.ensure(nc * sizeof(sq::BatchCircuit))) return s;
  if (int s = b->h_table.ensure(nc * sizeof(sq::BatchCircuit))) return s;
  if (int s = b->d_energy.ensure(nc * sizeof(double))) return s;
  if (int s = b->h_energy.ensure(nc * sizeof(double))) return s;
  if (int s = b->d_counter.ensure(sizeof(unsigned))) return s;
  if (b->hams_uploaded != b->hams.size()) {
    if (int s = b->d_hams.ensure(b->hams.size() * sizeof(sq::PauliParams))) return s;
    SQB_CUDA(cudaMemcpy(b->d_hams.p, b->hams.data(), b->hams.size() * sizeof(sq::PauliParams),
                        cudaMemcpyHostToDevice));
    b->hams_uploaded = b->hams.size();
  }
  // Pinned staging: packed plans and the sorted table.
  auto *tab = static_cast<sq::BatchCircuit *>(b->h_table.p);
  unsigned char *hp = static_cast<unsigned char *>(b->h_plans.p);
  size_t off = 0;
  b->plan_at.assign(nc, 0);
  b->plan_size.assign(nc, 0);
  for (size_t pos = 0; pos < nc; ++pos) {
    const uint32_t id = b->order[pos];
    const Circ &c = b->circs[id];
    std::memcpy(hp + off, packed[id].data(), packed[id].size());
    b->plan_at[id] = off;
    b->plan_size[id] = packed[id].size();
    sq::BatchCircuit &t = tab[pos];
    t.n = c.n;
    t.nsweeps = uint32_t(nsweeps[id]);
    t.ham = c.ham;
    t.keep = b->keep ? 1u : 0u;
    t.state_off = b->state_off[id] == ~uint64_t(0) ? 0 : b->state_off[id];
    t.plan_off = off;
    t.nrev = 0;
    t.lam_off = t.occ_off = 0;
    // A streamed state (n > M) leaves its energy to the grid-wide pass.
    t.defer = c.n > M || group_of[id] >= 0 ? 1u : 0u;
    if (t.defer) b->deferred.push_back(uint32_t(pos));
    off += packed[id].size();
  }
  for (auto &G : b->groups) {
    G.pool_off = tab[G.first].state_off;
    G.plan_off = tab[G.first].plan_off;
  }
  // Work items of the energy pass: chunks of 2^kEnergyChunkBits pairs.
  // Staged as [deferred | item_off (ndef+1)]; the kernel finds an item's
  // circuit by binary search over item_off.
  {
    std::vector<uint32_t> item_off{0};
    for (uint32_t k = 0; k < b->deferred.size(); ++k) {
      const uint32_t n = tab[b->deferred[k]].n;
      const uint32_t chunks = n - 1 > sq::kEnergyChunkBits ? 1u << (n - 1 - sq::kEnergyChunkBits) : 1u;
      item_off.push_back(item_off.back() + chunks);
    }
    b->nitems = item_off.back();
    std::vector<uint32_t> staged(b->deferred);
    staged.insert(staged.end(), item_off.begin(), item_off.end());
    b->def_words = staged.size();
    if (int s = b->d_def.ensure(staged.size() * sizeof(uint32_t))) return s;
    if (int s = b->h_def.ensure(staged.size() * sizeof(uint32_t))) return s;
    std::memcpy(b->h_def.p, staged.data(), staged.size() * sizeof(uint32_t));
  }
    // Staging buffers may have moved: the graph is captured again.
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->planned_version = b->version;
    b->planned_m = M;
    b->planned_l = b->low_bits;
    b->planned_ops = b->max_ops;
    b->planned_bytes = plan_bytes;
  }  // replan
  // Kernel configuration.
  int sms = 0;
  SQB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  const int cps = b->ctas_per_sm ? std::min<int>(per_sm, int(b->ctas_per_sm)) : per_sm;
  const uint32_t grid =
      uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(b->n_interp, uint64_t(cps) * uint64_t(sms))));
  if (!b->ev0) {
    SQB_CUDA(cudaEventCreate(&b->ev0));
    SQB_CUDA(cudaEventCreate(&b->ev1));
  }
  // Grid-wide energy pass over the streamed states: 4 blocks per SM.
  uint32_t ndef = uint32_t(b->deferred.size());
  const uint32_t egrid = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(b->nitems, uint64_t(sms) * 8)));
  if (int s = b->d_part.ensure(std::max<size_t>(b->nitems, 1) * sizeof(double))) return s;
  // (Re)capture the graph when sizes or the stream changed.
  if (!b->graph || b->graph_plan_bytes != plan_bytes || b->graph_ncirc != nc ||
      b->graph_stream != st || b->graph_grid != grid || b->graph_fn != fn) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    cudaStream_t cs;
    SQB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    sq::BatchParams P;
    std::memset(&P, 0, sizeof(P));
    P.circuits = static_cast<const sq::BatchCircuit *>(b->d_table.p);
    P.plans = static_cast<const unsigned char *>(b->d_plans.p);
    P.hams = static_cast<const sq::PauliParams *>(b->d_hams.p);
    P.ncircuits = b->n_interp;
    P.counter = static_cast<unsigned *>(b->d_counter.p);
    P.energies = static_cast<double *>(b->d_energy.p);
    C2 *poolp = static_cast<C2 *>(b->d_pool.p);
    void *args[] = {&poolp, &P};
    cudaGraph_t g;
    auto capture = [&]() -> int {
      SQB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      cudaMemcpyAsync(b->d_plans.p, b->h_plans.p, plan_bytes, cudaMemcpyHostToDevice, cs);
      cudaMemcpyAsync(b->d_table.p, b->h_table.p, nc * sizeof(sq::BatchCircuit),
                      cudaMemcpyHostToDevice, cs);
      cudaMemsetAsync(b->d_counter.p, 0, sizeof(unsigned), cs);
      // External event nodes, so the kernel's device time can be read back.
      cudaEventRecordWithFlags(b->ev0, cs, cudaEventRecordExternal);
      if (b->n_interp) cudaLaunchKernel(fn, dim3(grid), dim3(threads), args, smem, cs);
      // Structure groups: |0...0> in every state, then one launch per sweep.
      const uint32_t MJ = batch_default_bits<Real>();
      for (const MultiGroup &G : b->groups) {
        C2 *gpsi = poolp + G.pool_off;
        const uint64_t total = uint64_t(G.count) << G.n;
        const uint32_t ig = uint32_t(std::min<uint64_t>((total + 255) / 256, uint64_t(sms) * 8));
        if (!G.zero_first) sq::batch_group_init<Real><<<ig, 256, 0, cs>>>(gpsi, total, G.n);
        for (const MultiSweep &w : G.sweeps) {
          sq::MultiParams Q;
          Q.coefs = static_cast<const unsigned char *>(b->d_plans.p) + G.plan_off + w.coef_at;
          Q.stride = G.rec_bytes;
          Q.tile_shift = G.n - MJ;
          Q.tiles = uint64_t(G.count) << Q.tile_shift;
          Q.ncoef = w.ncoef;
          const uint64_t mg = std::min<uint64_t>(Q.tiles, uint64_t(w.per_sm) * uint64_t(sms));
          void *margs[] = {&gpsi, &Q};
          cudaLaunchKernel(w.fn, dim3(unsigned(mg)), dim3(1u << (MJ - sq::kRegBits)), margs, w.smem, cs);
        }
      }
      if (ndef) {
        cudaMemcpyAsync(b->d_def.p, b->h_def.p, b->def_words * sizeof(uint32_t), cudaMemcpyHostToDevice, cs);
        const uint32_t *defp = static_cast<const uint32_t *>(b->d_def.p);
        const uint32_t *offp = defp + ndef;
        double *partp = static_cast<double *>(b->d_part.p);
        const C2 *cpool = poolp;
        uint32_t nitems = b->nitems;
        void *gargs[] = {&cpool, &P, &defp, &offp, &ndef, &nitems, &partp};
        cudaLaunchKernel(reinterpret_cast<const void *>(&sq::batch_energy_grid<Real>), dim3(egrid),
                         dim3(sq::kReduceThreads), gargs, 0, cs);
        sq::batch_energy_finalize<<<ndef, sq::kReduceThreads, 0, cs>>>(partp, offp, defp, P.energies);
      }
      cudaEventRecordWithFlags(b->ev1, cs, cudaEventRecordExternal);
      cudaMemcpyAsync(b->h_energy.p, b->d_energy.p, nc * sizeof(double), cudaMemcpyDeviceToHost, cs);
      SQB_CUDA(cudaStreamEndCapture(cs, &g));
      return SQ_OK;
    };
    const int s1 = capture();
    cudaStreamDestroy(cs);
    if (s1 != SQ_OK) return s1;
    const cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(SQ_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    b->graph_plan_bytes = plan_bytes;
    b->graph_ncirc = nc;
    b->graph_stream = st;
    b->graph_grid = grid;
    b->graph_fn = fn;
  }
  SQB_CUDA(cudaGraphLaunch(b->graph, st));
  SQB_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f;
  SQB_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  b->last_ms = ms;
  b->last_ctas = grid;
  const double *he = static_cast<const double *>(b->h_energy.p);
  for (size_t pos = 0; pos < nc; ++pos) energies[b->order[pos]] = he[pos];
  return SQ_OK;
}

// Plans one circuit of a gradient run: forward sweeps then reverse two-state
// sweeps (adjoint_plan.cc), packed back to back.  Returns false with `err`.
template <typename Real>
bool plan_gradient_circuit(const Circ &c, uint32_t m, std::vector<unsigned char> &out, uint32_t &nfwd,
                           uint32_t &nrev, std::vector<std::pair<int32_t, double>> &occ, std::string &err,
                           PlanShare *share = nullptr) {
  try {
    sq::AdjointPlan ap;
    sq::build_adjoint(c.ops.data(), uint32_t(c.ops.size()), c.n, ap);
    sq::PlanOptions fopt;
    fopt.tile_bits = m;
    fopt.max_dense_k = sizeof(Real) == 4 ? 4 : 3;
    sq::PlanOptions ropt;
    ropt.tile_bits = m;
    ropt.reg_bits = sq::kAdjRegBits;
    ropt.max_dense_k = sq::kAdjRegBits;
    const auto fplan = share ? share->plan(ap.forward, c.n, fopt) : sq::plan_sweeps(ap.forward, c.n, fopt);
    const auto rplan = share ? share->plan(ap.reverse, c.n, ropt) : sq::plan_sweeps(ap.reverse, c.n, ropt);
    nfwd = nrev = 0;
    for (const auto &pl : fplan) {
      if (!pl.is_sweep) {
        err = "batch: a gate wider than a sweep's registers (use the single-state API)";
        return false;
      }
      pack_sweep<Real>(pl.sweep, out);
      ++nfwd;
    }
    for (const auto &pl : rplan) {
      if (!pl.is_sweep) {
        err = "batch: a gate wider than a reverse sweep's registers (use sq_adjoint_gradient)";
        return false;
      }
      pack_sweep<Real>(pl.sweep, out);
      ++nrev;
    }
    occ = ap.occurrences;
    return true;
  } catch (const std::exception &e) {
    err = std::string("batch gradient planner: ") + e.what();
    return false;
  }
}

// True when every circuit streams its states (n > M) and all packed plans are
// identical except for their coefficient values (SQ_JIT=0 turns the JIT path
// off).
template <typename Real>
bool uniform_plans(const sq_batch *b, const std::vector<std::vector<unsigned char>> &packed,
                   const std::vector<uint32_t> &nfwd, const std::vector<uint32_t> &nrev,
                   const std::vector<std::vector<std::pair<int32_t, double>>> &occs, uint32_t M) {
  const char *env = std::getenv("SQ_JIT");
  if ((env && env[0] == '0') || !sq::jit_available() || b->circs.empty()) return false;
  const size_t nc = b->circs.size();
  const uint32_t n = b->circs[0].n;
  if (n <= M) return false;
  const std::vector<unsigned char> &p0 = packed[0];
  const auto holes = coef_ranges<Real>(p0);
  for (size_t i = 1; i < nc; ++i)
    if (b->circs[i].n != n || nfwd[i] != nfwd[0] || nrev[i] != nrev[0] || occs[i] != occs[0] ||
        !same_structure(p0, packed[i], holes))
      return false;
  return true;
}

template <typename Real>
int run_gradient_impl(sq_batch *b, uint32_t n_params, double *energies, double *grads, cudaStream_t st) {
  using C2 = typename sq::Vec2<Real>::T;
  // Tile bits of the gradient kernel: the batch's SQ_BOPT_TILE_BITS when a
  // gradient kernel of that size exists, else the precision's default.
  const uint32_t M = batch_adj_fn<Real>(b->tile_bits) ? b->tile_bits : batch_default_bits<Real>();
  const size_t nc = b->circs.size();
  if (nc == 0) return SQ_OK;
  // This run restages the shared buffers: the energy run's plan cache and
  // graph are no longer valid.
  b->planned_version = ~uint64_t(0);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  std::vector<std::vector<unsigned char>> packed(nc);
  std::vector<uint32_t> nfwd(nc, 0), nrev(nc, 0);
  std::vector<std::vector<std::pair<int32_t, double>>> occs(nc);
  std::vector<std::string> errs(nc);
  std::vector<char> ok(nc, 0);
  std::atomic<size_t> next{0};
  const unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  PlanShare share;
  std::vector<std::thread> workers;
  for (unsigned t = 0; t < nth; ++t)
    workers.emplace_back([&]() {
      for (size_t i = next++; i < nc; i = next++)
        ok[i] = plan_gradient_circuit<Real>(b->circs[i], M, packed[i], nfwd[i], nrev[i], occs[i], errs[i], &share);
    });
  for (auto &th : workers) th.join();
  for (size_t i = 0; i < nc; ++i) {
    if (!ok[i]) return fail(SQ_ERR_UNSUPPORTED, errs[i]);
    for (const auto &o : occs[i])
      if (o.first >= int32_t(n_params))
        return fail(SQ_ERR_INVALID, "batch gradient: parameter index " + std::to_string(o.first) +
                                        " >= n_params " + std::to_string(n_params));
  }
  // Circuits that all share one plan structure (many parameter sets of one
  // circuit) and stream their states get a JIT-specialised kernel.
  const void *jit_fn = nullptr;
  if (uniform_plans<Real>(b, packed, nfwd, nrev, occs, M)) {
    // Looked up by plan structure: a repeated gradient run of the same
    // circuit skips generating (and hashing) the kernel's source.
    static std::mutex memo_mu;
    static std::map<std::tuple<uint64_t, uint64_t, uint64_t>, const void *> memo;
    const auto sk = structure_key(packed[0], coef_ranges<Real>(packed[0]), b->circs[0].n);
    const std::tuple<uint64_t, uint64_t, uint64_t> key{
        sk.first, sk.second, (uint64_t(nfwd[0]) << 32) | (uint64_t(nrev[0]) << 8) | (M << 1) | (sizeof(Real) == 4)};
    {
      std::lock_guard<std::mutex> lk(memo_mu);
      auto it = memo.find(key);
      if (it != memo.end()) jit_fn = it->second;
    }
    if (!jit_fn) {
      std::string err;
      jit_fn = sq::jit_batch_adjoint_kernel(packed[0].data(), nfwd[0], nrev[0], b->circs[0].n, M,
                                            sizeof(Real) == 4, err);
      if (jit_fn) {
        std::lock_guard<std::mutex> lk(memo_mu);
        memo[key] = jit_fn;
      }
    }
  }
  // Largest work first.
  b->order.resize(nc);
  for (size_t i = 0; i < nc; ++i) b->order[i] = uint32_t(i);
  std::stable_sort(b->order.begin(), b->order.end(), [&](uint32_t x, uint32_t y) {
    const uint64_t cx = (uint64_t(1) << b->circs[x].n) * (uint64_t(nfwd[x]) + 2 * nrev[x] + 2);
    const uint64_t cy = (uint64_t(1) << b->circs[y].n) * (uint64_t(nfwd[y]) + 2 * nrev[y] + 2);
    return cx > cy;
  });
  // psi and lambda of every circuit larger than a tile live in the pool.
  uint64_t pool_amps = 0, nocc = 0;
  std::vector<uint64_t> psi_off(nc, 0), lam_off(nc, 0), occ_off(nc, 0);
  for (uint32_t id : b->order) {
    const Circ &c = b->circs[id];
    if (c.n > M) {
      psi_off[id] = pool_amps;
      lam_off[id] = pool_amps + (uint64_t(1) << c.n);
      pool_amps += uint64_t(2) << c.n;
    }
    occ_off[id] = nocc;
    nocc += occs[id].size();
  }
  size_t plan_bytes = 0;
  for (size_t i = 0; i < nc; ++i) plan_bytes += packed[i].size();
  SQB_CUDA(cudaSetDevice(b->device));
  if (int s = b->d_pool.ensure(std::max<uint64_t>(pool_amps, 1) * sizeof(C2))) return s;
  if (int s = b->d_plans.ensure(plan_bytes + 16)) return s;
  if (int s = b->h_plans.ensure(plan_bytes + 16)) return s;
  if (int s = b->d_table.ensure(nc * sizeof(sq::BatchCircuit))) return s;
  if (int s = b->h_table.ensure(nc * sizeof(sq::BatchCircuit))) return s;
  if (int s = b->d_energy.ensure(nc * sizeof(double))) return s;
  if (int s = b->h_energy.ensure(nc * sizeof(double))) return s;
  if (int s = b->d_counter.ensure(sizeof(unsigned))) return s;
  if (int s = b->d_occ.ensure(std::max<uint64_t>(nocc, 1) * sizeof(double2))) return s;
  if (int s = b->h_occ.ensure(std::max<uint64_t>(nocc, 1) * sizeof(double2))) return s;
  if (b->hams_uploaded != b->hams.size()) {
    if (int s = b->d_hams.ensure(b->hams.size() * sizeof(sq::PauliParams))) return s;
    SQB_CUDA(cudaMemcpy(b->d_hams.p, b->hams.data(), b->hams.size() * sizeof(sq::PauliParams),
                        cudaMemcpyHostToDevice));
    b->hams_uploaded = b->hams.size();
  }
  auto *tab = static_cast<sq::BatchCircuit *>(b->h_table.p);
  unsigned char *hp = static_cast<unsigned char *>(b->h_plans.p);
  size_t off = 0;
  for (size_t pos = 0; pos < nc; ++pos) {
    const uint32_t id = b->order[pos];
    const Circ &c = b->circs[id];
    std::memcpy(hp + off, packed[id].data(), packed[id].size());
    sq::BatchCircuit &t = tab[pos];
    std::memset(&t, 0, sizeof(t));
    t.n = c.n;
    t.nsweeps = nfwd[id];
    t.nrev = nrev[id];
    t.ham = c.ham;
    t.state_off = psi_off[id];
    t.lam_off = lam_off[id];
    t.occ_off = occ_off[id];
    t.plan_off = off;
    off += packed[id].size();
  }
  const void *fn = jit_fn ? jit_fn : batch_adj_fn<Real>(M);
  const uint32_t L = uint32_t(sq::sweep_low_bits(int(M)));
  const int threads = 1 << (M - sq::kAdjRegBits);
  const size_t nw = size_t(threads + 31) / 32;
  const size_t smem = 4 * (size_t(1) << M) * sizeof(C2) + size_t(sq::kMaxCoef) * sizeof(C2) +
                      (jit_fn ? 0 : (size_t(1) << (M - L)) * sizeof(uint64_t)) +
                      nw * sq::kMaxInner * sizeof(double2);
  b->last_jit = jit_fn != nullptr;
  if (jit_fn) sq::jit_note_launch(true);
  SQB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  int per_sm = 0, sms = 0;
  SQB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
  SQB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  const uint32_t grid = uint32_t(std::max<uint64_t>(
      1, std::min<uint64_t>(nc, uint64_t(std::max(per_sm, 1)) * uint64_t(sms))));
  if (!b->ev0) {
    SQB_CUDA(cudaEventCreate(&b->ev0));
    SQB_CUDA(cudaEventCreate(&b->ev1));
  }
  sq::BatchParams P;
  std::memset(&P, 0, sizeof(P));
  P.circuits = static_cast<const sq::BatchCircuit *>(b->d_table.p);
  P.plans = static_cast<const unsigned char *>(b->d_plans.p);
  P.hams = static_cast<const sq::PauliParams *>(b->d_hams.p);
  P.ncircuits = uint32_t(nc);
  P.counter = static_cast<unsigned *>(b->d_counter.p);
  P.energies = static_cast<double *>(b->d_energy.p);
  C2 *poolp = static_cast<C2 *>(b->d_pool.p);
  double2 *occp = static_cast<double2 *>(b->d_occ.p);
  void *args[] = {&poolp, &P, &occp};
  SQB_CUDA(cudaMemcpyAsync(b->d_plans.p, b->h_plans.p, plan_bytes, cudaMemcpyHostToDevice, st));
  SQB_CUDA(cudaMemcpyAsync(b->d_table.p, b->h_table.p, nc * sizeof(sq::BatchCircuit),
                           cudaMemcpyHostToDevice, st));
  SQB_CUDA(cudaMemsetAsync(b->d_counter.p, 0, sizeof(unsigned), st));
  SQB_CUDA(cudaMemsetAsync(b->d_occ.p, 0, std::max<uint64_t>(nocc, 1) * sizeof(double2), st));
  SQB_CUDA(cudaEventRecord(b->ev0, st));
  SQB_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(threads), args, smem, st));
  SQB_CUDA(cudaGetLastError());
  SQB_CUDA(cudaEventRecord(b->ev1, st));
  SQB_CUDA(cudaMemcpyAsync(b->h_energy.p, b->d_energy.p, nc * sizeof(double), cudaMemcpyDeviceToHost, st));
  SQB_CUDA(cudaMemcpyAsync(b->h_occ.p, b->d_occ.p, std::max<uint64_t>(nocc, 1) * sizeof(double2),
                           cudaMemcpyDeviceToHost, st));
  SQB_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f;
  SQB_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  b->last_ms = ms;
  b->last_ctas = grid;
  const double *he = static_cast<const double *>(b->h_energy.p);
  const double2 *ho = static_cast<const double2 *>(b->h_occ.p);
  for (size_t pos = 0; pos < nc; ++pos) energies[b->order[pos]] = he[pos];
  for (size_t id = 0; id < nc; ++id) {
    double *g = grads + id * n_params;
    for (uint32_t p = 0; p < n_params; ++p) g[p] = 0.0;
    for (size_t s = 0; s < occs[id].size(); ++s) {
      const auto &o = occs[id][s];
      if (o.first >= 0) g[o.first] += 2.0 * ho[occ_off[id] + s].x * o.second;
    }
  }
  return SQ_OK;
}

}  // namespace

extern "C" {

int sq_batch_create(int dtype, sq_batch **out) {
  if (!out) return fail(SQ_ERR_INVALID, "null pointer");
  if (dtype != SQ_C128 && dtype != SQ_C64) return fail(SQ_ERR_INVALID, "bad dtype");
  auto b = std::make_unique<sq_batch>();
  b->dtype = dtype;
  SQB_CUDA(cudaGetDevice(&b->device));
  *out = b.release();
  return SQ_OK;
}

int sq_batch_destroy(sq_batch *b) {
  if (!b) return SQ_OK;
  std::unique_ptr<sq_batch> holder(b);
  cudaSetDevice(b->device);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  b->d_pool.release();
  b->d_plans.release();
  b->d_table.release();
  b->d_hams.release();
  b->d_energy.release();
  b->d_counter.release();
  b->d_occ.release();
  b->h_occ.release();
  b->d_def.release();
  b->d_part.release();
  b->h_def.release();
  b->h_plans.release();
  b->h_table.release();
  b->h_energy.release();
  return SQ_OK;
}

int sq_batch_set_option(sq_batch *b, int option, int64_t value) {
  if (!b) return fail(SQ_ERR_INVALID, "null batch");
  switch (option) {
    case SQ_BOPT_KEEP_STATES:
      b->keep = value != 0;
      b->version++;
      return SQ_OK;
    case SQ_BOPT_TILE_BITS:
      if (value != 0 && (value < 10 || value > 12))
        return fail(SQ_ERR_INVALID, "SQ_BOPT_TILE_BITS takes 0 or 10..12");
      b->tile_bits = uint32_t(value);
      return SQ_OK;
    case SQ_BOPT_LOW_BITS:
      if (value < 0 || value > 8) return fail(SQ_ERR_INVALID, "SQ_BOPT_LOW_BITS takes 0..8");
      b->low_bits = uint32_t(value);
      return SQ_OK;
    case SQ_BOPT_MAX_OPS:
      if (value < 0 || value > sq::kMaxOps)
        return fail(SQ_ERR_INVALID, "SQ_BOPT_MAX_OPS takes 0.." + std::to_string(sq::kMaxOps));
      b->max_ops = uint32_t(value);
      return SQ_OK;
    case SQ_BOPT_CTAS_PER_SM:
      if (value < 0 || value > 32) return fail(SQ_ERR_INVALID, "SQ_BOPT_CTAS_PER_SM takes 0..32");
      b->ctas_per_sm = uint32_t(value);
      return SQ_OK;
  }
  return fail(SQ_ERR_INVALID, "unknown batch option");
}

int sq_batch_add_hamiltonian(sq_batch *b, uint32_t num_qubits, const char *paulis,
                             const double *weights, uint32_t n_terms, uint32_t *ham_id) {
  if (!b || !ham_id || (n_terms && (!paulis || !weights))) return fail(SQ_ERR_INVALID, "null pointer");
  if (num_qubits < 4 || num_qubits > 30) return fail(SQ_ERR_UNSUPPORTED, "batch: 4..30 qubits");
  sq::PauliParams P;
  if (int s = build_pauli(num_qubits, paulis, weights, n_terms, P)) return s;
  b->hams.push_back(P);
  b->ham_n.push_back(num_qubits);
  *ham_id = uint32_t(b->hams.size() - 1);
  return SQ_OK;
}

int sq_batch_add_circuit(sq_batch *b, uint32_t num_qubits, const sq_circuit_op *ops, uint32_t nops,
                         uint32_t ham_id, uint32_t *circuit_id) {
  if (!b || !circuit_id || (nops && !ops)) return fail(SQ_ERR_INVALID, "null pointer");
  if (ham_id >= b->hams.size() || b->ham_n[ham_id] != num_qubits)
    return fail(SQ_ERR_INVALID, "batch: Hamiltonian id / qubit count mismatch");
  Circ c;
  c.n = num_qubits;
  c.ham = ham_id;
  c.ops.assign(ops, ops + nops);
  for (auto &op : c.ops) {
    if (op.k > 4) return fail(SQ_ERR_UNSUPPORTED, "batch: gates act on at most 4 qubits");
    uint64_t seen = 0;
    for (uint32_t j = 0; j < op.k; ++j) {
      if (op.qubits[j] >= num_qubits || ((seen >> op.qubits[j]) & 1))
        return fail(SQ_ERR_INVALID, "batch: bad or repeated qubit");
      seen |= uint64_t(1) << op.qubits[j];
    }
    if (op.gate < 0) {
      if (!op.matrix) return fail(SQ_ERR_INVALID, "batch: null matrix");
      const size_t d = size_t(1) << op.k;
      c.fixed.emplace_back(d * d);
      std::memcpy(c.fixed.back().data(), op.matrix, d * d * sizeof(cplx));
      op.matrix = reinterpret_cast<const double *>(c.fixed.back().data());
    } else if (sq::gate_qubits(op.gate) != int(op.k)) {
      return fail(SQ_ERR_INVALID, "batch: qubit count does not match the gate");
    }
  }
  b->circs.push_back(std::move(c));
  b->version++;
  *circuit_id = uint32_t(b->circs.size() - 1);
  return SQ_OK;
}

int sq_batch_set_angles(sq_batch *b, uint32_t circuit, const double *angles, uint32_t count) {
  if (!b || (count && !angles)) return fail(SQ_ERR_INVALID, "null pointer");
  if (circuit >= b->circs.size()) return fail(SQ_ERR_INVALID, "batch: bad circuit id");
  uint32_t k = 0;
  for (auto &op : b->circs[circuit].ops)
    for (uint32_t j = 0; j < op.nangles; ++j) {
      if (k >= count) return fail(SQ_ERR_INVALID, "batch: too few angles");
      op.angles[j] = angles[k++];
    }
  if (k != count) return fail(SQ_ERR_INVALID, "batch: angle count mismatch");
  b->values_version++;
  return SQ_OK;
}

int sq_batch_num_circuits(const sq_batch *b, uint32_t *count) {
  if (!b || !count) return fail(SQ_ERR_INVALID, "null pointer");
  *count = uint32_t(b->circs.size());
  return SQ_OK;
}

int sq_batch_run(sq_batch *b, double *energies, void *stream) {
  if (!b || (!energies && !b->circs.empty())) return fail(SQ_ERR_INVALID, "null pointer");
  auto st = static_cast<cudaStream_t>(stream);
  return b->dtype == SQ_C64 ? run_impl<float>(b, energies, st) : run_impl<double>(b, energies, st);
}

int sq_batch_autotune(sq_batch *b, uint32_t reps, sq_batch_config *best, void *stream) {
  if (!b) return fail(SQ_ERR_INVALID, "null batch");
  if (b->circs.empty()) return fail(SQ_ERR_INVALID, "batch autotune: no circuits");
  auto st = static_cast<cudaStream_t>(stream);
  reps = std::max<uint32_t>(1, std::min<uint32_t>(reps, 16));
  std::vector<double> e(b->circs.size());
  const uint32_t saved[4] = {b->tile_bits, b->low_bits, b->max_ops, b->ctas_per_sm};
  sq_batch_config bc{};
  bc.kernel_ms = -1.0;
  int status = SQ_OK;
  const bool c64 = b->dtype == SQ_C64;
  for (uint32_t m : {10u, 11u, 12u}) {
    const void *fn = nullptr;
    int threads = 0, per_sm = 0;
    size_t smem = 0;
    status = c64 ? batch_shape<float>(m, fn, threads, smem, per_sm)
                 : batch_shape<double>(m, fn, threads, smem, per_sm);
    if (status != SQ_OK) break;
    for (uint32_t l : {0u, 3u})
      for (uint32_t ops : {32u, 64u}) {
        // CTAs per SM from 1 up to the occupancy limit (at most 4 candidates).
        for (int cps = 1; cps <= std::min(per_sm, 4) && status == SQ_OK; ++cps) {
          b->tile_bits = m;
          b->low_bits = l;
          b->max_ops = ops;
          b->ctas_per_sm = uint32_t(cps);
          double t = 1e30;
          for (uint32_t r = 0; r < reps && status == SQ_OK; ++r) {
            status = c64 ? run_impl<float>(b, e.data(), st) : run_impl<double>(b, e.data(), st);
            t = std::min(t, double(b->last_ms));
          }
          if (status == SQ_OK && (bc.kernel_ms < 0 || t < bc.kernel_ms)) {
            bc.tile_bits = m;
            bc.low_bits = l;
            bc.max_ops = ops;
            bc.ctas_per_sm = uint32_t(cps);
            bc.kernel_ms = t;
          }
        }
      }
    if (status != SQ_OK) break;
  }
  if (status != SQ_OK) {
    b->tile_bits = saved[0];
    b->low_bits = saved[1];
    b->max_ops = saved[2];
    b->ctas_per_sm = saved[3];
    return status;
  }
  b->tile_bits = bc.tile_bits;
  b->low_bits = bc.low_bits;
  b->max_ops = bc.max_ops;
  b->ctas_per_sm = bc.ctas_per_sm;
  if (best) *best = bc;
  return SQ_OK;
}

int sq_batch_run_gradients(sq_batch *b, uint32_t n_params, double *energies, double *grads,
                           void *stream) {
  if (!b || !energies || (n_params && !grads)) return fail(SQ_ERR_INVALID, "null pointer");
  auto st = static_cast<cudaStream_t>(stream);
  return b->dtype == SQ_C64 ? run_gradient_impl<float>(b, n_params, energies, grads, st)
                            : run_gradient_impl<double>(b, n_params, energies, grads, st);
}

int sq_jit_batch_adjoint_source(uint32_t num_qubits, int dtype, const sq_circuit_op *ops, uint32_t nops,
                                char *buf, uint64_t cap, uint64_t *len) {
  if ((nops && !ops) || !len) return fail(SQ_ERR_INVALID, "null pointer");
  if (dtype != SQ_C128 && dtype != SQ_C64) return fail(SQ_ERR_INVALID, "bad dtype");
  const bool c64 = dtype == SQ_C64;
  const uint32_t M = c64 ? sq::kBatchTileBitsC64 : sq::kBatchTileBitsC128;
  if (num_qubits <= M || num_qubits > 30) return fail(SQ_ERR_INVALID, "num_qubits must exceed the tile bits");
  Circ c;
  c.n = num_qubits;
  c.ops.assign(ops, ops + nops);
  std::vector<unsigned char> packed;
  uint32_t nf = 0, nr = 0;
  std::vector<std::pair<int32_t, double>> occ;
  std::string err;
  const bool ok = c64 ? plan_gradient_circuit<float>(c, M, packed, nf, nr, occ, err)
                      : plan_gradient_circuit<double>(c, M, packed, nf, nr, occ, err);
  if (!ok) return fail(SQ_ERR_UNSUPPORTED, err);
  const std::string body = sq::jit_batch_adjoint_body(packed.data(), nf, nr, num_qubits, M, c64);
  const std::string src = body.empty() ? std::string() : sq::jit_batch_source(body);
  *len = src.size();
  if (buf && cap) {
    const size_t n = std::min<size_t>(cap - 1, src.size());
    std::memcpy(buf, src.data(), n);
    buf[n] = '\0';
  }
  return SQ_OK;
}

int sq_jit_multi_source(uint32_t num_qubits, int dtype, const sq_circuit_op *ops, uint32_t nops,
                        uint32_t sweep_index, int from_zero, char *buf, uint64_t cap, uint64_t *len,
                        uint32_t *nsweeps) {
  if ((nops && !ops) || !len) return fail(SQ_ERR_INVALID, "null pointer");
  if (dtype != SQ_C128 && dtype != SQ_C64) return fail(SQ_ERR_INVALID, "bad dtype");
  const bool c64 = dtype == SQ_C64;
  const uint32_t M = c64 ? sq::kBatchTileBitsC64 : sq::kBatchTileBitsC128;
  if (num_qubits <= M || num_qubits > 30) return fail(SQ_ERR_INVALID, "num_qubits must exceed the tile bits");
  Circ c;
  c.n = num_qubits;
  c.ops.assign(ops, ops + nops);
  std::vector<unsigned char> packed;
  std::string err;
  const int sel = multi_select();
  const int ns = c64 ? plan_circuit<float>(c, M, 0, 0, packed, err, sel)
                     : plan_circuit<double>(c, M, 0, 0, packed, err, sel);
  if (ns < 0) return fail(SQ_ERR_UNSUPPORTED, err);
  if (nsweeps) *nsweeps = uint32_t(ns);
  if (sweep_index >= uint32_t(ns)) return fail(SQ_ERR_INVALID, "no such sweep");
  std::vector<uint64_t> coef_at;
  const auto sweeps = unpack_sweeps(packed, coef_at);
  const sq::PlannedSweep &ps = sweeps[sweep_index];
  const std::string body = sq::jit_body(ps, c64, sq::jit_minb(c64, ps.h.m), true, from_zero != 0);
  const std::string src =
      body.empty() ? std::string() : sq::jit_source(ps, c64, sq::jit_minb(c64, ps.h.m), true, from_zero != 0);
  *len = src.size();
  if (buf && cap) {
    const size_t n = std::min<size_t>(cap - 1, src.size());
    std::memcpy(buf, src.data(), n);
    buf[n] = '\0';
  }
  return SQ_OK;
}

int sq_batch_groups(const sq_batch *b, uint32_t *groups, uint32_t *circuits) {
  if (!b) return fail(SQ_ERR_INVALID, "null batch");
  uint32_t c = 0;
  for (const auto &g : b->groups) c += g.count;
  if (groups) *groups = uint32_t(b->groups.size());
  if (circuits) *circuits = c;
  return SQ_OK;
}

int sq_batch_state(sq_batch *b, uint32_t circuit, void *host_dst, void *stream) {
  if (!b || !host_dst) return fail(SQ_ERR_INVALID, "null pointer");
  if (circuit >= b->state_off.size() || b->state_off[circuit] == ~uint64_t(0))
    return fail(SQ_ERR_INVALID, "batch: state not kept (set SQ_BOPT_KEEP_STATES before run)");
  const size_t amp = b->dtype == SQ_C64 ? 8 : 16;
  const size_t n = size_t(1) << b->circs[circuit].n;
  auto st = static_cast<cudaStream_t>(stream);
  SQB_CUDA(cudaMemcpyAsync(host_dst, static_cast<char *>(b->d_pool.p) + b->state_off[circuit] * amp,
                           n * amp, cudaMemcpyDeviceToHost, st));
  SQB_CUDA(cudaStreamSynchronize(st));
  return SQ_OK;
}

int sq_batch_stats(const sq_batch *b, uint64_t *streamed, uint64_t *sweeps, uint64_t *hbm_bytes) {
  if (!b) return fail(SQ_ERR_INVALID, "null batch");
  if (streamed) *streamed = b->stat_streamed;
  if (sweeps) *sweeps = b->stat_sweeps;
  if (hbm_bytes) *hbm_bytes = b->stat_bytes;
  return SQ_OK;
}

int sq_batch_last_timing(const sq_batch *b, double *kernel_ms, uint32_t *ctas) {
  if (!b || !kernel_ms || !ctas) return fail(SQ_ERR_INVALID, "null pointer");
  *kernel_ms = b->last_ms;
  *ctas = b->last_ctas;
  return SQ_OK;
}

}  // extern "C"

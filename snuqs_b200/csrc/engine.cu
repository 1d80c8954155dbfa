// snuqs_b200 engine: state handles, the gate queue, launches, and the C ABI
// declared in include/snuqs_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdlib>
#include <cstdio>
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/snuqs_b200.h"
#include "adjoint_kernels.cuh"
#include "adjoint_plan.h"
#include "engine_internal.h"
#include "host_ops.h"
#include "jit.h"
#include "reduce_kernels.cuh"
#include "sweep_kernels.cuh"
#include "sweep_registry.h"

using sq::cplx;

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

// For the library's other translation units: record an error, return `code`.
int sq_detail_fail(int code, const char *msg) { return fail(code, "%s", msg); }

#define SQ_CUDA(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(e_ == cudaErrorMemoryAllocation ? SQ_ERR_OOM : SQ_ERR_CUDA,          \
                  "%s: %s (%s)", #call, cudaGetErrorString(e_), cudaGetErrorName(e_)); \
  } while (0)

#define SQ_TRY(expr)            \
  do {                          \
    int s_ = (expr);            \
    if (s_ != SQ_OK) return s_; \
  } while (0)

// ---------------------------------------------------------------------------
// State
// ---------------------------------------------------------------------------
struct PendingOp {
  std::vector<cplx> m;
  std::vector<uint32_t> qubits;
  std::vector<uint32_t> controls;
  std::vector<uint8_t> cvals;
};

// Qubit remapping in fused sweeps (SQ_OPT_REMAP), off by default: measured on
// B200 it saves sweeps (30-qubit mix: 26 instead of 27; QV-28: 37 instead of
// 41) but costs more per sweep (fewer sweeps can load and store straight
// between HBM and registers, and the permuted copy-out meets bank
// conflicts): 197 vs 188 ms per 30-qubit step, 167 vs 157 ms for QV-28.
// SQ_REMAP=1 turns the default on.
static int default_remap() {
  static const int v = [] {
    const char *e = std::getenv("SQ_REMAP");
    return e && *e ? (e[0] == '0' ? 0 : 1) : 0;
  }();
  return v;
}

struct sq_state {
  uint32_t n = 0;
  int dtype = SQ_C128;
  void *data = nullptr;
  bool owns = true;
  int device = 0;
  int fusion = 1;
  uint32_t tile_bits = 0;  // 0: the precision's default
  int reorder = 1;
  std::vector<PendingOp> pending;
  double *scratch = nullptr;  // reduction partials + result
  uint32_t scratch_len = 0;
  uint64_t launches = 0;
  int timing = 0;
  uint32_t low_bits = 0;  // 0: automatic
  int jit = -1;  // -1: automatic (states of >= kJitMinQubits qubits), 0: off, 1: on
  int remap = default_remap();  // SQ_OPT_REMAP
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> sweep_events;
  // Device word a sweep kernel sets when one of its bounded waits gives up
  // (sq::kKernelErrTimeout); read and cleared by sq_state_check.
  uint32_t *errword = nullptr;
  void *rscratch = nullptr;  // result kernels' scratch (results.cu)
  size_t rscratch_bytes = 0;
  void *hscratch = nullptr;  // pinned host staging of results with host buffers
  size_t hscratch_bytes = 0;
  // The last plans, reused for the same gate sequence with other values (a
  // circuit run again with other angles): sq::rebuild_plan re-emits them
  // from their recipes without planning.  Keyed by the ops' signature hash
  // and the plan options.
  struct PlanMemo {
    std::pair<uint64_t, uint64_t> sig{0, 0};
    uint64_t opts = ~uint64_t(0);
    std::vector<sq::PlannedLaunch> plan;
  };
  PlanMemo flush_memo, fwd_memo, rev_memo;
};

// Plans `ops`, or re-emits the memo's plan when the ops have its signature
// and options (and every sweep of it has a recipe); the memo then holds the
// new plan.  Throws what plan_sweeps throws.
static std::vector<sq::PlannedLaunch> plan_memo(sq_state::PlanMemo &memo, const std::vector<sq::HostOp> &ops,
                                                uint32_t n, const sq::PlanOptions &opt) {
  const auto sig = sq::op_signature_hash(ops);
  const uint64_t key = sq::plan_options_key(opt);
  if (memo.opts == key && memo.sig == sig) {
    std::vector<sq::PlannedLaunch> plan = memo.plan;
    if (sq::rebuild_plan(plan, ops, n)) {
      memo.plan = plan;
      return plan;
    }
  }
  std::vector<sq::PlannedLaunch> plan = sq::plan_sweeps(ops, n, opt);
  memo.sig = sig;
  memo.opts = key;
  memo.plan = plan;
  return plan;
}

// JIT-specialised sweeps pay a one-off NVRTC compile per distinct sweep
// structure; below this size the generic kernel's sweeps are too short for
// the compile to pay back within a few circuit runs.
static constexpr uint32_t kJitMinQubits = 20;

static bool use_jit(const sq_state *s) {
  static const bool env_off = [] {
    const char *e = std::getenv("SQ_JIT");
    return e && e[0] == '0';
  }();
  if (s->jit == 0 || !sq::jit_available()) return false;
  if (s->jit == 1) return true;
  return !env_off && s->n >= kJitMinQubits;
}

static size_t amp_bytes(int dtype) { return dtype == SQ_C64 ? 8 : 16; }

static int use_device(int dev) {
  int cur = -1;
  SQ_CUDA(cudaGetDevice(&cur));
  if (cur != dev) SQ_CUDA(cudaSetDevice(dev));
  return SQ_OK;
}

struct DeviceInfo {
  int sms = 0;
};
static std::mutex g_dev_mu;
static std::map<int, DeviceInfo> g_devs;

// Compiled sweep kernel for (precision, tile bits m); nullptr if none.
template <typename Real>
static const void *sweep_fn(uint32_t m) {
  if constexpr (sizeof(Real) == 8) {
    switch (m) {
      case 4: return SQ_SWEEP_PTR_NAME(double, 4)();
      case 7: return SQ_SWEEP_PTR_NAME(double, 7)();
      case 10: return SQ_SWEEP_PTR_NAME(double, 10)();
      case 11: return SQ_SWEEP_PTR_NAME(double, 11)();
      case 12: return SQ_SWEEP_PTR_NAME(double, 12)();
    }
  } else {
    switch (m) {
      case 4: return SQ_SWEEP_PTR_NAME(float, 4)();
      case 7: return SQ_SWEEP_PTR_NAME(float, 7)();
      case 10: return SQ_SWEEP_PTR_NAME(float, 10)();
      case 12: return SQ_SWEEP_PTR_NAME(float, 12)();
    }
  }
  return nullptr;
}

// Largest compiled tile size <= min(n, requested).
static uint32_t pick_tile_bits(int dtype, uint32_t n, uint32_t requested) {
  const uint32_t cap = std::min(n, requested);
  uint32_t best = 0;
  if (dtype == SQ_C64) {
    for (int m : sq::kTileBitsC64)
      if (uint32_t(m) <= cap) best = uint32_t(m);
  } else {
    for (int m : sq::kTileBitsC128)
      if (uint32_t(m) <= cap) best = uint32_t(m);
  }
  return best;
}

template <typename Real>
static const void *adjoint_fn(uint32_t m) {
  if constexpr (sizeof(Real) == 8) {
    switch (m) {
      case 4: return SQ_ADJOINT_PTR_NAME(double, 4)();
      case 7: return SQ_ADJOINT_PTR_NAME(double, 7)();
      case 10: return SQ_ADJOINT_PTR_NAME(double, 10)();
    }
  } else {
    switch (m) {
      case 4: return SQ_ADJOINT_PTR_NAME(float, 4)();
      case 7: return SQ_ADJOINT_PTR_NAME(float, 7)();
      case 11: return SQ_ADJOINT_PTR_NAME(float, 11)();
    }
  }
  return nullptr;
}

static uint32_t pick_adjoint_tile_bits(int dtype, uint32_t n) {
  uint32_t best = 0;
  if (dtype == SQ_C64) {
    for (int m : sq::kAdjTileBitsC64)
      if (uint32_t(m) <= n) best = uint32_t(m);
  } else {
    for (int m : sq::kAdjTileBitsC128)
      if (uint32_t(m) <= n) best = uint32_t(m);
  }
  return best;
}

template <typename Real>
static size_t adjoint_smem(uint32_t m, uint32_t ncoef) {
  const uint32_t l = uint32_t(sq::sweep_low_bits(int(m)));
  const uint32_t nt = 1u << (m - sq::kAdjRegBits);
  const uint32_t nw = (nt + 31) / 32;
  return 4 * (size_t(1) << m) * 2 * sizeof(Real) + size_t((ncoef + 1) & ~1u) * 2 * sizeof(Real) +
         (size_t(1) << (m - l)) * 8 + size_t(nw) * sq::kMaxInner * sizeof(double2);
}

template <typename Real>
static int set_sweep_attributes() {
  for (uint32_t m = 4; m <= uint32_t(sq::kMaxTileBits); ++m) {
    const void *fn = adjoint_fn<Real>(m);
    if (!fn) continue;
    SQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(adjoint_smem<Real>(m, sq::kMaxCoef))));
  }
  for (uint32_t m = 4; m <= uint32_t(sq::kMaxTileBits); ++m) {
    const void *fn = sweep_fn<Real>(m);
    if (!fn) continue;
    const int max_smem = 2 * (1 << m) * int(2 * sizeof(Real)) + sq::kMaxCoef * int(2 * sizeof(Real)) +
                         (1 << m) * 8;
    SQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
  }
  return SQ_OK;
}

static int device_info(int dev, DeviceInfo &out) {
  std::lock_guard<std::mutex> lk(g_dev_mu);
  auto it = g_devs.find(dev);
  if (it != g_devs.end()) {
    out = it->second;
    return SQ_OK;
  }
  DeviceInfo di;
  SQ_CUDA(cudaDeviceGetAttribute(&di.sms, cudaDevAttrMultiProcessorCount, dev));
  // Kernel attributes are per device; set them while we hold the lock.
  SQ_TRY(set_sweep_attributes<double>());
  SQ_TRY(set_sweep_attributes<float>());
  SQ_CUDA(cudaFuncSetAttribute(sq::gate_kernel_large<double>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, 1024 * 16));
  SQ_CUDA(cudaFuncSetAttribute(sq::gate_kernel_large<float>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, 1024 * 16));
  g_devs[dev] = di;
  out = di;
  return SQ_OK;
}

// ---------------------------------------------------------------------------
// Launch helpers
// ---------------------------------------------------------------------------
template <typename Real>
static int launch_sweep(sq_state *s, const sq::PlannedSweep &ps, cudaStream_t st) {
  using C2 = typename sq::Vec2<Real>::T;
  DeviceInfo di;
  SQ_TRY(device_info(s->device, di));
  auto P = std::make_unique<sq::SweepParams<Real>>();
  std::memset(P.get(), 0, sizeof(*P));
  P->h = ps.h;
  if (ps.ph.size() > size_t(sq::kMaxPhases) || ps.op.size() > size_t(sq::kMaxOps) ||
      ps.coef.size() > size_t(sq::kMaxCoef))
    return fail(SQ_ERR_INVALID, "internal: sweep plan exceeds its budget");
  std::copy(ps.ph.begin(), ps.ph.end(), P->ph);
  std::copy(ps.op.begin(), ps.op.end(), P->op);
  for (size_t i = 0; i < ps.coef.size(); ++i) {
    P->coef[2 * i] = Real(ps.coef[i].real());
    P->coef[2 * i + 1] = Real(ps.coef[i].imag());
  }
  const uint32_t m = ps.h.m, l = ps.h.l;
  const int threads = 1 << (m - sq::kRegBits);
  const size_t smem = 2 * (size_t(1) << m) * sizeof(C2) +
                      size_t((ps.h.ncoef + 1) & ~1u) * sizeof(C2) +
                      (size_t(1) << (m - l)) * sizeof(uint64_t);
  int per_sm = 0;
  const void *fn = nullptr;
  size_t launch_smem = smem;
  if (use_jit(s)) {
    std::string err;
    const size_t jsmem = sq::jit_smem(ps, sizeof(Real) == 4);
    fn = sq::jit_sweep_kernel(ps, sizeof(Real) == 4, err);
    if (fn && cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(jsmem)) != cudaSuccess) {
      cudaGetLastError();
      fn = nullptr;
    }
    if (fn && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, jsmem) != cudaSuccess) {
      cudaGetLastError();
      per_sm = sq::jit_minb(sizeof(Real) == 4, m);
    }
    if (fn) launch_smem = jsmem;
    sq::jit_note_launch(fn != nullptr);
  }
  if (!fn) {
    if (ps.h.flags & sq::kRemap) return fail(SQ_ERR_INVALID, "internal: remapping sweep without its JIT kernel");
    fn = sweep_fn<Real>(m);
    if (!fn) return fail(SQ_ERR_INVALID, "internal: no sweep kernel for %u tile bits", m);
    SQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
  }
  if (per_sm < 1) per_sm = 1;
  const uint64_t grid = std::min<uint64_t>(ps.h.num_tiles, uint64_t(per_sm) * di.sms);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (s->timing) {
    SQ_CUDA(cudaEventCreate(&e0));
    SQ_CUDA(cudaEventCreate(&e1));
    SQ_CUDA(cudaEventRecord(e0, st));
  }
  C2 *psi = reinterpret_cast<C2 *>(s->data);
  uint32_t *errp = s->errword;
  void *args[] = {&psi, P.get(), &errp};  // the generic kernel takes the first two
  SQ_CUDA(cudaLaunchKernel(fn, dim3(unsigned(grid)), dim3(threads), args, launch_smem, st));
  SQ_CUDA(cudaGetLastError());
  if (s->timing) {
    SQ_CUDA(cudaEventRecord(e1, st));
    s->sweep_events.emplace_back(e0, e1);
  }
  s->launches++;
  return SQ_OK;
}

template <typename Real, int K>
static int launch_gate_small(void *data, uint32_t n, const sq::HostOp &op, const void *dmat,
                             cudaStream_t st, int sms) {
  using C2 = typename sq::Vec2<Real>::T;
  auto P = std::make_unique<sq::GateParams<Real>>();
  std::memset(P.get(), 0, sizeof(*P));
  P->n = n;
  P->k = K;
  P->cmask = op.cmask;
  P->cval = op.cval;
  std::vector<int> sorted(op.tbits.begin(), op.tbits.end());
  std::sort(sorted.begin(), sorted.end());
  for (int j = 0; j < K; ++j) {
    P->tbit[j] = uint8_t(op.tbits[j]);
    P->tsorted[j] = uint8_t(sorted[j]);
  }
  if (!dmat)
    for (size_t i = 0; i < op.m.size(); ++i) {
      P->coef[2 * i] = Real(op.m[i].real());
      P->coef[2 * i + 1] = Real(op.m[i].imag());
    }
  const uint64_t groups = (uint64_t(1) << n) >> K;
  const uint64_t blocks = std::max<uint64_t>(
      1, std::min<uint64_t>((groups + 255) / 256, uint64_t(sms) * 8));
  sq::gate_kernel<Real, K><<<unsigned(blocks), 256, 0, st>>>(
      reinterpret_cast<C2 *>(data), *P, reinterpret_cast<const C2 *>(dmat));
  SQ_CUDA(cudaGetLastError());
  return SQ_OK;
}

template <typename Real>
static int launch_gate_large(void *data, uint32_t n, const sq::HostOp &op, cudaStream_t st,
                             int sms) {
  using C2 = typename sq::Vec2<Real>::T;
  const uint32_t k = uint32_t(op.tbits.size());
  const uint32_t D = 1u << k;
  sq::LargeGateParams P;
  std::memset(&P, 0, sizeof(P));
  P.n = n;
  P.k = k;
  P.cmask = op.cmask;
  P.cval = op.cval;
  std::vector<int> sorted(op.tbits.begin(), op.tbits.end());
  std::sort(sorted.begin(), sorted.end());
  for (uint32_t j = 0; j < k; ++j) {
    P.tbit[j] = uint8_t(op.tbits[j]);
    P.tsorted[j] = uint8_t(sorted[j]);
  }
  std::vector<C2> mt(size_t(D) * D);
  for (uint32_t r = 0; r < D; ++r)
    for (uint32_t c = 0; c < D; ++c) {
      C2 v;
      v.x = Real(op.m[size_t(r) * D + c].real());
      v.y = Real(op.m[size_t(r) * D + c].imag());
      mt[size_t(c) * D + r] = v;
    }
  void *dm = nullptr;
  SQ_CUDA(cudaMallocAsync(&dm, mt.size() * sizeof(C2), st));
  // Pageable source: the copy is staged before cudaMemcpyAsync returns, so
  // `mt` may go out of scope afterwards.
  SQ_CUDA(cudaMemcpyAsync(dm, mt.data(), mt.size() * sizeof(C2), cudaMemcpyHostToDevice, st));
  const uint64_t groups = (uint64_t(1) << n) >> k;
  const uint64_t blocks = std::max<uint64_t>(1, std::min<uint64_t>(groups, uint64_t(sms) * 4));
  sq::gate_kernel_large<Real><<<unsigned(blocks), D, D * sizeof(C2), st>>>(
      reinterpret_cast<C2 *>(data), P, reinterpret_cast<const C2 *>(dm));
  SQ_CUDA(cudaGetLastError());
  SQ_CUDA(cudaFreeAsync(dm, st));
  return SQ_OK;
}

template <typename Real>
static int launch_gate(void *data, uint32_t n, const sq::HostOp &op, const void *dmat,
                       cudaStream_t st, int sms) {
  switch (op.tbits.size()) {
    case 0: return launch_gate_small<Real, 0>(data, n, op, dmat, st, sms);
    case 1: return launch_gate_small<Real, 1>(data, n, op, dmat, st, sms);
    case 2: return launch_gate_small<Real, 2>(data, n, op, dmat, st, sms);
    case 3: return launch_gate_small<Real, 3>(data, n, op, dmat, st, sms);
    case 4: return launch_gate_small<Real, 4>(data, n, op, dmat, st, sms);
    default:
      if (dmat) return fail(SQ_ERR_UNSUPPORTED, "device-matrix gates support k <= 4");
      return launch_gate_large<Real>(data, n, op, st, sms);
  }
}

// Expand a diagonal HostOp (which may fold controls) to the dense form the
// unfused kernels take.
static sq::HostOp as_dense(const sq::HostOp &op) {
  if (op.kind == sq::kOpDense) return op;
  sq::HostOp d;
  d.kind = sq::kOpDense;
  d.tbits = op.tbits;
  const size_t D = op.m.size();
  d.m.assign(D * D, cplx(0, 0));
  for (size_t i = 0; i < D; ++i) d.m[i * D + i] = op.m[i];
  return d;
}

static int flush_impl(sq_state *s, cudaStream_t st) {
  if (s->pending.empty()) return SQ_OK;
  SQ_TRY(use_device(s->device));
  DeviceInfo di;
  SQ_TRY(device_info(s->device, di));
  const uint32_t n = s->n;
  const bool fused = s->fusion && n >= uint32_t(sq::kRegBits);
  const bool c64 = s->dtype == SQ_C64;
  std::vector<sq::HostOp> ops;
  ops.reserve(s->pending.size());
  for (const PendingOp &p : s->pending) {
    std::vector<int> tb;
    for (uint32_t q : p.qubits) tb.push_back(int(n - 1 - q));
    uint64_t cmask = 0, cval = 0;
    for (size_t i = 0; i < p.controls.size(); ++i) {
      const uint64_t bit = uint64_t(1) << (n - 1 - p.controls[i]);
      cmask |= bit;
      if (p.cvals[i]) cval |= bit;
    }
    if (fused) {
      sq::HostOp h;
      if (sq::analyse_op(p.m, tb, cmask, cval, h)) ops.push_back(std::move(h));
    } else {
      sq::HostOp h;
      h.kind = sq::kOpDense;
      h.tbits = tb;
      h.cmask = cmask;
      h.cval = cval;
      h.m = p.m;
      ops.push_back(std::move(h));
    }
  }
  s->pending.clear();
  if (!fused) {
    for (const auto &op : ops) {
      SQ_TRY(c64 ? launch_gate<float>(s->data, n, op, nullptr, st, di.sms)
                 : launch_gate<double>(s->data, n, op, nullptr, st, di.sms));
      s->launches++;
    }
    return SQ_OK;
  }
  std::vector<sq::PlannedLaunch> plan;
  sq::PlanOptions opt;
  try {
    opt.tile_bits = pick_tile_bits(s->dtype, n, s->tile_bits);
    if (opt.tile_bits < uint32_t(sq::kRegBits)) return fail(SQ_ERR_INVALID, "internal: no tile size");
    opt.reorder = s->reorder != 0;
    opt.max_dense_k = c64 ? 4 : 3;
    // Runs of 128 bytes leave the planner more free tile bits than 512-byte
    // runs and still read whole cache lines; measured faster on B200 for
    // multi-tile states.
    if (s->low_bits && s->low_bits + uint32_t(sq::kRegBits) <= opt.tile_bits)
      opt.low_bits = s->low_bits;
    else
      opt.low_bits = sq::auto_low_bits(c64, n, opt.tile_bits);
    // Remapping sweeps exist only as JIT-specialised kernels.
    opt.remap = s->remap && use_jit(s);
    plan = plan_memo(s->flush_memo, ops, n, opt);
  } catch (const std::exception &e) {
    return fail(SQ_ERR_INVALID, "planner: %s", e.what());
  }
  if (use_jit(s)) {
    std::vector<const sq::PlannedSweep *> sweeps;
    for (const auto &pl : plan)
      if (pl.is_sweep) sweeps.push_back(&pl.sweep);
    sq::jit_prepare(sweeps, c64);
    // A remapping sweep whose kernel did not compile cannot fall back to the
    // generic kernel: plan again without remapping.
    bool ready = true;
    for (const auto *ps : sweeps) {
      std::string err;
      if ((ps->h.flags & sq::kRemap) && !sq::jit_sweep_kernel(*ps, c64, err)) ready = false;
    }
    if (!ready) {
      try {
        opt.remap = false;
        plan = plan_memo(s->flush_memo, ops, n, opt);
      } catch (const std::exception &e) {
        return fail(SQ_ERR_INVALID, "planner: %s", e.what());
      }
      sweeps.clear();
      for (const auto &pl : plan)
        if (pl.is_sweep) sweeps.push_back(&pl.sweep);
      sq::jit_prepare(sweeps, c64);
    }
  }
  for (const auto &pl : plan) {
    if (pl.is_sweep) {
      SQ_TRY(c64 ? launch_sweep<float>(s, pl.sweep, st) : launch_sweep<double>(s, pl.sweep, st));
    } else {
      const sq::HostOp d = as_dense(pl.gate);
      SQ_TRY(c64 ? launch_gate<float>(s->data, n, d, nullptr, st, di.sms)
                 : launch_gate<double>(s->data, n, d, nullptr, st, di.sms));
      s->launches++;
    }
  }
  return SQ_OK;
}

static int alloc_errword(sq_state *s) {
  SQ_CUDA(cudaMalloc(&s->errword, sizeof(uint32_t)));
  SQ_CUDA(cudaMemset(s->errword, 0, sizeof(uint32_t)));
  return SQ_OK;
}

// Reads (and clears) the word a sweep kernel sets when a bounded wait gives
// up; the caller has synchronised the stream the kernels ran on.
static int take_kernel_error(sq_state *s) {
  if (!s->errword) return SQ_OK;
  uint32_t w = 0;
  SQ_CUDA(cudaMemcpy(&w, s->errword, sizeof(w), cudaMemcpyDeviceToHost));
  if (!w) return SQ_OK;
  SQ_CUDA(cudaMemset(s->errword, 0, sizeof(uint32_t)));
  return fail(SQ_ERR_TIMEOUT, "a sweep kernel gave up waiting for its tile copies (error word 0x%x); "
              "the state is invalid", w);
}

int sq_detail_state_scratch(sq_state *s, size_t bytes, void **out) {
  if (s->rscratch_bytes < bytes) {
    SQ_TRY(use_device(s->device));
    if (s->rscratch) SQ_CUDA(cudaFree(s->rscratch));
    s->rscratch = nullptr;
    s->rscratch_bytes = 0;
    SQ_CUDA(cudaMalloc(&s->rscratch, bytes));
    s->rscratch_bytes = bytes;
  }
  *out = s->rscratch;
  return SQ_OK;
}

int sq_detail_state_host_scratch(sq_state *s, size_t bytes, void **out) {
  if (s->hscratch_bytes < bytes) {
    if (s->hscratch) SQ_CUDA(cudaFreeHost(s->hscratch));
    s->hscratch = nullptr;
    s->hscratch_bytes = 0;
    SQ_CUDA(cudaHostAlloc(&s->hscratch, bytes, cudaHostAllocDefault));
    s->hscratch_bytes = bytes;
  }
  *out = s->hscratch;
  return SQ_OK;
}

static int ensure_scratch(sq_state *s, uint32_t len) {
  if (s->scratch_len >= len) return SQ_OK;
  if (s->scratch) SQ_CUDA(cudaFree(s->scratch));
  s->scratch = nullptr;
  s->scratch_len = 0;
  SQ_CUDA(cudaMalloc(&s->scratch, size_t(len) * sizeof(double)));
  s->scratch_len = len;
  return SQ_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char *sq_version(void) { return "snuqs_b200 0.1.0 (sm_100a)"; }
const char *sq_last_error(void) { return g_err.c_str(); }

int sq_device_count(int *count) {
  if (!count) return fail(SQ_ERR_INVALID, "null pointer");
  SQ_CUDA(cudaGetDeviceCount(count));
  return SQ_OK;
}
int sq_get_device(int *device) {
  if (!device) return fail(SQ_ERR_INVALID, "null pointer");
  SQ_CUDA(cudaGetDevice(device));
  return SQ_OK;
}
int sq_set_device(int device) {
  SQ_CUDA(cudaSetDevice(device));
  return SQ_OK;
}
int sq_device_synchronize(void) {
  SQ_CUDA(cudaDeviceSynchronize());
  return SQ_OK;
}
int sq_mem_info(size_t *free_bytes, size_t *total_bytes) {
  if (!free_bytes || !total_bytes) return fail(SQ_ERR_INVALID, "null pointer");
  SQ_CUDA(cudaMemGetInfo(free_bytes, total_bytes));
  return SQ_OK;
}

int sq_stream_create(void **stream, int nonblocking) {
  if (!stream) return fail(SQ_ERR_INVALID, "null pointer");
  cudaStream_t st = nullptr;
  SQ_CUDA(nonblocking ? cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) : cudaStreamCreate(&st));
  *stream = st;
  return SQ_OK;
}
int sq_stream_destroy(void *stream) {
  if (stream) SQ_CUDA(cudaStreamDestroy(static_cast<cudaStream_t>(stream)));
  return SQ_OK;
}
int sq_stream_synchronize(void *stream) {
  SQ_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  return SQ_OK;
}
int sq_stream_wait_event(void *stream, void *event) {
  if (!event) return fail(SQ_ERR_INVALID, "null event");
  SQ_CUDA(cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), static_cast<cudaEvent_t>(event), 0));
  return SQ_OK;
}
int sq_event_create(void **event) {
  if (!event) return fail(SQ_ERR_INVALID, "null pointer");
  cudaEvent_t e = nullptr;
  SQ_CUDA(cudaEventCreate(&e));
  *event = e;
  return SQ_OK;
}
int sq_event_destroy(void *event) {
  if (event) SQ_CUDA(cudaEventDestroy(static_cast<cudaEvent_t>(event)));
  return SQ_OK;
}
int sq_event_record(void *event, void *stream) {
  if (!event) return fail(SQ_ERR_INVALID, "null event");
  SQ_CUDA(cudaEventRecord(static_cast<cudaEvent_t>(event), static_cast<cudaStream_t>(stream)));
  return SQ_OK;
}
int sq_event_synchronize(void *event) {
  if (!event) return fail(SQ_ERR_INVALID, "null event");
  SQ_CUDA(cudaEventSynchronize(static_cast<cudaEvent_t>(event)));
  return SQ_OK;
}
int sq_event_elapsed(void *start, void *stop, float *ms) {
  if (!start || !stop || !ms) return fail(SQ_ERR_INVALID, "null pointer");
  SQ_CUDA(cudaEventElapsedTime(ms, static_cast<cudaEvent_t>(start), static_cast<cudaEvent_t>(stop)));
  return SQ_OK;
}
int sq_host_alloc(void **ptr, size_t bytes) {
  if (!ptr) return fail(SQ_ERR_INVALID, "null pointer");
  SQ_CUDA(cudaHostAlloc(ptr, bytes, cudaHostAllocDefault));
  return SQ_OK;
}
int sq_host_free(void *ptr) {
  if (ptr) SQ_CUDA(cudaFreeHost(ptr));
  return SQ_OK;
}

int sq_gate_qubits(int gate) { return sq::gate_qubits(gate); }

int sq_gate_matrix_derivative(int gate, const double *angles, uint32_t nangles, uint32_t param,
                              double *out, uint32_t *k) {
  if (!out || (nangles && !angles)) return fail(SQ_ERR_INVALID, "null pointer");
  std::vector<cplx> m;
  const int kk = sq::gate_matrix_derivative(gate, angles, nangles, int(param), m);
  if (kk < 0) return fail(SQ_ERR_INVALID, "gate %d has no angle %u", gate, param);
  std::memcpy(out, m.data(), m.size() * sizeof(cplx));
  if (k) *k = uint32_t(kk);
  return SQ_OK;
}

int sq_gate_matrix(int gate, const double *angles, uint32_t nangles, double *out, uint32_t *k) {
  if (!out) return fail(SQ_ERR_INVALID, "null output");
  if (nangles && !angles) return fail(SQ_ERR_INVALID, "null angles");
  std::vector<cplx> m;
  const int kk = sq::gate_matrix(gate, angles, nangles, m);
  if (kk < 0) return fail(SQ_ERR_INVALID, "unknown gate %d or too few angles (%u)", gate, nangles);
  std::memcpy(out, m.data(), m.size() * sizeof(cplx));
  if (k) *k = uint32_t(kk);
  return SQ_OK;
}

int sq_state_create(uint32_t num_qubits, int dtype, sq_state **out) {
  if (!out) return fail(SQ_ERR_INVALID, "null output");
  if (dtype != SQ_C128 && dtype != SQ_C64) return fail(SQ_ERR_INVALID, "bad dtype %d", dtype);
  if (num_qubits > 40) return fail(SQ_ERR_UNSUPPORTED, "%u qubits exceed one GPU", num_qubits);
  auto s = std::make_unique<sq_state>();
  s->n = num_qubits;
  s->dtype = dtype;
  s->tile_bits = dtype == SQ_C64 ? sq::kDefaultTileBitsC64 : sq::kDefaultTileBitsC128;
  SQ_CUDA(cudaGetDevice(&s->device));
  const size_t bytes = (size_t(1) << num_qubits) * amp_bytes(dtype);
  const cudaError_t e = cudaMalloc(&s->data, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    s->data = nullptr;
    return fail(SQ_ERR_OOM, "cannot allocate %zu bytes of device memory for a %u-qubit state", bytes,
                num_qubits);
  }
  SQ_CUDA(e);
  const int es = alloc_errword(s.get());
  if (es != SQ_OK) {
    cudaFree(s->data);
    return es;
  }
  *out = s.release();
  return SQ_OK;
}

int sq_state_wrap(void *device_ptr, uint32_t num_qubits, int dtype, sq_state **out) {
  if (!out || !device_ptr) return fail(SQ_ERR_INVALID, "null pointer");
  if (dtype != SQ_C128 && dtype != SQ_C64) return fail(SQ_ERR_INVALID, "bad dtype %d", dtype);
  if (reinterpret_cast<uintptr_t>(device_ptr) % 16)
    return fail(SQ_ERR_INVALID, "state memory must be 16-byte aligned");
  auto s = std::make_unique<sq_state>();
  s->n = num_qubits;
  s->dtype = dtype;
  s->data = device_ptr;
  s->owns = false;
  s->tile_bits = dtype == SQ_C64 ? sq::kDefaultTileBitsC64 : sq::kDefaultTileBitsC128;
  SQ_CUDA(cudaGetDevice(&s->device));
  SQ_TRY(alloc_errword(s.get()));
  *out = s.release();
  return SQ_OK;
}

int sq_state_destroy(sq_state *s) {
  if (!s) return SQ_OK;
  std::unique_ptr<sq_state> holder(s);
  SQ_TRY(use_device(s->device));
  if (s->owns && s->data) SQ_CUDA(cudaFree(s->data));
  if (s->scratch) SQ_CUDA(cudaFree(s->scratch));
  if (s->errword) SQ_CUDA(cudaFree(s->errword));
  if (s->rscratch) SQ_CUDA(cudaFree(s->rscratch));
  if (s->hscratch) SQ_CUDA(cudaFreeHost(s->hscratch));
  for (auto &ev : s->sweep_events) {
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
  }
  return SQ_OK;
}

void *sq_state_data(const sq_state *s) { return s ? s->data : nullptr; }
uint32_t sq_state_num_qubits(const sq_state *s) { return s ? s->n : 0; }
int sq_state_dtype(const sq_state *s) { return s ? s->dtype : -1; }

int sq_set_option(sq_state *s, int option, int64_t value) {
  if (!s) return fail(SQ_ERR_INVALID, "null state");
  switch (option) {
    case SQ_OPT_FUSION: s->fusion = value != 0; return SQ_OK;
    case SQ_OPT_TILE_BITS:
      if (value < 4 || value > sq::kMaxTileBits)
        return fail(SQ_ERR_INVALID, "tile bits must be in [4, %d]", sq::kMaxTileBits);
      s->tile_bits = uint32_t(value);
      return SQ_OK;
    case SQ_OPT_REORDER: s->reorder = value != 0; return SQ_OK;
    case SQ_OPT_TIMING: s->timing = value != 0; return SQ_OK;
    case SQ_OPT_REMAP: s->remap = value != 0; return SQ_OK;
    case SQ_OPT_LOW_BITS:
      if (value < 0 || value > 8) return fail(SQ_ERR_INVALID, "SQ_OPT_LOW_BITS takes 0..8");
      s->low_bits = uint32_t(value);
      return SQ_OK;
    case SQ_OPT_JIT:
      if (value < -1 || value > 1) return fail(SQ_ERR_INVALID, "SQ_OPT_JIT takes -1, 0 or 1");
      s->jit = int(value);
      return SQ_OK;
    default: return fail(SQ_ERR_INVALID, "unknown option %d", option);
  }
}

int sq_init_zero(sq_state *s, void *stream) {
  if (!s) return fail(SQ_ERR_INVALID, "null state");
  SQ_TRY(use_device(s->device));
  s->pending.clear();
  const size_t bytes = (size_t(1) << s->n) * amp_bytes(s->dtype);
  SQ_CUDA(cudaMemsetAsync(s->data, 0, bytes, static_cast<cudaStream_t>(stream)));
  return SQ_OK;
}

int sq_init_basis(sq_state *s, uint64_t index, void *stream) {
  if (!s) return fail(SQ_ERR_INVALID, "null state");
  if (index >= (uint64_t(1) << s->n)) return fail(SQ_ERR_INVALID, "basis index out of range");
  SQ_TRY(sq_init_zero(s, stream));
  auto st = static_cast<cudaStream_t>(stream);
  if (s->dtype == SQ_C64)
    sq::set_amplitude_kernel<float><<<1, 1, 0, st>>>(static_cast<float2 *>(s->data), index, 1.f, 0.f);
  else
    sq::set_amplitude_kernel<double><<<1, 1, 0, st>>>(static_cast<double2 *>(s->data), index, 1.0, 0.0);
  SQ_CUDA(cudaGetLastError());
  return SQ_OK;
}

static int validate_qubits(const sq_state *s, const uint32_t *q, uint32_t k, const uint32_t *c,
                           uint32_t nc) {
  uint64_t seen = 0;
  for (uint32_t i = 0; i < k + nc; ++i) {
    const uint32_t x = i < k ? q[i] : c[i - k];
    if (x >= s->n) return fail(SQ_ERR_INVALID, "qubit %u out of range for %u qubits", x, s->n);
    if ((seen >> x) & 1) return fail(SQ_ERR_INVALID, "qubit %u repeated", x);
    seen |= uint64_t(1) << x;
  }
  return SQ_OK;
}

int sq_apply_controlled_matrix(sq_state *s, const double *matrix, const uint32_t *qubits,
                               uint32_t k, const uint32_t *controls,
                               const uint8_t *control_values, uint32_t nc, void *stream) {
  (void)stream;
  if (!s || !matrix) return fail(SQ_ERR_INVALID, "null pointer");
  if (k > 10) return fail(SQ_ERR_UNSUPPORTED, "gates act on at most 10 qubits (got %u)", k);
  if ((k && !qubits) || (nc && !controls)) return fail(SQ_ERR_INVALID, "null qubit list");
  SQ_TRY(validate_qubits(s, qubits, k, controls, nc));
  PendingOp p;
  const size_t d = size_t(1) << k;
  p.m.resize(d * d);
  std::memcpy(p.m.data(), matrix, d * d * sizeof(cplx));
  p.qubits.assign(qubits, qubits + k);
  if (nc) {
    p.controls.assign(controls, controls + nc);
    p.cvals.assign(nc, 1);
    if (control_values)
      for (uint32_t i = 0; i < nc; ++i) p.cvals[i] = control_values[i] ? 1 : 0;
  }
  s->pending.push_back(std::move(p));
  return SQ_OK;
}

int sq_apply_matrix(sq_state *s, const double *matrix, const uint32_t *qubits, uint32_t k,
                    void *stream) {
  return sq_apply_controlled_matrix(s, matrix, qubits, k, nullptr, nullptr, 0, stream);
}

int sq_apply_gate(sq_state *s, int gate, const uint32_t *qubits, uint32_t k, const double *angles,
                  uint32_t nangles, void *stream) {
  if (!s) return fail(SQ_ERR_INVALID, "null state");
  std::vector<cplx> m;
  const int kk = sq::gate_matrix(gate, angles, nangles, m);
  if (kk < 0) return fail(SQ_ERR_INVALID, "unknown gate %d or too few angles (%u)", gate, nangles);
  if (uint32_t(kk) != k) return fail(SQ_ERR_INVALID, "gate %d acts on %d qubits, got %u", gate, kk, k);
  return sq_apply_matrix(s, reinterpret_cast<const double *>(m.data()), qubits, k, stream);
}

int sq_flush(sq_state *s, void *stream) {
  if (!s) return fail(SQ_ERR_INVALID, "null state");
  return flush_impl(s, static_cast<cudaStream_t>(stream));
}

int sq_pending(const sq_state *s, uint32_t *count) {
  if (!s || !count) return fail(SQ_ERR_INVALID, "null pointer");
  *count = uint32_t(s->pending.size());
  return SQ_OK;
}

int sq_launch_count(const sq_state *s, uint64_t *count) {
  if (!s || !count) return fail(SQ_ERR_INVALID, "null pointer");
  *count = s->launches;
  return SQ_OK;
}

int sq_sweep_timing(sq_state *s, double *total_ms, uint64_t *launches) {
  if (!s || !total_ms || !launches) return fail(SQ_ERR_INVALID, "null pointer");
  double tot = 0.0;
  int status = SQ_OK;
  for (auto &ev : s->sweep_events) {
    float ms = 0.f;
    cudaError_t e = cudaEventSynchronize(ev.second);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev.first, ev.second);
    if (e != cudaSuccess && status == SQ_OK)
      status = fail(SQ_ERR_CUDA, "sweep timing: %s", cudaGetErrorString(e));
    tot += ms;
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
  }
  *launches = s->sweep_events.size();
  *total_ms = tot;
  s->sweep_events.clear();
  return status;
}

int sq_apply_gate_buffer(void *buffer, const void *gate_device, const uint64_t *targets,
                         uint32_t ntargets, uint32_t nqubits, uint64_t nelems, void *stream) {
  if (!buffer || (!gate_device) || (ntargets && !targets))
    return fail(SQ_ERR_INVALID, "null pointer");
  if (nqubits > 40 || nelems != (uint64_t(1) << nqubits))
    return fail(SQ_ERR_INVALID, "nelems must be 2^nqubits");
  if (ntargets > uint32_t(sq::kSmallK))
    return fail(SQ_ERR_UNSUPPORTED, "cu::applyGate replacement supports up to 4 targets");
  uint64_t seen = 0;
  sq::HostOp op;
  op.kind = sq::kOpDense;
  for (uint32_t i = 0; i < ntargets; ++i) {
    if (targets[i] >= nqubits || ((seen >> targets[i]) & 1))
      return fail(SQ_ERR_INVALID, "bad or repeated target %llu", (unsigned long long)targets[i]);
    seen |= uint64_t(1) << targets[i];
    op.tbits.push_back(int(nqubits - 1 - targets[i]));
  }
  int dev = 0;
  SQ_CUDA(cudaGetDevice(&dev));
  DeviceInfo di;
  SQ_TRY(device_info(dev, di));
  return launch_gate<double>(buffer, nqubits, op, gate_device, static_cast<cudaStream_t>(stream),
                             di.sms);
}

int sq_copy_to_host(sq_state *s, void *dst, void *stream) {
  if (!s || !dst) return fail(SQ_ERR_INVALID, "null pointer");
  SQ_TRY(flush_impl(s, static_cast<cudaStream_t>(stream)));
  SQ_CUDA(cudaMemcpyAsync(dst, s->data, (size_t(1) << s->n) * amp_bytes(s->dtype),
                          cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
  return SQ_OK;
}

int sq_state_check(sq_state *s, void *stream) {
  if (!s) return fail(SQ_ERR_INVALID, "null pointer");
  SQ_TRY(use_device(s->device));
  SQ_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  return take_kernel_error(s);
}

int sq_copy_from_host(sq_state *s, const void *src, void *stream) {
  if (!s || !src) return fail(SQ_ERR_INVALID, "null pointer");
  SQ_TRY(use_device(s->device));
  s->pending.clear();
  SQ_CUDA(cudaMemcpyAsync(s->data, src, (size_t(1) << s->n) * amp_bytes(s->dtype),
                          cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream)));
  return SQ_OK;
}

int sq_copy_state(sq_state *dst, sq_state *src, void *stream) {
  if (!dst || !src) return fail(SQ_ERR_INVALID, "null pointer");
  if (dst->n != src->n || dst->dtype != src->dtype)
    return fail(SQ_ERR_INVALID, "copy between states of different size or dtype");
  SQ_TRY(flush_impl(src, static_cast<cudaStream_t>(stream)));
  dst->pending.clear();
  SQ_CUDA(cudaMemcpyAsync(dst->data, src->data, (size_t(1) << src->n) * amp_bytes(src->dtype),
                          cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)));
  return SQ_OK;
}

int sq_probabilities(sq_state *s, double *out_device, void *stream) {
  if (!s || !out_device) return fail(SQ_ERR_INVALID, "null pointer");
  auto st = static_cast<cudaStream_t>(stream);
  SQ_TRY(flush_impl(s, st));
  DeviceInfo di;
  SQ_TRY(device_info(s->device, di));
  const uint64_t N = uint64_t(1) << s->n;
  const uint64_t blocks =
      std::max<uint64_t>(1, std::min<uint64_t>((N + 255) / 256, uint64_t(di.sms) * 8));
  if (s->dtype == SQ_C64)
    sq::probabilities_kernel<float><<<unsigned(blocks), 256, 0, st>>>(
        static_cast<const float2 *>(s->data), N, out_device);
  else
    sq::probabilities_kernel<double><<<unsigned(blocks), 256, 0, st>>>(
        static_cast<const double2 *>(s->data), N, out_device);
  SQ_CUDA(cudaGetLastError());
  return SQ_OK;
}

// Groups Pauli terms by (flip mask, Y parity) and runs the expectation
// kernel over each batch of groups; returns the FP64 sum.
static int expect_impl(sq_state *s, const std::vector<uint64_t> &xm,
                       const std::vector<uint64_t> &zym, const std::vector<int> &ny,
                       const std::vector<double> &w, double *out, cudaStream_t st) {
  SQ_TRY(flush_impl(s, st));
  DeviceInfo di;
  SQ_TRY(device_info(s->device, di));
  const uint32_t n = s->n;
  // Sort term indices by (x, parity).
  std::vector<size_t> idx(xm.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
    if (xm[a] != xm[b]) return xm[a] < xm[b];
    return (ny[a] & 1) < (ny[b] & 1);
  });
  const uint64_t pairs = n ? (uint64_t(1) << (n - 1)) : 1;
  const uint32_t blocks = uint32_t(std::max<uint64_t>(
      1, std::min<uint64_t>((pairs + sq::kReduceThreads - 1) / sq::kReduceThreads,
                            uint64_t(di.sms) * 4)));
  SQ_TRY(ensure_scratch(s, blocks + 1));
  auto P = std::make_unique<sq::PauliParams>();
  bool first_launch = true;
  size_t pos = 0;
  while (pos < idx.size() || first_launch) {
    std::memset(P.get(), 0, sizeof(*P));
    P->n = n;
    uint32_t nt = 0;
    while (pos < idx.size()) {
      const size_t i0 = idx[pos];
      size_t end = pos;
      while (end < idx.size() && xm[idx[end]] == xm[i0] && ((ny[idx[end]] & 1) == (ny[i0] & 1)))
        ++end;
      const size_t cnt = end - pos;
      if (P->ngroups >= uint32_t(sq::kMaxGroups) || nt + cnt > size_t(sq::kMaxTerms)) {
        if (nt == 0) return fail(SQ_ERR_UNSUPPORTED, "more than %d terms share one Pauli group",
                                 sq::kMaxTerms);
        break;
      }
      sq::PauliGroup &g = P->g[P->ngroups++];
      g.x = xm[i0];
      g.odd = ny[i0] & 1;
      g.t0 = nt;
      for (size_t e = pos; e < end; ++e) {
        const size_t t = idx[e];
        // (-i)^ny folded into a real factor: even ny -> Re((-i)^ny) = (-1)^(ny/2);
        // odd ny -> -Im((-i)^ny) = (-1)^((ny-1)/2).
        const int half = ny[t] / 2;
        const double sign = (half & 1) ? -1.0 : 1.0;
        P->zy[nt] = zym[t];
        P->f[nt] = w[t] * sign;
        ++nt;
      }
      g.t1 = nt;
      pos = end;
    }
    if (s->dtype == SQ_C64)
      sq::pauli_expect_kernel<float><<<blocks, sq::kReduceThreads, 0, st>>>(
          static_cast<const float2 *>(s->data), *P, s->scratch, first_launch ? 0 : 1);
    else
      sq::pauli_expect_kernel<double><<<blocks, sq::kReduceThreads, 0, st>>>(
          static_cast<const double2 *>(s->data), *P, s->scratch, first_launch ? 0 : 1);
    SQ_CUDA(cudaGetLastError());
    first_launch = false;
  }
  sq::finalize_sum_kernel<<<1, sq::kReduceThreads, 0, st>>>(s->scratch, blocks, s->scratch + blocks);
  SQ_CUDA(cudaGetLastError());
  SQ_CUDA(cudaMemcpyAsync(out, s->scratch + blocks, sizeof(double), cudaMemcpyDeviceToHost, st));
  SQ_CUDA(cudaStreamSynchronize(st));
  return take_kernel_error(s);
}

int sq_expect_pauli(sq_state *s, const char *paulis, const double *weights, uint32_t n_terms,
                    double *out, void *stream) {
  if (!s || !out || (n_terms && (!paulis || !weights))) return fail(SQ_ERR_INVALID, "null pointer");
  SQ_TRY(use_device(s->device));
  const uint32_t n = s->n;
  std::vector<uint64_t> xm(n_terms), zym(n_terms);
  std::vector<int> ny(n_terms);
  std::vector<double> w(weights, weights + n_terms);
  for (uint32_t t = 0; t < n_terms; ++t) {
    for (uint32_t q = 0; q < n; ++q) {
      const uint64_t bit = uint64_t(1) << (n - 1 - q);
      switch (paulis[size_t(t) * n + q]) {
        case 'I': case 'i': break;
        case 'X': case 'x': xm[t] |= bit; break;
        case 'Y': case 'y': xm[t] |= bit; zym[t] |= bit; ny[t]++; break;
        case 'Z': case 'z': zym[t] |= bit; break;
        default:
          return fail(SQ_ERR_INVALID, "term %u: bad Pauli character at qubit %u", t, q);
      }
    }
  }
  return expect_impl(s, xm, zym, ny, w, out, static_cast<cudaStream_t>(stream));
}

// Pauli strings -> (flip mask, Z-or-Y mask, Y count) per term.
static int parse_paulis(uint32_t n, const char *paulis, uint32_t n_terms, std::vector<uint64_t> &xm,
                        std::vector<uint64_t> &zym, std::vector<int> &ny) {
  xm.assign(n_terms, 0);
  zym.assign(n_terms, 0);
  ny.assign(n_terms, 0);
  for (uint32_t t = 0; t < n_terms; ++t) {
    for (uint32_t q = 0; q < n; ++q) {
      const uint64_t bit = uint64_t(1) << (n - 1 - q);
      switch (paulis[size_t(t) * n + q]) {
        case 'I': case 'i': break;
        case 'X': case 'x': xm[t] |= bit; break;
        case 'Y': case 'y': xm[t] |= bit; zym[t] |= bit; ny[t]++; break;
        case 'Z': case 'z': zym[t] |= bit; break;
        default:
          return fail(SQ_ERR_INVALID, "term %u: bad Pauli character at qubit %u", t, q);
      }
    }
  }
  return SQ_OK;
}

int sq_variance_pauli(sq_state *s, const char *paulis, const double *weights, uint32_t n_terms,
                      double *out, void *stream) {
  if (!s || !out || (n_terms && (!paulis || !weights))) return fail(SQ_ERR_INVALID, "null pointer");
  if (n_terms > 1024) return fail(SQ_ERR_UNSUPPORTED, "sq_variance_pauli: more than 1024 terms");
  SQ_TRY(use_device(s->device));
  const uint32_t n = s->n;
  auto st = static_cast<cudaStream_t>(stream);
  std::vector<uint64_t> xm, zym;
  std::vector<int> ny;
  SQ_TRY(parse_paulis(n, paulis, n_terms, xm, zym, ny));
  std::vector<double> w(weights, weights + n_terms);
  double e1 = 0.0;
  SQ_TRY(expect_impl(s, xm, zym, ny, w, &e1, st));
  // H^2 = sum_{s,t} w_s w_t P_s P_t.  With P = i^ny X^x Z^z (x = flip mask,
  // z = Z-or-Y mask): P_s P_t = i^(ny_s + ny_t) (-1)^popc(z_s & x_t)
  // X^(x_s ^ x_t) Z^(z_s ^ z_t), which is i^(ny_s + ny_t - ny_u) (-1)^...
  // times the Pauli string P_u with x_u = x_s ^ x_t, z_u = z_s ^ z_t.
  std::map<std::pair<uint64_t, uint64_t>, std::complex<double>> acc;
  for (uint32_t a = 0; a < n_terms; ++a)
    for (uint32_t b = 0; b < n_terms; ++b) {
      const uint64_t xu = xm[a] ^ xm[b], zu = zym[a] ^ zym[b];
      const int nyu = __builtin_popcountll(xu & zu);
      int ph = (ny[a] + ny[b] - nyu) % 4;
      if (ph < 0) ph += 4;
      if (__builtin_popcountll(zym[a] & xm[b]) & 1) ph = (ph + 2) % 4;
      static const std::complex<double> ipow[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
      acc[{xu, zu}] += ipow[ph] * (w[a] * w[b]);
    }
  std::vector<uint64_t> x2, z2;
  std::vector<int> ny2;
  std::vector<double> w2;
  for (const auto &kv : acc) {
    if (kv.second.real() == 0.0) continue;  // anticommuting pairs cancel
    x2.push_back(kv.first.first);
    z2.push_back(kv.first.second);
    ny2.push_back(__builtin_popcountll(kv.first.first & kv.first.second));
    w2.push_back(kv.second.real());
  }
  if (x2.empty()) {
    x2.push_back(0);
    z2.push_back(0);
    ny2.push_back(0);
    w2.push_back(0.0);
  }
  double e2 = 0.0;
  SQ_TRY(expect_impl(s, x2, z2, ny2, w2, &e2, st));
  *out = e2 - e1 * e1;
  return SQ_OK;
}

int sq_norm2(sq_state *s, double *out, void *stream) {
  if (!s || !out) return fail(SQ_ERR_INVALID, "null pointer");
  SQ_TRY(use_device(s->device));
  return expect_impl(s, {0}, {0}, {0}, {1.0}, out, static_cast<cudaStream_t>(stream));
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Adjoint gradient
// ---------------------------------------------------------------------------
namespace {

// lambda = H psi (Pauli-string sum) and E = Re <psi|lambda>, on `st`.
template <typename Real>
int pauli_apply(sq_state *psi, sq_state *lam, const char *paulis, const double *w, uint32_t nt,
                double *partial, uint32_t blocks, double *e_dev, cudaStream_t st) {
  using C2 = typename sq::Vec2<Real>::T;
  const uint32_t n = psi->n;
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
        default: return fail(SQ_ERR_INVALID, "term %u: bad Pauli character", t);
      }
    }
  std::vector<uint32_t> idx(nt);
  for (uint32_t i = 0; i < nt; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return xm[a] < xm[b]; });
  auto P = std::make_unique<sq::PauliApplyParams>();
  std::memset(P.get(), 0, sizeof(*P));
  P->n = n;
  uint32_t k = 0;
  for (uint32_t pos = 0; pos < nt;) {
    uint32_t end = pos;
    while (end < nt && xm[idx[end]] == xm[idx[pos]]) ++end;
    if (P->ngroups >= uint32_t(sq::kMaxGroups) || nt > uint32_t(sq::kMaxTerms))
      return fail(SQ_ERR_UNSUPPORTED, "adjoint: at most %d terms in %d flip groups",
                  sq::kMaxTerms, sq::kMaxGroups);
    const uint32_t gi = P->ngroups++;
    sq::PauliApplyGroup &g = P->g[gi];
    g.x = xm[idx[pos]];
    g.t0 = k;
    bool real = true;
    for (uint32_t e = pos; e < end; ++e) {
      const uint32_t t = idx[e];
      static const double pr[4] = {1, 0, -1, 0}, pi[4] = {0, -1, 0, 1};  // (-i)^ny
      P->zy[k] = zym[t];
      P->wr[k] = w[t] * pr[ny[t] & 3];
      P->wi[k] = w[t] * pi[ny[t] & 3];
      real = real && P->wi[k] == 0.0;
      const uint32_t top = uint32_t(zym[t] >> (n - 2)) & 3u;
      for (uint32_t r = 0; r < 4; ++r)
        if (__builtin_popcount(r & top) & 1) P->sgn[k] |= uint8_t(1u << r);
      ++k;
    }
    if (real) P->real[gi >> 5] |= 1u << (gi & 31);
    g.t1 = k;
    pos = end;
  }
  sq::pauli_apply_kernel<Real><<<blocks, sq::kReduceThreads, 0, st>>>(
      static_cast<const C2 *>(psi->data), static_cast<C2 *>(lam->data), *P, partial);
  SQ_CUDA(cudaGetLastError());
  sq::finalize_sum_kernel<<<1, sq::kReduceThreads, 0, st>>>(partial, blocks, e_dev);
  SQ_CUDA(cudaGetLastError());
  return SQ_OK;
}

template <typename Real>
int adjoint_sweep(sq_state *psi, sq_state *lam, const sq::PlannedSweep &ps, double2 *partials,
                  size_t partial_rows, double2 *ipvals, int sms, cudaStream_t st) {
  using C2 = typename sq::Vec2<Real>::T;
  auto P = std::make_unique<sq::SweepParams<Real>>();
  std::memset(P.get(), 0, sizeof(*P));
  P->h = ps.h;
  std::copy(ps.ph.begin(), ps.ph.end(), P->ph);
  std::copy(ps.op.begin(), ps.op.end(), P->op);
  for (size_t i = 0; i < ps.coef.size(); ++i) {
    P->coef[2 * i] = Real(ps.coef[i].real());
    P->coef[2 * i + 1] = Real(ps.coef[i].imag());
  }
  const uint32_t m = ps.h.m;
  const int threads = 1 << (m - sq::kAdjRegBits);
  const int nw = (threads + 31) / 32;
  const void *fn = nullptr;
  size_t smem = 0;
  int per_sm = 0;
  if (use_jit(psi)) {
    std::string err;
    fn = sq::jit_adjoint_kernel(ps, sizeof(Real) == 4, err);
    smem = sq::jit_adjoint_smem(ps, sizeof(Real) == 4);
    if (fn && cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) {
      cudaGetLastError();
      fn = nullptr;
    }
    if (fn && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) {
      cudaGetLastError();
      per_sm = 1;
    }
    sq::jit_note_launch(fn != nullptr);
  }
  if (!fn) {
    fn = adjoint_fn<Real>(m);
    if (!fn) return fail(SQ_ERR_INVALID, "internal: no adjoint kernel for %u tile bits", m);
    smem = adjoint_smem<Real>(m, ps.h.ncoef);
    SQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
  }
  if (per_sm < 1) per_sm = 1;
  const uint64_t grid = std::min<uint64_t>(
      std::min<uint64_t>(ps.h.num_tiles, uint64_t(per_sm) * sms), partial_rows / uint64_t(nw));
  C2 *a = static_cast<C2 *>(psi->data);
  C2 *b = static_cast<C2 *>(lam->data);
  void *args[] = {&a, &b, P.get(), &partials};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (psi->timing) {
    SQ_CUDA(cudaEventCreate(&e0));
    SQ_CUDA(cudaEventCreate(&e1));
    SQ_CUDA(cudaEventRecord(e0, st));
  }
  SQ_CUDA(cudaLaunchKernel(fn, dim3(unsigned(grid)), dim3(threads), args, smem, st));
  if (psi->timing) {
    SQ_CUDA(cudaEventRecord(e1, st));
    psi->sweep_events.emplace_back(e0, e1);
  }
  psi->launches++;
  if (!ps.inner_global.empty()) {
    sq::InnerSlots S;
    std::memset(&S, 0, sizeof(S));
    S.nslots = uint32_t(ps.inner_global.size());
    S.nrows = uint32_t(grid) * uint32_t(nw);
    std::copy(ps.inner_global.begin(), ps.inner_global.end(), S.global);
    sq::inner_reduce_kernel<<<S.nslots, sq::kReduceThreads, 0, st>>>(partials, S, ipvals);
    SQ_CUDA(cudaGetLastError());
  }
  return SQ_OK;
}

template <typename Real>
int adjoint_impl(sq_state *psi, sq_state *lam, const sq::AdjointPlan &ap, const char *paulis,
                 const double *w, uint32_t nt, double *energy, std::vector<double2> &ip,
                 cudaStream_t st) {
  DeviceInfo di;
  SQ_TRY(device_info(psi->device, di));
  const uint32_t n = psi->n;
  // Forward pass on psi.
  SQ_TRY(sq_init_basis(psi, 0, st));
  sq::PlanOptions fopt;
  fopt.tile_bits = pick_tile_bits(psi->dtype, n, psi->tile_bits);
  fopt.max_dense_k = sizeof(Real) == 4 ? 4 : 3;
  std::vector<sq::PlannedLaunch> fplan, rplan;
  sq::PlanOptions ropt;
  ropt.tile_bits = pick_adjoint_tile_bits(psi->dtype, n);
  ropt.reg_bits = sq::kAdjRegBits;
  ropt.max_dense_k = sq::kAdjRegBits;
  // The reverse pass is planned (and its JIT kernels looked up or compiled)
  // on a second host thread while this one plans and launches the forward
  // pass, so its planning overlaps the forward sweeps on the device.
  std::string rerr;
  const bool jit = use_jit(psi);
  std::thread rthread([&] {
    try {
      rplan = plan_memo(psi->rev_memo, ap.reverse, n, ropt);
      if (jit) {
        std::vector<const sq::PlannedSweep *> sweeps;
        for (const auto &pl : rplan)
          if (pl.is_sweep) sweeps.push_back(&pl.sweep);
        sq::jit_prepare_adjoint(sweeps, sizeof(Real) == 4);
      }
    } catch (const std::exception &e) {
      rerr = e.what();
    }
  });
  struct Joiner {
    std::thread &t;
    ~Joiner() {
      if (t.joinable()) t.join();
    }
  } joiner{rthread};
  try {
    fplan = plan_memo(psi->fwd_memo, ap.forward, n, fopt);
  } catch (const std::exception &e) {
    return fail(SQ_ERR_INVALID, "adjoint planner: %s", e.what());
  }
  for (const auto &pl : fplan) {
    if (pl.is_sweep) {
      SQ_TRY(launch_sweep<Real>(psi, pl.sweep, st));
    } else {
      SQ_TRY(launch_gate<Real>(psi->data, n, as_dense(pl.gate), nullptr, st, di.sms));
    }
  }
  rthread.join();
  if (!rerr.empty()) return fail(SQ_ERR_INVALID, "adjoint planner: %s", rerr.c_str());
  // Device scratch for this call (stream-ordered).
  const uint32_t red_blocks = uint32_t(std::max<uint64_t>(
      1, std::min<uint64_t>(((uint64_t(1) << n) + sq::kReduceThreads - 1) / sq::kReduceThreads,
                            uint64_t(di.sms) * 4)));
  const size_t rows = size_t(di.sms) * 64;  // blocks x warps of one adjoint launch, at most
  const size_t nip = std::max<size_t>(1, ap.occurrences.size());
  void *scratch = nullptr;
  const size_t bytes = (red_blocks + 2) * sizeof(double) + nip * sizeof(double2) +
                       rows * sq::kMaxInner * sizeof(double2) + 64;
  SQ_CUDA(cudaMallocAsync(&scratch, bytes, st));
  auto *red = static_cast<double *>(scratch);
  auto *e_dev = red + red_blocks;
  auto *ipvals = reinterpret_cast<double2 *>(
      (reinterpret_cast<uintptr_t>(e_dev + 2) + 15) & ~uintptr_t(15));
  auto *partials = ipvals + nip;
  int status = SQ_OK;
  auto run = [&]() -> int {
    SQ_CUDA(cudaMemsetAsync(ipvals, 0, nip * sizeof(double2), st));
    SQ_TRY(pauli_apply<Real>(psi, lam, paulis, w, nt, red, red_blocks, e_dev, st));
    for (const auto &pl : rplan) {
      if (pl.is_sweep) {
        SQ_TRY(adjoint_sweep<Real>(psi, lam, pl.sweep, partials, rows, ipvals, di.sms, st));
      } else {
        const sq::HostOp d = as_dense(pl.gate);
        SQ_TRY(launch_gate<Real>(psi->data, n, d, nullptr, st, di.sms));
        SQ_TRY(launch_gate<Real>(lam->data, n, d, nullptr, st, di.sms));
      }
    }
    ip.assign(nip, make_double2(0.0, 0.0));
    SQ_CUDA(cudaMemcpyAsync(ip.data(), ipvals, nip * sizeof(double2), cudaMemcpyDeviceToHost, st));
    SQ_CUDA(cudaMemcpyAsync(energy, e_dev, sizeof(double), cudaMemcpyDeviceToHost, st));
    SQ_CUDA(cudaStreamSynchronize(st));
    return SQ_OK;
  };
  status = run();
  cudaFreeAsync(scratch, st);
  return status;
}

}  // namespace

extern "C" int sq_adjoint_gradient(sq_state *psi, sq_state *lam, const sq_circuit_op *ops,
                                   uint32_t nops, const char *paulis, const double *weights,
                                   uint32_t n_terms, uint32_t n_params, double *energy,
                                   double *grad, void *stream) {
  if (!psi || !lam || (nops && !ops) || (n_terms && (!paulis || !weights)) || !energy ||
      (n_params && !grad))
    return fail(SQ_ERR_INVALID, "null pointer");
  if (psi == lam || psi->n != lam->n || psi->dtype != lam->dtype)
    return fail(SQ_ERR_INVALID, "adjoint: psi and lam must be two states of one size and precision");
  if (psi->n < uint32_t(sq::kRegBits))
    return fail(SQ_ERR_UNSUPPORTED, "adjoint: needs at least 4 qubits");
  SQ_TRY(use_device(psi->device));
  psi->pending.clear();
  lam->pending.clear();
  sq::AdjointPlan ap;
  try {
    sq::build_adjoint(ops, nops, psi->n, ap);
  } catch (const std::exception &e) {
    return fail(SQ_ERR_INVALID, "%s", e.what());
  }
  for (const auto &oc : ap.occurrences)
    if (oc.first >= int32_t(n_params))
      return fail(SQ_ERR_INVALID, "adjoint: parameter index %d >= n_params %u", oc.first, n_params);
  std::vector<double2> ip;
  auto st = static_cast<cudaStream_t>(stream);
  SQ_TRY(psi->dtype == SQ_C64
             ? adjoint_impl<float>(psi, lam, ap, paulis, weights, n_terms, energy, ip, st)
             : adjoint_impl<double>(psi, lam, ap, paulis, weights, n_terms, energy, ip, st));
  for (uint32_t p = 0; p < n_params; ++p) grad[p] = 0.0;
  for (size_t s = 0; s < ap.occurrences.size(); ++s) {
    const auto &oc = ap.occurrences[s];
    if (oc.first >= 0) grad[oc.first] += 2.0 * ip[s].x * oc.second;
  }
  return SQ_OK;
}

// JIT-specialised sweep kernels.
//
// For every planned sweep, generate a kernel whose phases are straight-line
// code: register positions, op kinds, masks and coefficient offsets are
// compile-time constants (the coefficient VALUES stay kernel parameters, so
// one compiled kernel serves every angle of the same circuit structure).
// Without a runtime op loop the compiler keeps each gate's results in fresh
// registers instead of moving them back after every gate, and no op is
// dispatched; measured on B200 this cuts the per-gate cost inside a sweep by
// about 4x.  Kernels are compiled with NVRTC (loaded with dlopen, so the
// library still loads where NVRTC is absent), loaded with
// cudaLibraryLoadData, and cached in memory and on disk by a hash of the
// generated source.  When NVRTC is unavailable or a compile fails, the engine
// runs the same sweep with the generic (runtime-dispatched) sweep kernel.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/snuqs_b200.h"
#include "adjoint_plan.h"
#include "host_ops.h"
#include "jit.h"
#include "jit_batch.cuh"
#include "jit_kernels.cuh"
#include "sweep_kernels.cuh"

int sq_detail_fail(int code, const char *msg);  // engine.cu: sets sq_last_error()

namespace sq {

namespace {

#include "jit_sources.inc"  // kJit{Plan,Sweep,Kernels,Reduce,Batch}Source (generated by build.py)

// --- NVRTC through dlopen -------------------------------------------------
typedef int nvrtcResult_t;
typedef struct _nvrtcProgram *nvrtcProgram_t;
struct Nvrtc {
  bool ok = false;
  nvrtcResult_t (*create)(nvrtcProgram_t *, const char *, const char *, int, const char *const *,
                          const char *const *) = nullptr;
  nvrtcResult_t (*compile)(nvrtcProgram_t, int, const char *const *) = nullptr;
  nvrtcResult_t (*log_size)(nvrtcProgram_t, size_t *) = nullptr;
  nvrtcResult_t (*log)(nvrtcProgram_t, char *) = nullptr;
  nvrtcResult_t (*cubin_size)(nvrtcProgram_t, size_t *) = nullptr;
  nvrtcResult_t (*cubin)(nvrtcProgram_t, char *) = nullptr;
  nvrtcResult_t (*destroy)(nvrtcProgram_t *) = nullptr;
};

Nvrtc &nvrtc() {
  static Nvrtc n;
  static std::once_flag once;
  std::call_once(once, [] {
    const char *names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
    void *h = nullptr;
    for (const char *nm : names)
      if ((h = dlopen(nm, RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) return;
    n.create = reinterpret_cast<decltype(n.create)>(dlsym(h, "nvrtcCreateProgram"));
    n.compile = reinterpret_cast<decltype(n.compile)>(dlsym(h, "nvrtcCompileProgram"));
    n.log_size = reinterpret_cast<decltype(n.log_size)>(dlsym(h, "nvrtcGetProgramLogSize"));
    n.log = reinterpret_cast<decltype(n.log)>(dlsym(h, "nvrtcGetProgramLog"));
    n.cubin_size = reinterpret_cast<decltype(n.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
    n.cubin = reinterpret_cast<decltype(n.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
    n.destroy = reinterpret_cast<decltype(n.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
    n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
  });
  return n;
}

uint64_t fnv1a(const std::string &s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

std::string cache_dir() {
  const char *e = std::getenv("SQ_JIT_CACHE");
  std::string d;
  if (e && *e) {
    d = e;
  } else {
    const char *home = std::getenv("HOME");
    d = std::string(home && *home ? home : "/tmp") + "/.cache/snuqs_b200_jit";
  }
  return d;
}

void mkdirs(const std::string &path) {
  std::string cur;
  std::stringstream ss(path);
  std::string part;
  if (!path.empty() && path[0] == '/') cur = "/";
  while (std::getline(ss, part, '/')) {
    if (part.empty()) continue;
    cur += part + "/";
    mkdir(cur.c_str(), 0755);
  }
}

struct Entry {
  cudaLibrary_t lib = nullptr;
  cudaKernel_t kernel = nullptr;
  bool failed = false;
  std::string err;
};

std::mutex g_mu;
std::map<uint64_t, Entry> g_cache;

// NVRTC compile of one kernel source -> cubin bytes.
bool compile(const std::string &src, std::vector<char> &cubin, std::string &err) {
  Nvrtc &nv = nvrtc();
  if (!nv.ok) {
    err = "NVRTC not available";
    return false;
  }
  nvrtcProgram_t prog = nullptr;
  if (nv.create(&prog, src.c_str(), "sq_jit.cu", 0, nullptr, nullptr) != 0) {
    err = "nvrtcCreateProgram failed";
    return false;
  }
  const char *opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-DSQ_JIT=1", "-lineinfo"};
  const int rc = nv.compile(prog, 4, opts);
  if (rc != 0) {
    size_t n = 0;
    nv.log_size(prog, &n);
    std::string log(n, '\0');
    if (n) nv.log(prog, &log[0]);
    err = "NVRTC compile failed: " + log.substr(0, 2000);
    nv.destroy(&prog);
    return false;
  }
  size_t n = 0;
  nv.cubin_size(prog, &n);
  cubin.resize(n);
  nv.cubin(prog, cubin.data());
  nv.destroy(&prog);
  return true;
}

// Header sources generated kernels are compiled with, and their hash.
struct Prelude {
  std::string text;
  uint64_t hash;
};

Prelude make_prelude(bool batch) {
  Prelude p;
  p.text = std::string("typedef unsigned char uint8_t;\ntypedef unsigned short uint16_t;\n"
                       "typedef unsigned int uint32_t;\ntypedef unsigned long long uint64_t;\n"
                       "typedef int int32_t;\ntypedef long long int64_t;\n") +
           kJitPlanSource + "\n" + kJitSweepSource + "\n" + kJitKernelsSource + "\n";
  if (batch) p.text += std::string(kJitReduceSource) + "\n" + kJitBatchSource + "\n";
  p.text += "using namespace sq;\n";
  p.hash = fnv1a(p.text);
  return p;
}

// Sweep kernels (single- and two-state).
const Prelude &sweep_prelude() {
  static const Prelude p = make_prelude(false);
  return p;
}

// Batched-gradient kernels (also need the Pauli and batch types).
const Prelude &batch_prelude() {
  static const Prelude p = make_prelude(true);
  return p;
}

const std::string &prelude() { return sweep_prelude().text; }

// Loads (compiling when not cached) the kernel whose generated part is `body`.
Entry &get_entry(const std::string &body, const char *name = "sq_jit_sweep",
                 const Prelude &pre = sweep_prelude()) {
  const uint64_t key = fnv1a(body) ^ (pre.hash * 0x9e3779b97f4a7c15ull);
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_cache.find(key);
    if (it != g_cache.end() && (it->second.kernel || it->second.failed)) return it->second;
  }
  Entry e;
  char hex[32];
  std::snprintf(hex, sizeof(hex), "%016llx", static_cast<unsigned long long>(key));
  const std::string dir = cache_dir();
  const std::string file = dir + "/" + hex + ".cubin";
  std::vector<char> cubin;
  {
    std::ifstream in(file, std::ios::binary);
    if (in) cubin.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
  }
  if (cubin.empty()) {
    if (compile(pre.text + body, cubin, e.err)) {
      mkdirs(dir);
      const std::string tmp = file + "." + std::to_string(getpid()) + "." +
                              std::to_string(std::hash<std::thread::id>()(std::this_thread::get_id())) +
                              ".tmp";
      std::ofstream out(tmp, std::ios::binary);
      out.write(cubin.data(), std::streamsize(cubin.size()));
      out.close();
      if (out) std::rename(tmp.c_str(), file.c_str());
      else std::remove(tmp.c_str());
    } else {
      e.failed = true;
    }
  }
  if (!e.failed) {
    cudaError_t ce = cudaLibraryLoadData(&e.lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (ce == cudaSuccess) ce = cudaLibraryGetKernel(&e.kernel, e.lib, name);
    if (ce != cudaSuccess) {
      e.failed = true;
      e.kernel = nullptr;
      e.err = std::string("loading JIT kernel: ") + cudaGetErrorString(ce);
      cudaGetLastError();
    }
  }
  std::lock_guard<std::mutex> lk(g_mu);
  auto &slot = g_cache[key];
  if (!slot.kernel && !slot.failed) slot = e;
  else if (e.lib && e.lib != slot.lib) cudaLibraryUnload(e.lib);
  return slot;
}

const char *op_routine(const SweepOp &op, bool c64, std::string &tmpl, int na = 16) {
  const char *R = c64 ? "float" : "double";
  const int V = op.vmask;
  std::ostringstream o;
  const bool pure = op.aux & kAuxPure;
  switch (op.kind) {
    case kSwPhase:
      o << "op_phase<" << R << ", " << na << ", " << (pure ? "true" : "false") << ">";
      break;
    case kSwDiag:
      o << "op_diag<" << R << ", " << na << ", " << V << ">";
      break;
    case kSwAnti1:
      o << "op_anti1<" << R << ", " << na << ", " << V << ", " << (pure ? "true" : "false") << ">";
      break;
    case kSwSwap2:
      o << "op_swap2<" << R << ", " << na << ", " << V << ", " << (pure ? "true" : "false") << ">";
      break;
    case kSwXRot:
      o << "op_xrot<" << R << ", " << na << ", " << V << ", " << int(op.aux & kAuxXMask) << ", "
        << ((op.aux & kAuxImag) ? "true" : "false") << ">";
      break;
    default:
      o << "op_dense<" << R << ", " << na << ", " << V << ">";
      break;
  }
  tmpl = o.str();
  return tmpl.c_str();
}

std::atomic<uint64_t> g_launches{0}, g_fallbacks{0};

}  // namespace

bool jit_available() { return nvrtc().ok; }

void jit_note_launch(bool jit) { (jit ? g_launches : g_fallbacks)++; }

// Tile positions of the thread bits of a phase: the lane bits that share a
// shared-memory wavefront (the low W) go on non-register positions whose
// swizzle images are linearly independent, the rest ascending.  A phase that
// stores straight to HBM keeps all thread bits ascending (the lanes then
// cover contiguous amplitudes).
std::vector<int> thread_positions(const SweepPhase &ph, int m, bool c64, bool direct_store,
                                  int nreg = kRegBits, const uint8_t *outbits = nullptr) {
  const int W = c64 ? Swz<float>::W : Swz<double>::W;
  const uint8_t *img = c64 ? Swz<float>::kImage : Swz<double>::kImage;
  uint32_t regs = 0;
  for (int b = 0; b < nreg; ++b) regs |= 1u << ph.reg[b];
  std::vector<int> nonreg;
  for (int p = 0; p < m; ++p)
    if (!((regs >> p) & 1)) nonreg.push_back(p);
  if (direct_store) {
    // Lanes on the positions stored to the lowest global bits first.
    if (outbits)
      std::stable_sort(nonreg.begin(), nonreg.end(), [&](int a, int b) { return outbits[a] < outbits[b]; });
    return nonreg;
  }
  std::vector<int> lanes;
  int basis[8] = {0};
  for (int p : nonreg) {
    if (int(lanes.size()) == W) break;
    int x = img[p];
    for (int b = W - 1; b >= 0 && x; --b)
      if ((x >> b) & 1) {
        if (!basis[b]) {
          basis[b] = x;
          lanes.push_back(p);
          x = 0;
        } else {
          x ^= basis[b];
        }
      }
  }
  if (int(lanes.size()) < W || int(nonreg.size()) < W) return nonreg;
  std::vector<int> out = lanes;
  for (int p : nonreg)
    if (std::find(lanes.begin(), lanes.end(), p) == lanes.end()) out.push_back(p);
  return out;
}

// Ops whose coefficients are read from a shared-memory copy rather than the
// parameter block: a diagonal op whose coefficient index depends on tile bits
// that differ across the lanes (a lane-divergent constant read serialises),
// and dense matrices, whose many coefficients are re-read for every register
// group (one 16-byte shared load per complex entry beats two constant loads;
// measured 5x cheaper per 2-qubit dense gate on B200).
bool lane_indexed(const SweepOp &op) {
  if (op.kind == kSwDense) return true;
  if (op.kind != kSwDiag) return false;
  for (int t = 0; t < op.ndt; ++t)
    if (op.dsrc[t] != kSrcGlobal) return true;
  return false;
}

// Call of the inner-product routine of a kSwInnerDiag / kSwInnerDense op
// (`bits`: the statement that sets b, the op's non-register target bits),
// accumulating into doubles sr, si.  Pauli-form ops (kAuxPauli) take the
// four-FMA-per-amplitude routines.
std::string inner_call(const SweepOp &op, const char *R, const std::string &bits) {
  std::ostringstream s;
  const bool pauli = op.aux & kAuxPauli;
  if (op.kind == kSwInnerDiag) {
    s << bits << " ";
    if (pauli)
      s << "inner_diag_pauli<" << R << ", " << int(op.vmask) << ", " << int(op.aux & 7) << ">";
    else
      s << "inner_diag<" << R << ", " << int(op.vmask) << ">";
    s << "(F, G, coef + " << op.coef << ", b, sr, si); ";
  } else {
    if (pauli)
      s << "inner_dense_pauli<" << R << ", " << int(op.vmask) << ", " << int(op.aux & 7) << ", "
        << int((op.aux >> 3) & 7) << ">";
    else
      s << "inner_dense<" << R << ", " << int(op.vmask) << ">";
    s << "(F, G, coef + " << op.coef << ", sr, si); ";
  }
  return s.str();
}

// Fused code for a run of consecutive diagonal ops of one phase (kSwDiag,
// kSwPhase): instead of one complex multiply per amplitude per op, the run's
// factors are multiplied together first and applied once.  Each op's factor
// depends on its register bits V (plus per-thread bits: non-register targets,
// conditions): ops with V = 0 fold into a scalar, ops with the same V into a
// table of 2^|V| entries, and the tables combine into one table T over the
// union U of their register bits, grown one table at a time (2^|U'| products
// each); then every amplitude is multiplied by its T entry.  `coef(op)` is
// the op's coefficient accessor; `na` amplitudes per thread.
namespace {

int bit_ext(int x, int mask) {  // bits of x at mask's positions, packed
  int y = 0, k = 0;
  for (int b = 0; b < 8; ++b)
    if ((mask >> b) & 1) y |= ((x >> b) & 1) << k++;
  return y;
}

int bit_dep(int y, int mask) {  // y's bits deposited at mask's positions
  int x = 0, k = 0;
  for (int b = 0; b < 8; ++b)
    if ((mask >> b) & 1) x |= ((y >> k++) & 1) << b;
  return x;
}

std::string cond_prefix(const SweepOp &op) {
  if (!op.gmask && !op.lmask) return std::string();
  std::ostringstream s;
  s << "if (";
  if (op.gmask) s << "(gbase & 0x" << std::hex << op.gmask << "ull) == 0x" << op.gval << "ull" << std::dec;
  if (op.gmask && op.lmask) s << " && ";
  if (op.lmask) s << "(jb & 0x" << std::hex << op.lmask << "u) == 0x" << op.lval << "u" << std::dec;
  s << ") ";
  return s.str();
}

std::string diag_bits_src(const SweepOp &op) {
  std::ostringstream b;
  b << "uint32_t b = 0;";
  for (int t = 0; t < op.ndt; ++t) {
    if (op.dsrc[t] == kSrcGlobal)
      b << " b = (b << 1) | (uint32_t(gbase >> " << int(op.dpos[t]) << ") & 1u);";
    else
      b << " b = (b << 1) | ((jb >> " << int(op.dpos[t]) << ") & 1u);";
  }
  return b.str();
}

std::string nonreg_cond(const SweepOp &op) {
  std::ostringstream c;
  c << "true";
  if (op.gmask) c << " && (gbase & 0x" << std::hex << op.gmask << "ull) == 0x" << op.gval << "ull" << std::dec;
  if (op.lmask) c << " && (jb & 0x" << std::hex << op.lmask << "u) == 0x" << op.lval << "u" << std::dec;
  return c.str();
}

}  // namespace

// Diagonal runs are fused unless SQ_JIT_FUSE_DIAG=0.
bool jit_fuse_diag() {
  static const bool on = [] {
    const char *e = std::getenv("SQ_JIT_FUSE_DIAG");
    return !(e && e[0] == '0');
  }();
  return on;
}

// An op a fused diagonal run may hold: a diagonal op without conditions, or
// a conditional phase.
bool fusable_diag(const SweepOp &op) {
  return (op.kind == kSwDiag && !op.gmask && !op.lmask && !op.rmask) || op.kind == kSwPhase;
}

// Emission order of one phase's ops: single ops, and runs of diagonal ops
// to fuse.  A diagonal op moves later past the non-diagonal ops it commutes
// with (their targets miss its register bits: conditions are diagonal), so
// the diagonal ops between such ops gather into one run; the order among
// diagonal ops and among the others is kept.
std::vector<std::vector<uint32_t>> phase_items(const SweepOp *ops, const SweepPhase &ph, bool two_state = false) {
  std::vector<std::vector<uint32_t>> items;
  std::vector<uint32_t> pending;
  uint32_t pending_bits = 0;
  auto flush = [&] {
    if (pending.size() >= 2) {
      items.push_back(pending);
    } else {
      for (uint32_t i : pending) items.push_back({i});
    }
    pending.clear();
    pending_bits = 0;
  };
  for (uint32_t oi = ph.op_begin; oi < ph.op_end; ++oi) {
    const SweepOp &op = ops[oi];
    // Two-state sweeps: the inner products of diagonal generators join the
    // runs too (they commute with every diagonal op).
    if (jit_fuse_diag() && (fusable_diag(op) || (two_state && op.kind == kSwInnerDiag))) {
      pending.push_back(oi);
      pending_bits |= op.kind == kSwPhase ? op.rmask : op.vmask;
      continue;
    }
    // An op moves ahead of the pending run when the run's diagonal ops (and
    // the generators of its inner products) commute with it.
    const bool commutes = (two_state || (op.kind != kSwInnerDiag && op.kind != kSwInnerDense)) &&
                          !(op.vmask & pending_bits);
    if (!commutes) flush();
    items.push_back({oi});
  }
  flush();
  return items;
}

std::string diag_run_src(const std::vector<const SweepOp *> &run, const char *R, int na,
                         const std::function<std::string(const SweepOp &)> &coef,
                         const std::vector<std::string> &states = {"A"}) {
  std::ostringstream s;
  s << "      { // " << run.size() << " diagonal ops, fused\n";
  s << "        " << R << " s_r = 1, s_i = 0;\n";
  // Factor tables by register mask, in first-use order.
  std::vector<int> masks;
  std::map<int, bool> started;
  for (const SweepOp *op : run) {
    const int V = op->kind == kSwPhase ? op->rmask : op->vmask;
    const int nv = __builtin_popcount(uint32_t(V)), N = 1 << nv;
    s << "        {\n";
    if (op->kind == kSwDiag) {
      s << "          uint32_t b = 0;";
      for (int t = 0; t < op->ndt; ++t) {
        if (op->dsrc[t] == kSrcGlobal)
          s << " b = (b << 1) | (uint32_t(gbase >> " << int(op->dpos[t]) << ") & 1u);";
        else
          s << " b = (b << 1) | ((jb >> " << int(op->dpos[t]) << ") & 1u);";
      }
      s << "\n          const auto c = " << coef(*op) << ";\n";
    } else {
      s << "          const bool on = " << nonreg_cond(*op) << ";\n";
      if (!(op->aux & kAuxPure)) s << "          const auto c = " << coef(*op) << ";\n";
    }
    const int yv = op->kind == kSwPhase ? bit_ext(op->rval, V) : -1;
    auto factor = [&](int y, std::string &fr, std::string &fi) -> bool {  // false: factor is 1
      if (op->kind == kSwDiag) {
        std::ostringstream a, b;
        a << "c[(b << " << nv << ") | " << y << "u].x";
        b << "c[(b << " << nv << ") | " << y << "u].y";
        fr = a.str();
        fi = b.str();
        return true;
      }
      if (y != yv) return false;
      if (op->aux & kAuxPure) {
        fr = std::string("(on ? ") + R + "(-1) : " + R + "(1))";
        fi = std::string(R) + "(0)";
      } else {
        fr = std::string("(on ? ") + R + "(c[0].x) : " + R + "(1))";
        fi = std::string("(on ? ") + R + "(c[0].y) : " + R + "(0))";
      }
      return true;
    };
    if (V == 0) {
      std::string fr, fi;
      if (factor(0, fr, fi)) s << "          jit_cmul_acc(s_r, s_i, " << R << "(" << fr << "), " << R << "(" << fi << "));\n";
    } else if (!started[V]) {
      started[V] = true;
      masks.push_back(V);
      for (int y = 0; y < N; ++y) {
        std::string fr, fi;
        if (!factor(y, fr, fi)) {
          fr = std::string(R) + "(1)";
          fi = std::string(R) + "(0)";
        }
        s << "          f" << V << "_r[" << y << "] = " << fr << "; f" << V << "_i[" << y << "] = " << fi << ";\n";
      }
    } else {
      for (int y = 0; y < N; ++y) {
        std::string fr, fi;
        if (factor(y, fr, fi))
          s << "          jit_cmul_acc(f" << V << "_r[" << y << "], f" << V << "_i[" << y << "], " << R << "(" << fr
            << "), " << R << "(" << fi << "));\n";
      }
    }
    s << "        }\n";
  }
  // The tables are declared before the op blocks that fill them.
  std::ostringstream decl;
  for (int V : masks) {
    const int N = 1 << __builtin_popcount(uint32_t(V));
    decl << "        " << R << " f" << V << "_r[" << N << "], f" << V << "_i[" << N << "];\n";
  }
  // T over the growing union U, starting from the scalar.
  std::ostringstream t;
  int U = 0;
  t << "        " << R << " t0_r[1] = {s_r}, t0_i[1] = {s_i};\n";
  int step = 0;
  for (int V : masks) {
    const int U2 = U | V, N2 = 1 << __builtin_popcount(uint32_t(U2));
    t << "        " << R << " t" << step + 1 << "_r[" << N2 << "], t" << step + 1 << "_i[" << N2 << "];\n";
    for (int x = 0; x < N2; ++x) {
      const int full = bit_dep(x, U2);
      const int xu = bit_ext(full, U), xv = bit_ext(full, V);
      t << "        jit_cmul(t" << step << "_r[" << xu << "], t" << step << "_i[" << xu << "], f" << V << "_r[" << xv
        << "], f" << V << "_i[" << xv << "], t" << step + 1 << "_r[" << x << "], t" << step + 1 << "_i[" << x << "]);\n";
    }
    U = U2;
    ++step;
  }
  for (const std::string &st : states)
    for (int ri = 0; ri < na; ++ri) {
      const int xu = bit_ext(ri, U);
      t << "        jit_cmul_acc(" << st << ".re[" << ri << "], " << st << ".im[" << ri << "], t" << step << "_r[" << xu
        << "], t" << step << "_i[" << xu << "]);\n";
    }
  const std::string body = s.str();
  const size_t cut = body.find('\n') + 1;  // after the opening line
  std::ostringstream out;
  out << body.substr(0, cut) << decl.str() << body.substr(cut) << t.str() << "      }\n";
  return out.str();
}

// Code of one single-state phase's ops on the registers A (16 amplitudes):
// fused diagonal runs, the other ops one by one.  coef(op): the op's
// coefficient accessor.
void one_state_ops_src(const SweepOp *ops, const SweepPhase &ph, const char *R, bool c64,
                       const std::function<std::string(const SweepOp &)> &coef, std::ostream &s) {
  for (const auto &item : phase_items(ops, ph)) {
    if (item.size() >= 2) {
      std::vector<const SweepOp *> run;
      for (uint32_t oi : item) run.push_back(&ops[oi]);
      s << diag_run_src(run, R, kRegAmps, coef);
      continue;
    }
    const SweepOp &op = ops[item[0]];
    std::string tmpl;
    op_routine(op, c64, tmpl);
    s << "      " << cond_prefix(op);
    if (op.kind == kSwDiag)
      s << "{ " << diag_bits_src(op) << " " << tmpl << "(A, " << coef(op) << ", b); }\n";
    else
      s << tmpl << "(A, " << coef(op) << ", " << int(op.rmask) << ", " << int(op.rval) << ");\n";
  }
}

// Code of one two-state (reverse adjoint) phase's ops on F (phi) and G
// (lambda), coefficients from the shared-memory copy `coef`.  A run of
// diagonal ops and inner products of diagonal generators is emitted as: every
// inner product first (the run's diagonal ops commute with the generators and
// act on both states alike, so they leave <lambda|K|phi> unchanged), the
// Pauli-Z ones from one shared set of products conj(lambda_r) phi_r; then
// the run's diagonal ops, fused, on both states.  False when an op is not
// covered (an inner product with conditions).
bool two_state_ops_src(const SweepOp *ops, const SweepPhase &ph, const char *R, bool c64, int NT, std::ostream &s) {
  auto cf = [](const SweepOp &o) { return "(coef + " + std::to_string(o.coef) + ")"; };
  auto inner_plain = [&](const SweepOp &op) {
    s << "      { double sr = 0.0, si = 0.0; " << inner_call(op, R, diag_bits_src(op)) << "jit_inner_acc<" << NT
      << ", " << op.slot << ">(acc, sr, si); }\n";
  };
  auto single = [&](const SweepOp &op) {
    std::string tmpl;
    op_routine(op, c64, tmpl, kAdjAmps);
    s << "      " << cond_prefix(op);
    if (op.kind == kSwDiag)
      s << "{ " << diag_bits_src(op) << " " << tmpl << "(F, " << cf(op) << ", b); " << tmpl << "(G, " << cf(op)
        << ", b); }\n";
    else
      s << "{ " << tmpl << "(F, " << cf(op) << ", " << int(op.rmask) << ", " << int(op.rval) << "); " << tmpl
        << "(G, " << cf(op) << ", " << int(op.rmask) << ", " << int(op.rval) << "); }\n";
  };
  for (const auto &item : phase_items(ops, ph, true)) {
    for (uint32_t oi : item) {
      const SweepOp &op = ops[oi];
      if ((op.kind == kSwInnerDiag || op.kind == kSwInnerDense) &&
          (op.gmask || op.lmask || op.rmask || op.slot >= uint32_t(kMaxInner)))
        return false;
    }
    if (item.size() == 1) {
      const SweepOp &op = ops[item[0]];
      if (op.kind == kSwInnerDiag || op.kind == kSwInnerDense)
        inner_plain(op);
      else
        single(op);
      continue;
    }
    std::vector<const SweepOp *> diag, pauli;
    for (uint32_t oi : item) {
      const SweepOp &op = ops[oi];
      if (op.kind == kSwInnerDiag && (op.aux & kAuxPauli))
        pauli.push_back(&op);
      else if (op.kind == kSwInnerDiag)
        inner_plain(op);
      else
        diag.push_back(&op);
    }
    if (!pauli.empty()) {
      s << "      { // " << pauli.size() << " Pauli-Z inner products from shared products\n";
      for (int ri = 0; ri < kAdjAmps; ++ri)
        s << "        const double p" << ri << "r = fma(double(G.re[" << ri << "]), double(F.re[" << ri
          << "]), double(G.im[" << ri << "]) * double(F.im[" << ri << "])), p" << ri << "i = fma(double(G.re["
          << ri << "]), double(F.im[" << ri << "]), -double(G.im[" << ri << "]) * double(F.re[" << ri << "]));\n";
      for (const SweepOp *op : pauli) {
        const int V = op->vmask, Z = op->aux & 7, nv = __builtin_popcount(uint32_t(V));
        std::ostringstream qr, qi;
        for (int ri = 0; ri < kAdjAmps; ++ri) {
          const bool neg = __builtin_popcount(uint32_t(bit_ext(ri, V) & Z)) & 1;
          qr << (neg ? " - " : " + ") << "p" << ri << "r";
          qi << (neg ? " - " : " + ") << "p" << ri << "i";
        }
        s << "        { double qr = 0.0" << qr.str() << ", qi = 0.0" << qi.str() << ";";
        if (Z >> nv)
          s << " " << diag_bits_src(*op) << " if (__popc(b & " << (Z >> nv) << "u) & 1) { qr = -qr; qi = -qi; }";
        s << "\n          const auto a = " << cf(*op) << "[0];\n"
          << "          jit_inner_acc<" << NT << ", " << op->slot << ">(acc, double(a.x) * qr - double(a.y) * qi, "
          << "double(a.x) * qi + double(a.y) * qr); }\n";
      }
      s << "      }\n";
    }
    if (diag.size() >= 2)
      s << diag_run_src(diag, R, kAdjAmps, cf, {"F", "G"});
    else if (diag.size() == 1)
      single(*diag[0]);
  }
  return true;
}

struct JitShape {
  bool smem_coef = false, dload = false, dstore = false;
  int stages = 0;     // > 0: bulk-copy pipeline with this many tiles in flight per CTA
  bool work = false;  // pipeline: some phase passes the tile through the work buffer
  bool early = false; // direct load of the next tile's first phase before this tile's phases
};

// Early first-phase loads (jit_sweep_early) for direct-load sweeps, on by
// default: measured on B200 at 30 qubits, 6.84 vs 7.11 ms per complex128
// sweep and 3.59 vs 3.81 ms per complex64 sweep (with direct loads, which
// alone measured slower for complex64).  SQ_JIT_EARLY=0 turns them off.
bool jit_early() {
  static const int env = [] {
    const char *e = std::getenv("SQ_JIT_EARLY");
    return e && *e ? std::atoi(e) : 1;
  }();
  return env == 1;
}

// Tiles in flight per CTA of a pipelined (bulk-copy) sweep; 0 turns the
// pipeline off.  SQ_JIT_STAGES overrides.
int jit_stages(bool c64) {
  static const int env = [] {
    const char *e = std::getenv("SQ_JIT_STAGES");
    return e && *e ? std::atoi(e) : -1;
  }();
  if (env >= 0 && env <= 4) return env;
  // Measured on B200 (30-qubit complex128 mix, 128-byte runs): 11.2 ms per
  // sweep with one stage and 16.4 ms with two, against 7.2 ms for register
  // loads: one cp.async.bulk per 128-byte run is bound by the copy engine's
  // request rate.  Off by default.
  (void)c64;
  return 0;
}

// Direct loads (first phase from HBM, no prefetch into a second tile buffer)
// measured faster on B200 for complex128 (7.10 vs 7.38 ms per 30-qubit sweep)
// and, without early loads, slightly slower for complex64 (3.86 vs 3.76 ms);
// SQ_JIT_DLOAD=0/1 overrides the choice for both precisions.
JitShape jit_shape(const PlannedSweep &ps, bool c64, bool multi = false) {
  static const int dload_env = [] {
    const char *e = std::getenv("SQ_JIT_DLOAD");
    return e && *e ? (e[0] == '0' ? 0 : 1) : -1;
  }();
  const bool dload_on = dload_env < 0 ? (!c64 || jit_early()) : dload_env == 1;
  JitShape j;
  for (const SweepOp &op : ps.op) j.smem_coef |= lane_indexed(op);
  j.dload = dload_on && (ps.h.flags & kDirectLoad);
  j.dstore = (ps.h.flags & kDirectStore) != 0;
  // A one-phase remapping sweep cannot place its lanes for both a coalesced
  // load and a coalesced permuted store: it stores through shared memory.
  if ((ps.h.flags & kRemap) && ps.h.nphases == 1 && (ps.h.flags & kDirectLoad)) j.dstore = false;
  // The pipeline needs a first phase whose lanes cover the low tile bits (a
  // direct-load sweep) and runs of at least 16 bytes.
  // Warp 0 issues the copies: tiles of at least 2^9 amplitudes (32 threads).
  // Multi-state sweeps reload the coefficients per state: always from
  // shared memory, and no bulk-copy pipeline.
  if (multi) j.smem_coef = true;
  const int st = multi ? 0 : jit_stages(c64);
  if (st > 0 && (ps.h.flags & kDirectLoad) && ps.h.m >= 9u &&
      ((1u << ps.h.l) * (c64 ? 8u : 16u)) % 16u == 0) {
    j.stages = st;
    j.dload = false;
    j.work = ps.h.nphases > 1 || !j.dstore;
  } else if (j.dload && jit_early()) {
    j.early = true;
  }
  return j;
}

// Source of the JIT kernel of one planned sweep.  multi: the multi-state
// form sq_jit_msweep (one launch over K states sharing the sweep's
// structure, coefficients per state); empty when the sweep remaps qubits
// (not covered by that form).
std::string jit_body(const PlannedSweep &ps, bool c64, int minb, bool multi, bool from_zero) {
  const char *R = c64 ? "float" : "double";
  const int M = int(ps.h.m);
  const JitShape js = jit_shape(ps, c64, multi);
  if (multi && (ps.h.flags & kRemap)) return std::string();
  // From |0...0>: the first phase must take its registers from HBM (which it
  // then does not read).
  if (from_zero && (!multi || !(js.early || js.dload))) return std::string();
  std::ostringstream nm;
  nm << "0x" << std::hex << ((uint64_t(1) << ps.h.n) - 1) << "ull";
  std::ostringstream s;
  if (multi)
    s << "extern \"C\" __global__ void __launch_bounds__(" << (1 << (M - kRegBits)) << ", " << minb
      << ")\nsq_jit_msweep(Vec2<" << R << ">::T *__restrict__ psi, const __grid_constant__ MultiParams Q) {\n";
  else
    s << "extern \"C\" __global__ void __launch_bounds__(" << (1 << (M - kRegBits)) << ", " << minb
      << ")\nsq_jit_sweep(Vec2<" << R << ">::T *__restrict__ psi, const __grid_constant__ SweepParams<"
      << R << "> P, uint32_t *__restrict__ err) {\n";
  s << "  using C2 = Vec2<" << R << ">::T;\n";
  s << "  using Tile = JitTile<" << M << ", " << ps.h.l;
  for (uint32_t i = 0; i < ps.h.m - ps.h.l; ++i) s << ", " << int(ps.h.hi[i]);
  s << ">;\n";
  const bool remap = (ps.h.flags & kRemap) != 0;
  if (remap) {
    s << "  using TileOut = JitTileMap<" << M;
    for (int p = 0; p < M; ++p) s << ", " << int(ps.h.out[p]);
    s << ">;\n";
  } else {
    s << "  using TileOut = Tile;\n";
  }
  auto tf = [](bool b) { return b ? "true" : "false"; };
  const bool pipe = js.stages > 0;
  if (pipe)
    s << "  jit_sweep_pipe<" << R << ", " << M << ", Tile, " << tf(js.smem_coef) << ", " << tf(js.work) << ", "
      << tf(js.dstore) << ", " << js.stages
      << ", TileOut>(psi, P, err, [&](const C2 *stage, C2 *tile, const C2 *coef, uint64_t gbase, const PipeCtl<" << R
      << ", " << M << ", Tile, " << js.stages << "> &ctl) {\n";
  else if (js.early) {
    // The first phase's register load, shared by the loop's look-ahead.
    const SweepPhase &p0 = ps.ph[0];
    s << (multi ? "" : "  (void)err;\n") << "  using Ph0 = JitPhase<" << R << ", " << M << ", Tile, "
      << int(p0.reg[0]) << ", " << int(p0.reg[1]) << ", " << int(p0.reg[2]) << ", " << int(p0.reg[3]);
    for (int t : thread_positions(p0, M, c64, true)) s << ", " << t;
    s << ">;\n";
    if (multi)
      s << "  jit_msweep_early<" << R << ", " << M << ", Tile, " << tf(js.dstore) << ">(psi, Q, ";
    else
      s << "  jit_sweep_early<" << R << ", " << M << ", Tile, " << tf(js.smem_coef) << ", " << tf(js.dstore)
        << ", TileOut>(psi, P, ";
    if (from_zero)
      s << "[&](Amps<" << R << "> &A, uint64_t gb) { Ph0::zero_state(A, gb, Ph0::jb(threadIdx.x), " << nm.str()
        << "); }, ";
    else
      s << "[&](Amps<" << R << "> &A, uint64_t gb) { Ph0::load(A, psi, gb, Ph0::jb(threadIdx.x)); }, ";
    s << "[&](const Amps<" << R << "> &A0, C2 *tile, const C2 *coef, uint64_t gbase) {\n";
  } else if (multi)
    s << "  jit_msweep<" << R << ", " << M << ", Tile, " << tf(js.dload) << ", " << tf(js.dstore)
      << ">(psi, Q, [&](C2 *tile, const C2 *coef, uint64_t gbase) {\n";
  else
    s << "  (void)err;\n  jit_sweep<" << R << ", " << M << ", Tile, " << tf(js.smem_coef) << ", " << tf(js.dload)
      << ", " << tf(js.dstore) << ", TileOut>(psi, P, [&](C2 *tile, const C2 *coef, uint64_t gbase) {\n";
  const uint32_t last = ps.h.nphases - 1;
  for (uint32_t p = 0; p < ps.h.nphases; ++p) {
    const SweepPhase &ph = ps.ph[p];
    const bool from_stage = p == 0 && pipe;
    const bool from_hbm = p == 0 && js.dload, to_hbm = p == last && js.dstore;
    s << "    {\n      using Ph = JitPhase<" << R << ", " << M << ", Tile, " << int(ph.reg[0]) << ", "
      << int(ph.reg[1]) << ", " << int(ph.reg[2]) << ", " << int(ph.reg[3]);
    const auto tpos = thread_positions(ph, M, c64, from_hbm || from_stage || to_hbm, kRegBits,
                                       to_hbm && remap && !from_hbm && !from_stage ? ps.h.out : nullptr);
    for (int t : tpos) s << ", " << t;
    s << ">;\n";
    s << "      const uint32_t jb = Ph::jb(threadIdx.x);\n      Amps<" << R << "> A;\n";
    if (from_stage)
      s << "      Ph::gather_lin(A, stage, jb);\n      ctl.release();\n";
    else if (p == 0 && js.early)
      s << "      A = A0;\n";
    else if (from_hbm && from_zero)
      s << "      Ph::zero_state(A, gbase, jb, " << nm.str() << ");\n";
    else if (from_hbm)
      s << "      Ph::load(A, psi, gbase, jb);\n";
    else
      s << "      Ph::gather(A, tile, jb);\n";
    one_state_ops_src(ps.op.data(), ph, R, c64, [&](const SweepOp &o) {
      std::ostringstream c;
      if (multi || lane_indexed(o))
        c << "(coef + " << o.coef << ")";
      else
        c << "ParamCoef<" << R << ", " << o.coef << ">{P.coef}";
      return c.str();
    }, s);
    if (p == last && js.dstore && remap) {
      s << "      using PhO = JitPhase<" << R << ", " << M << ", TileOut, " << int(ph.reg[0]) << ", "
        << int(ph.reg[1]) << ", " << int(ph.reg[2]) << ", " << int(ph.reg[3]);
      for (int t : tpos) s << ", " << t;
      s << ">;\n      PhO::store(A, psi, gbase, jb);\n    }\n";
    } else if (p == last && js.dstore) {
      s << "      Ph::store(A, psi, gbase, jb);\n    }\n";
    } else {
      s << "      Ph::scatter(A, tile, jb);\n      __syncthreads();\n    }\n";
    }
  }
  s << "  });\n}\n";
  return s.str();
}

std::string jit_source(const PlannedSweep &ps, bool c64, int minb, bool multi, bool from_zero) {
  return prelude() + jit_body(ps, c64, minb, multi, from_zero);
}

// Source of the JIT kernel of one reverse (two-state) adjoint sweep; empty
// when the sweep holds an op the generated form does not cover (the generic
// adjoint kernel then runs it).
std::string jit_adjoint_body(const PlannedSweep &ps, bool c64, int minb) {
  const char *R = c64 ? "float" : "double";
  const int M = int(ps.h.m);
  const int NT = 1 << (M - kAdjRegBits);
  std::ostringstream s;
  s << "extern \"C\" __global__ void __launch_bounds__(" << NT << ", " << minb
    << ")\nsq_jit_adjoint(Vec2<" << R << ">::T *__restrict__ psi, Vec2<" << R
    << ">::T *__restrict__ lam, const __grid_constant__ SweepParams<" << R
    << "> P, double2 *__restrict__ partials) {\n";
  s << "  using C2 = Vec2<" << R << ">::T;\n";
  s << "  using Tile = JitTile<" << M << ", " << ps.h.l;
  for (uint32_t i = 0; i < ps.h.m - ps.h.l; ++i) s << ", " << int(ps.h.hi[i]);
  s << ">;\n";
  s << "  jit_adjoint_sweep<" << R << ", " << M
    << ", Tile>(psi, lam, P, partials, [&](C2 *ft, C2 *lt, const C2 *coef, uint64_t gbase, double2 *acc) {\n";
  for (uint32_t p = 0; p < ps.h.nphases; ++p) {
    const SweepPhase &ph = ps.ph[p];
    s << "    {\n      using Ph = JitPhase2<" << R << ", " << M << ", Tile, " << int(ph.reg[0]) << ", "
      << int(ph.reg[1]) << ", " << int(ph.reg[2]);
    for (int t : thread_positions(ph, M, c64, false, kAdjRegBits)) s << ", " << t;
    s << ">;\n";
    s << "      const uint32_t jb = Ph::jb(threadIdx.x);\n      Amps<" << R << ", " << kAdjAmps
      << "> F, G;\n      Ph::gather(F, G, ft, lt, jb);\n";
    // Inner products carry no conditions (as in the generic kernel).
    if (!two_state_ops_src(ps.op.data(), ph, R, c64, NT, s)) return std::string();
    s << "      Ph::scatter(F, G, ft, lt, jb);\n      __syncthreads();\n    }\n";
  }
  s << "  });\n}\n";
  return s.str();
}

// ---------------------------------------------------------------------------
// Batched gradients of circuits that share one plan structure: one kernel
// whose every sweep is straight-line code (coefficients per circuit from its
// packed plan, through shared memory).
// ---------------------------------------------------------------------------
namespace {

std::string tile_type(const SweepHeader &h) {
  std::ostringstream s;
  s << "JitTile<" << h.m << ", " << h.l;
  for (uint32_t i = 0; i < h.m - h.l; ++i) s << ", " << int(h.hi[i]);
  s << ">";
  return s.str();
}

}  // namespace

std::string jit_batch_adjoint_body(const unsigned char *plan, uint32_t nfwd, uint32_t nrev, uint32_t n,
                                   uint32_t M, bool c64) {
  const char *R = c64 ? "float" : "double";
  const int NT = 1 << (int(M) - kAdjRegBits), NT4 = 1 << (int(M) - kRegBits), NW = (NT + 31) / 32;
  // One __noinline__ device function per sweep (the compiler then works on
  // one sweep at a time), called in order by the kernel.
  std::ostringstream fns, calls;
  auto smem_ptrs = [&](std::ostringstream &o) {
    o << "  extern __shared__ __align__(16) unsigned char smem_raw[];\n"
      << "  C2 *bufs = reinterpret_cast<C2 *>(smem_raw);\n"
      << "  C2 *coef = bufs + 4 * (1u << " << M << ");\n"
      << "  double2 *acc = reinterpret_cast<double2 *>(coef + kMaxCoef);\n";
  };
  fns << "using C2 = Vec2<" << R << ">::T;\n";
  size_t off = 0;
  for (uint32_t k = 0; k < nfwd + nrev; ++k) {
    const PackedSweep &ps = *reinterpret_cast<const PackedSweep *>(plan + off);
    const SweepPhase *ph = reinterpret_cast<const SweepPhase *>(plan + off + ps.phase_off);
    const SweepOp *ops = reinterpret_cast<const SweepOp *>(plan + off + ps.op_off);
    const uint32_t *inner = ps.inner_off ? reinterpret_cast<const uint32_t *>(plan + off + ps.inner_off) : nullptr;
    if (ps.h.m != M) return std::string();
    const bool rev = k >= nfwd;
    if (k == nfwd)
      calls << "    sqb_energy(B, C, c, psi, lam);\n";
    fns << "__device__ __noinline__ void sqb_sweep" << k << "(C2 *__restrict__ psi, C2 *__restrict__ lam, "
        << "const unsigned char *rec, double2 *occc) {\n";
    smem_ptrs(fns);
    fns << "  using Tile = " << tile_type(ps.h) << ";\n"
        << "  jit_batch_coef<" << R << ">(coef, rec, " << (off + ps.coef_off) << "u, " << ps.h.ncoef << "u);\n";
    if (rev) fns << "  jit_batch_acc_zero(acc, " << NW << ");\n";
    fns << "  __syncthreads();\n";
    if (!rev)
      fns << "  jit_batch_fwd<" << R << ", " << M << ", Tile>(psi, bufs, " << ps.h.num_tiles
          << "ull, [&](C2 *tile, uint64_t gbase) {\n";
    else
      fns << "  jit_batch_rev<" << R << ", " << M << ", Tile>(psi, lam, bufs, " << ps.h.num_tiles
          << "ull, [&](C2 *ft, C2 *lt, uint64_t gbase) {\n";
    for (uint32_t p = 0; p < ps.h.nphases; ++p) {
      const SweepPhase &P = ph[p];
      if (!rev) {
        fns << "    { using Ph = JitPhase<" << R << ", " << M << ", Tile, " << int(P.reg[0]) << ", "
            << int(P.reg[1]) << ", " << int(P.reg[2]) << ", " << int(P.reg[3]);
        for (int t : thread_positions(P, int(M), c64, false)) fns << ", " << t;
        fns << ">;\n      if (threadIdx.x < " << NT4 << ") {\n"
            << "      const uint32_t jb = Ph::jb(threadIdx.x);\n      Amps<" << R
            << "> A;\n      Ph::gather(A, tile, jb);\n";
        for (uint32_t oi = P.op_begin; oi < P.op_end; ++oi)
          if (ops[oi].kind == kSwInnerDiag || ops[oi].kind == kSwInnerDense) return std::string();
        one_state_ops_src(ops, P, R, c64, [](const SweepOp &o) { return "(coef + " + std::to_string(o.coef) + ")"; },
                          fns);
        fns << "      Ph::scatter(A, tile, jb);\n      }\n      __syncthreads(); }\n";
      } else {
        fns << "    { using Ph = JitPhase2<" << R << ", " << M << ", Tile, " << int(P.reg[0]) << ", "
            << int(P.reg[1]) << ", " << int(P.reg[2]);
        for (int t : thread_positions(P, int(M), c64, false, kAdjRegBits)) fns << ", " << t;
        fns << ">;\n      const uint32_t jb = Ph::jb(threadIdx.x);\n      Amps<" << R << ", " << kAdjAmps
            << "> F, G;\n      Ph::gather(F, G, ft, lt, jb);\n";
        if (!two_state_ops_src(ops, P, R, c64, NT, fns)) return std::string();
        fns << "      Ph::scatter(F, G, ft, lt, jb);\n      __syncthreads(); }\n";
      }
    }
    fns << "  });\n";
    if (rev && inner) {
      fns << "  if (threadIdx.x == 0) {\n";
      for (uint32_t q = 0; q < inner[0]; ++q)
        fns << "    jit_batch_slot_add(acc, " << NW << ", " << q << ", occc + " << inner[1 + q] << "u);\n";
      fns << "  }\n  __syncthreads();\n";
    }
    fns << "}\n";
    calls << "    sqb_sweep" << k << "(psi, lam, rec, occ + C.occ_off);\n";
    off += ps.bytes;
  }
  if (nrev == 0) calls << "    sqb_energy(B, C, c, psi, lam);\n";
  std::ostringstream s;
  s << fns.str();
  s << "__device__ __noinline__ void sqb_energy(const BatchParams &B, const BatchCircuit &C, uint32_t c, "
       "C2 *psi, C2 *lam) {\n"
    << "  double e = batch_pauli_apply<" << R << ">(B.hams[C.ham], " << n
    << ", [&](uint64_t i) { return psi[i]; }, [&](uint64_t i, const C2 &v) { lam[i] = v; });\n"
    << "  e = block_sum(e);\n  if (threadIdx.x == 0) B.energies[c] = e;\n  __syncthreads();\n}\n";
  // sqb_energy is defined after its callers' definitions but before the kernel.
  s << "extern \"C\" __global__ void __launch_bounds__(" << NT << ", 1)\nsq_jit_batch_adjoint(C2 *__restrict__ pool, "
    << "const __grid_constant__ BatchParams B, double2 *__restrict__ occ) {\n"
    << "  __shared__ uint32_t s_next;\n"
    << "  for (;;) {\n"
    << "    if (threadIdx.x == 0) s_next = atomicAdd(B.counter, 1u);\n"
    << "    __syncthreads();\n"
    << "    const uint32_t c = s_next;\n"
    << "    __syncthreads();\n"
    << "    if (c >= B.ncircuits) break;\n"
    << "    const BatchCircuit C = B.circuits[c];\n"
    << "    C2 *psi = pool + C.state_off;\n"
    << "    C2 *lam = pool + C.lam_off;\n"
    << "    const unsigned char *rec = B.plans + C.plan_off;\n"
    << "    jit_batch_init<" << R << ">(psi, " << n << ");\n"
    << "    __syncthreads();\n"
    << calls.str() << "  }\n}\n";
  return s.str();
}

const void *jit_batch_adjoint_kernel(const unsigned char *plan, uint32_t nfwd, uint32_t nrev, uint32_t n,
                                     uint32_t M, bool c64, std::string &err) {
  if (!jit_available()) {
    err = "NVRTC not available";
    return nullptr;
  }
  const std::string body = jit_batch_adjoint_body(plan, nfwd, nrev, n, M, c64);
  if (body.empty()) {
    err = "plan not covered by the JIT batch form";
    return nullptr;
  }
  Entry &e = get_entry(body, "sq_jit_batch_adjoint", batch_prelude());
  if (e.failed) {
    err = e.err;
    return nullptr;
  }
  return reinterpret_cast<const void *>(e.kernel);
}

std::string jit_batch_source(const std::string &body) { return batch_prelude().text + body; }

size_t jit_adjoint_smem(const PlannedSweep &ps, bool c64) {
  return jit_adjoint_smem_bytes(int(ps.h.m), c64 ? 8 : 16, ps.h.ncoef);
}

// Kernel lookup by plan structure.  A generated kernel depends only on the
// sweep's header, phases and ops (and the process-wide tile-loop switches),
// not on its coefficient values, so a structure seen before skips source
// generation and hashing (the host cost of every flush and gradient of a
// repeated circuit).  Two independent 64-bit FNV-1a hashes of the raw bytes
// (the planner zero-fills every padding byte) form the key.
struct PlanKey {
  uint64_t a, b;
  bool operator<(const PlanKey &o) const { return a != o.a ? a < o.a : b < o.b; }
};

PlanKey plan_key(const PlannedSweep &ps, bool c64, int kind) {
  uint64_t a = 1469598103934665603ull, b = 0x9ae16a3b2f90404full;
  auto mix = [&](const void *p, size_t n) {
    const unsigned char *q = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < n; ++i) {
      a = (a ^ q[i]) * 1099511628211ull;
      b = (b ^ q[i]) * 0x100000001b3ull + 0x9e3779b97f4a7c15ull;
    }
  };
  mix(&ps.h, sizeof(ps.h));
  mix(ps.ph.data(), ps.ph.size() * sizeof(SweepPhase));
  mix(ps.op.data(), ps.op.size() * sizeof(SweepOp));
  const uint8_t extra[2] = {uint8_t(c64), uint8_t(kind)};
  mix(extra, sizeof(extra));
  return {a, b};
}

std::mutex g_plan_mu;
std::map<PlanKey, Entry *> g_plan_entries;  // nullptr: not covered by the generated form

// The cached entry for this structure (*found = false when it must be made).
Entry *plan_lookup(const PlanKey &k, bool *found) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto it = g_plan_entries.find(k);
  *found = it != g_plan_entries.end();
  return *found ? it->second : nullptr;
}

void plan_store(const PlanKey &k, Entry *e) {
  std::lock_guard<std::mutex> lk(g_plan_mu);
  g_plan_entries[k] = e;
}

// CTAs per SM of the two-state (reverse) JIT sweeps: complex128 fits 3
// (160-165 registers, 68 KB of shared memory per CTA for 2^10-amplitude
// tiles); complex64 (2^11 tiles, 256 threads) 2.
int jit_adjoint_minb(bool c64) { return c64 ? 2 : 3; }

Entry *adjoint_entry(const PlannedSweep &ps, bool c64) {
  const PlanKey k = plan_key(ps, c64, 1);
  bool found = false;
  Entry *e = plan_lookup(k, &found);
  if (found) return e;
  const std::string body = jit_adjoint_body(ps, c64, jit_adjoint_minb(c64));
  e = body.empty() ? nullptr : &get_entry(body, "sq_jit_adjoint");
  plan_store(k, e);
  return e;
}

Entry &sweep_entry(const PlannedSweep &ps, bool c64) {
  const PlanKey k = plan_key(ps, c64, 0);
  bool found = false;
  Entry *e = plan_lookup(k, &found);
  if (found) return *e;
  e = &get_entry(jit_body(ps, c64, jit_minb(c64, ps.h.m)));
  plan_store(k, e);
  return *e;
}

Entry *msweep_entry(const PlannedSweep &ps, bool c64, bool from_zero) {
  const PlanKey k = plan_key(ps, c64, from_zero ? 3 : 2);
  bool found = false;
  Entry *e = plan_lookup(k, &found);
  if (found) return e;
  const std::string body = jit_body(ps, c64, jit_minb(c64, ps.h.m), true, from_zero);
  e = body.empty() ? nullptr : &get_entry(body, "sq_jit_msweep");
  plan_store(k, e);
  return e;
}

const void *jit_adjoint_kernel(const PlannedSweep &ps, bool c64, std::string &err) {
  Entry *e = adjoint_entry(ps, c64);
  if (!e) {
    err = "sweep not covered by the JIT adjoint form";
    return nullptr;
  }
  if (e->failed) {
    err = e->err;
    return nullptr;
  }
  return reinterpret_cast<const void *>(e->kernel);
}

// Compiles (in parallel) the kernels of structures not seen before.
template <class F>
void prepare_parallel(const std::vector<const PlannedSweep *> &sweeps, F make) {
  std::vector<const PlannedSweep *> todo;
  for (const auto *ps : sweeps) todo.push_back(ps);
  std::atomic<size_t> next{0};
  const unsigned nth = std::max(1u, std::min<unsigned>(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < std::min<size_t>(nth, todo.size()); ++t)
    pool.emplace_back([&] {
      for (size_t i = next++; i < todo.size(); i = next++) make(*todo[i]);
    });
  for (auto &th : pool) th.join();
}

void jit_prepare_adjoint(const std::vector<const PlannedSweep *> &sweeps, bool c64) {
  if (!jit_available() || sweeps.empty()) return;
  std::vector<const PlannedSweep *> todo;
  for (const auto *ps : sweeps) {
    bool found = false;
    plan_lookup(plan_key(*ps, c64, 1), &found);
    if (!found) todo.push_back(ps);
  }
  prepare_parallel(todo, [&](const PlannedSweep &ps) { adjoint_entry(ps, c64); });
}

size_t jit_smem(const PlannedSweep &ps, bool c64) {
  const JitShape js = jit_shape(ps, c64);
  const uint32_t nc = js.smem_coef ? (ps.h.ncoef + 1) & ~1u : 0u;
  if (js.stages > 0) return jit_pipe_smem_bytes(int(ps.h.m), c64 ? 8 : 16, js.stages, js.work, nc);
  return jit_smem_bytes(int(ps.h.m), c64 ? 8 : 16, js.dload || js.early, nc);
}

int jit_minb(bool c64, uint32_t m) {
  // SQ_JIT_MINB overrides the CTAs per SM for every tile size (tuning).
  static const int env = [] {
    const char *e = std::getenv("SQ_JIT_MINB");
    return e && *e ? std::atoi(e) : 0;
  }();
  if (env > 0 && env <= 16) return env;
  // Early loads hold a second register set: one CTA fewer per SM.
  const int e = jit_early() ? 1 : 0;
  // Register budgets of the precompiled sweep instantiations.
  if (c64) return m == 10 ? 8 - 2 * e : m == 12 ? 2 : 1;
  return m == 10 ? 6 - 2 * e : m == 11 ? 3 - e : 1;
}

const void *jit_sweep_kernel(const PlannedSweep &ps, bool c64, std::string &err) {
  Entry &e = sweep_entry(ps, c64);
  if (e.failed) {
    err = e.err;
    return nullptr;
  }
  return reinterpret_cast<const void *>(e.kernel);
}

const void *jit_msweep_kernel(const PlannedSweep &ps, bool c64, std::string &err, bool from_zero) {
  Entry *e = msweep_entry(ps, c64, from_zero);
  if (!e) {
    err = "sweep not covered by the multi-state JIT form";
    return nullptr;
  }
  if (e->failed) {
    err = e->err;
    return nullptr;
  }
  return reinterpret_cast<const void *>(e->kernel);
}

size_t jit_msweep_smem(const PlannedSweep &ps, bool c64) {
  const JitShape js = jit_shape(ps, c64, true);
  return jit_smem_bytes(int(ps.h.m), c64 ? 8 : 16, js.dload || js.early, (ps.h.ncoef + 1) & ~1u);
}

void jit_prepare_multi(const std::vector<const PlannedSweep *> &sweeps, bool c64,
                       const std::vector<const PlannedSweep *> &from_zero) {
  if (!jit_available() || (sweeps.empty() && from_zero.empty())) return;
  std::vector<const PlannedSweep *> todo;
  std::vector<char> zero;
  for (int z = 0; z < 2; ++z)
    for (const auto *ps : z ? from_zero : sweeps) {
      bool found = false;
      plan_lookup(plan_key(*ps, c64, z ? 3 : 2), &found);
      if (!found) {
        todo.push_back(ps);
        zero.push_back(char(z));
      }
    }
  // Index of each task's variant: the tasks are distinct pointers per variant.
  std::vector<std::pair<const PlannedSweep *, bool>> tasks;
  for (size_t i = 0; i < todo.size(); ++i) tasks.emplace_back(todo[i], zero[i] != 0);
  std::atomic<size_t> next{0};
  const unsigned nth = std::max(1u, std::min<unsigned>(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < std::min<size_t>(nth, tasks.size()); ++t)
    pool.emplace_back([&] {
      for (size_t i = next++; i < tasks.size(); i = next++) msweep_entry(*tasks[i].first, c64, tasks[i].second);
    });
  for (auto &th : pool) th.join();
}

void jit_prepare(const std::vector<const PlannedSweep *> &sweeps, bool c64) {
  if (!jit_available() || sweeps.empty()) return;
  std::vector<const PlannedSweep *> todo;
  for (const auto *ps : sweeps) {
    bool found = false;
    plan_lookup(plan_key(*ps, c64, 0), &found);
    if (!found) todo.push_back(ps);
  }
  prepare_parallel(todo, [&](const PlannedSweep &ps) { sweep_entry(ps, c64); });
}

}  // namespace sq

extern "C" int sq_jit_info(int *available, uint64_t *jit_launches, uint64_t *fallbacks) {
  if (available) *available = sq::jit_available() ? 1 : 0;
  if (jit_launches) *jit_launches = sq::g_launches.load();
  if (fallbacks) *fallbacks = sq::g_fallbacks.load();
  return SQ_OK;
}

extern "C" int sq_jit_source(uint32_t num_qubits, int dtype, const sq_circuit_op *ops, uint32_t nops,
                             uint32_t sweep_index, char *buf, uint64_t cap, uint64_t *len,
                             uint32_t *nsweeps) {
  if ((nops && !ops) || !len) return sq_detail_fail(SQ_ERR_INVALID, "null pointer");
  if (dtype != SQ_C128 && dtype != SQ_C64) return sq_detail_fail(SQ_ERR_INVALID, "bad dtype");
  if (num_qubits < uint32_t(sq::kRegBits) || num_qubits > 40)
    return sq_detail_fail(SQ_ERR_INVALID, "num_qubits out of range");
  const bool c64 = dtype == SQ_C64;
  std::vector<sq::PlannedLaunch> plan;
  try {
    sq::AdjointPlan ap;
    sq::build_adjoint(ops, nops, num_qubits, ap);
    sq::PlanOptions opt;
    opt.tile_bits = 0;
    const uint32_t want = std::min<uint32_t>(
        num_qubits, uint32_t(c64 ? sq::kDefaultTileBitsC64 : sq::kDefaultTileBitsC128));
    if (c64) {
      for (int m : sq::kTileBitsC64)
        if (uint32_t(m) <= want) opt.tile_bits = uint32_t(m);
    } else {
      for (int m : sq::kTileBitsC128)
        if (uint32_t(m) <= want) opt.tile_bits = uint32_t(m);
    }
    opt.max_dense_k = c64 ? 4 : 3;
    opt.low_bits = sq::auto_low_bits(c64, num_qubits, opt.tile_bits);
    // As a state of the engine plans with its default options (remapping off
    // unless SQ_REMAP=1).
    const char *re = std::getenv("SQ_REMAP");
    opt.remap = re && re[0] == '1';
    plan = sq::plan_sweeps(ap.forward, num_qubits, opt);
  } catch (const std::exception &e) {
    return sq_detail_fail(SQ_ERR_INVALID, e.what());
  }
  std::vector<const sq::PlannedSweep *> sweeps;
  for (const auto &pl : plan)
    if (pl.is_sweep) sweeps.push_back(&pl.sweep);
  if (nsweeps) *nsweeps = uint32_t(sweeps.size());
  if (sweep_index >= sweeps.size()) return sq_detail_fail(SQ_ERR_INVALID, "no such sweep");
  const sq::PlannedSweep &ps = *sweeps[sweep_index];
  const std::string src = sq::jit_source(ps, c64, sq::jit_minb(c64, ps.h.m));
  *len = src.size();
  if (buf && cap) {
    const size_t n = std::min<size_t>(cap - 1, src.size());
    std::memcpy(buf, src.data(), n);
    buf[n] = '\0';
  }
  return SQ_OK;
}

extern "C" int sq_jit_adjoint_source(uint32_t num_qubits, int dtype, const sq_circuit_op *ops,
                                     uint32_t nops, uint32_t sweep_index, char *buf, uint64_t cap,
                                     uint64_t *len, uint32_t *nsweeps) {
  if ((nops && !ops) || !len) return sq_detail_fail(SQ_ERR_INVALID, "null pointer");
  if (dtype != SQ_C128 && dtype != SQ_C64) return sq_detail_fail(SQ_ERR_INVALID, "bad dtype");
  if (num_qubits < uint32_t(sq::kRegBits) || num_qubits > 40)
    return sq_detail_fail(SQ_ERR_INVALID, "num_qubits out of range");
  const bool c64 = dtype == SQ_C64;
  std::vector<sq::PlannedLaunch> plan;
  try {
    sq::AdjointPlan ap;
    sq::build_adjoint(ops, nops, num_qubits, ap);
    sq::PlanOptions opt;
    opt.tile_bits = 0;
    const auto &tb = c64 ? sq::kAdjTileBitsC64 : sq::kAdjTileBitsC128;
    for (int m : tb)
      if (uint32_t(m) <= num_qubits) opt.tile_bits = uint32_t(m);
    opt.reg_bits = sq::kAdjRegBits;
    opt.max_dense_k = sq::kAdjRegBits;
    plan = sq::plan_sweeps(ap.reverse, num_qubits, opt);
  } catch (const std::exception &e) {
    return sq_detail_fail(SQ_ERR_INVALID, e.what());
  }
  std::vector<const sq::PlannedSweep *> sweeps;
  for (const auto &pl : plan)
    if (pl.is_sweep) sweeps.push_back(&pl.sweep);
  if (nsweeps) *nsweeps = uint32_t(sweeps.size());
  if (sweep_index >= sweeps.size()) return sq_detail_fail(SQ_ERR_INVALID, "no such sweep");
  const std::string body = sq::jit_adjoint_body(*sweeps[sweep_index], c64, sq::jit_adjoint_minb(c64));
  const std::string src = body.empty() ? std::string() : sq::prelude() + body;
  *len = src.size();
  if (buf && cap) {
    const size_t n = std::min<size_t>(cap - 1, src.size());
    std::memcpy(buf, src.data(), n);
    buf[n] = '\0';
  }
  return SQ_OK;
}

extern "C" int sq_jit_compile(const char *source) {
  if (!source) return sq_detail_fail(SQ_ERR_INVALID, "null pointer");
  std::vector<char> cubin;
  std::string err;
  if (!sq::compile(source, cubin, err)) return sq_detail_fail(SQ_ERR_INVALID, err.c_str());
  return SQ_OK;
}

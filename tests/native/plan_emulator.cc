// TEST ONLY: executes the engine's fusion plans on the host, thread by
// thread, with the same index arithmetic as sweep_kernel / gate_kernel
// (snuqs_b200/csrc/sweep_kernels.cuh), so the planner and the gate analysis
// can be checked against the oracle on a machine without a GPU.  It is built
// into tests/native/libplan_emulator.so by tests/native/build.py and is never
// linked into the product.
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "adjoint_plan.h"
#include "host_ops.h"

using namespace sq;

namespace {

uint64_t insert_zero(uint64_t x, uint32_t p) {
  const uint64_t lo = x & ((uint64_t(1) << p) - 1);
  return ((x >> p) << (p + 1)) | lo;
}

// Coefficient index of register slot ri for a (inner) diagonal op.
uint32_t diag_index(const SweepOp &op, uint64_t gbase, uint32_t jb, int ri) {
  uint32_t base = 0;
  for (int t = 0; t < op.ndt; ++t) {
    const uint32_t bit = op.dsrc[t] == kSrcGlobal ? uint32_t(gbase >> op.dpos[t]) & 1u
                                                  : (jb >> op.dpos[t]) & 1u;
    base = (base << 1) | bit;
  }
  const int V = op.vmask;
  int r = 0, b = 0;
  for (int pp = 0; pp < 4; ++pp)
    if (V & (1 << pp)) {
      if (ri & (1 << pp)) r |= 1 << b;
      ++b;
    }
  return (base << __builtin_popcount(V)) | uint32_t(r);
}

// One sweep op on the NA register amplitudes v of one thread (the kernel's
// apply_op).  Inner-product ops are handled by the caller.
void apply_sweep_op(const SweepOp &op, const cplx *c, cplx *v, int NA, uint64_t gbase,
                    uint32_t jb) {
  if ((gbase & op.gmask) != op.gval || (jb & op.lmask) != op.lval) return;
  const int V = op.vmask;
  auto dep = [&](int x) {
    int r = 0, b = 0;
    for (int pp = 0; pp < 4; ++pp)
      if (V & (1 << pp)) {
        if (x & (1 << b)) r |= 1 << pp;
        ++b;
      }
    return r;
  };
  auto groups = [&](auto f) {
    for (int g = 0; g < NA; ++g)
      if (!(g & V) && ((g & op.rmask) == op.rval)) f(g);
  };
  const bool pure = op.aux & kAuxPure;
  switch (op.kind) {
    case kSwPhase:
      for (int ri = 0; ri < NA; ++ri)
        if ((ri & op.rmask) == op.rval) v[ri] = pure ? -v[ri] : c[0] * v[ri];
      break;
    case kSwDiag:
      for (int ri = 0; ri < NA; ++ri) v[ri] = c[diag_index(op, gbase, jb, ri)] * v[ri];
      break;
    case kSwAnti1:
      groups([&](int g) {
        const cplx a0 = v[g], a1 = v[g | V];
        v[g] = pure ? a1 : c[0] * a1;
        v[g | V] = pure ? a0 : c[1] * a0;
      });
      break;
    case kSwSwap2: {
      const int B1 = dep(1), B2 = dep(2);
      groups([&](int g) {
        const cplx a1 = v[g | B1], a2 = v[g | B2];
        v[g | B1] = pure ? a2 : c[0] * a2;
        v[g | B2] = pure ? a1 : c[1] * a1;
      });
    } break;
    case kSwXRot: {
      const int X = op.aux & kAuxXMask, D = 1 << __builtin_popcount(V);
      const cplx f = (op.aux & kAuxImag) ? cplx(0, 1) : cplx(1, 0);
      groups([&](int g) {
        cplx a[16], out[16];
        for (int x = 0; x < D; ++x) a[x] = v[g | dep(x)];
        for (int r = 0; r < D; ++r) out[r] = c[r].real() * a[r] + f * c[r].imag() * a[r ^ X];
        for (int r = 0; r < D; ++r) v[g | dep(r)] = out[r];
      });
    } break;
    default: {
      const int K = __builtin_popcount(V), D = 1 << K;
      groups([&](int g) {
        cplx a[16], out[16];
        for (int x = 0; x < D; ++x) a[x] = v[g | dep(x)];
        for (int r = 0; r < D; ++r) {
          cplx s = c[r * D] * a[0];
          for (int x = 1; x < D; ++x) s += c[r * D + x] * a[x];
          out[r] = s;
        }
        for (int r = 0; r < D; ++r) v[g | dep(r)] = out[r];
      });
    } break;
  }
}

// <lambda| K |phi> over one thread's NA amplitudes (the kernel's inner ops).
cplx inner_sweep_op(const SweepOp &op, const cplx *c, const cplx *phi, const cplx *lam, int NA,
                    uint64_t gbase, uint32_t jb) {
  cplx acc(0, 0);
  const int V = op.vmask;
  if (op.kind == kSwInnerDiag) {
    for (int ri = 0; ri < NA; ++ri) acc += std::conj(lam[ri]) * c[diag_index(op, gbase, jb, ri)] * phi[ri];
    return acc;
  }
  auto dep = [&](int x) {
    int r = 0, b = 0;
    for (int pp = 0; pp < 4; ++pp)
      if (V & (1 << pp)) {
        if (x & (1 << b)) r |= 1 << pp;
        ++b;
      }
    return r;
  };
  const int D = 1 << __builtin_popcount(V);
  for (int g = 0; g < NA; ++g) {
    if (g & V) continue;
    for (int r = 0; r < D; ++r) {
      cplx s(0, 0);
      for (int x = 0; x < D; ++x) s += c[r * D + x] * phi[g | dep(x)];
      acc += std::conj(lam[g | dep(r)]) * s;
    }
  }
  return acc;
}

// Sweeps one state (lam == nullptr) or two states with inner products
// accumulated into ip[global slot] (the adjoint kernel), with NA = 2^reg_bits
// register amplitudes per thread.
void emulate_sweep_n(cplx *psi, cplx *lam, const PlannedSweep &ps, int reg_bits,
                     std::vector<cplx> *ip) {
  const SweepHeader &h = ps.h;
  const int NA = 1 << reg_bits;
  const uint32_t m = h.m, l = h.l, nthr = 1u << (m - reg_bits);
  std::vector<uint64_t> hitab(size_t(1) << (m - l));
  for (uint32_t c = 0; c < hitab.size(); ++c) {
    uint64_t a = 0;
    for (uint32_t i = 0; i < m - l; ++i)
      if ((c >> i) & 1) a |= uint64_t(1) << h.hi[i];
    hitab[c] = a;
  }
  auto addr = [&](uint64_t gbase, uint32_t j) {
    return gbase | hitab[j >> l] | (j & ((1u << l) - 1));
  };
  std::vector<cplx> tile(size_t(1) << m), ltile(size_t(1) << m);
  for (uint64_t t = 0; t < h.num_tiles; ++t) {
    uint64_t gbase = t << l;
    for (uint32_t i = 0; i < m - l; ++i) gbase = insert_zero(gbase, h.hi[i]);
    for (uint32_t j = 0; j < (1u << m); ++j) {
      tile[j] = psi[addr(gbase, j)];
      if (lam) ltile[j] = lam[addr(gbase, j)];
    }
    for (uint32_t p = 0; p < h.nphases; ++p) {
      const SweepPhase &ph = ps.ph[p];
      for (uint32_t tid = 0; tid < nthr; ++tid) {
        uint32_t jb = tid;
        for (int b = 0; b < reg_bits; ++b) jb = uint32_t(insert_zero(jb, ph.reg[b]));
        cplx v[16], w[16];
        uint32_t jj[16];
        for (int ri = 0; ri < NA; ++ri) {
          uint32_t j = jb;
          for (int b = 0; b < reg_bits; ++b)
            if ((ri >> b) & 1) j |= 1u << ph.reg[b];
          jj[ri] = j;
          v[ri] = tile[j];
          if (lam) w[ri] = ltile[j];
        }
        for (uint32_t o = ph.op_begin; o < ph.op_end; ++o) {
          const SweepOp &op = ps.op[o];
          const cplx *c = ps.coef.data() + op.coef;
          if (op.kind == kSwInnerDiag || op.kind == kSwInnerDense) {
            (*ip)[ps.inner_global[op.slot]] += inner_sweep_op(op, c, v, w, NA, gbase, jb);
          } else {
            apply_sweep_op(op, c, v, NA, gbase, jb);
            if (lam) apply_sweep_op(op, c, w, NA, gbase, jb);
          }
        }
        for (int ri = 0; ri < NA; ++ri) {
          tile[jj[ri]] = v[ri];
          if (lam) ltile[jj[ri]] = w[ri];
        }
      }
    }
    // A remapping sweep stores tile position p to global bit out[p].
    auto addr_out = [&](uint32_t j) {
      if (!(h.flags & kRemap)) return addr(gbase, j);
      uint64_t a = gbase;
      for (uint32_t p = 0; p < m; ++p)
        if ((j >> p) & 1) a |= uint64_t(1) << h.out[p];
      return a;
    };
    for (uint32_t j = 0; j < (1u << m); ++j) {
      psi[addr_out(j)] = tile[j];
      if (lam) lam[addr_out(j)] = ltile[j];
    }
  }
}

void emulate_sweep(cplx *psi, const PlannedSweep &ps) { emulate_sweep_n(psi, nullptr, ps, kRegBits, nullptr); }

void emulate_gate(cplx *psi, uint32_t n, const HostOp &op0) {
  HostOp op = op0;
  if (op.kind == kOpDiag) {  // as the engine does: expand to dense
    const size_t D = op.m.size();
    std::vector<cplx> d(D * D, cplx(0, 0));
    for (size_t i = 0; i < D; ++i) d[i * D + i] = op.m[i];
    op.m = d;
  }
  const int k = int(op.tbits.size()), D = 1 << k;
  std::vector<int> sorted(op.tbits);
  std::sort(sorted.begin(), sorted.end());
  std::vector<uint64_t> off(D);
  for (int x = 0; x < D; ++x) {
    uint64_t o = 0;
    for (int j = 0; j < k; ++j)
      if ((x >> (k - 1 - j)) & 1) o |= uint64_t(1) << op.tbits[j];
    off[x] = o;
  }
  std::vector<cplx> a(D);
  for (uint64_t g = 0; g < ((uint64_t(1) << n) >> k); ++g) {
    uint64_t base = g;
    for (int j = 0; j < k; ++j) base = insert_zero(base, sorted[j]);
    if ((base & op.cmask) != op.cval) continue;
    for (int x = 0; x < D; ++x) a[x] = psi[base | off[x]];
    for (int r = 0; r < D; ++r) {
      cplx s = op.m[size_t(r) * D] * a[0];
      for (int x = 1; x < D; ++x) s += op.m[size_t(r) * D + x] * a[x];
      psi[base | off[r]] = s;
    }
  }
}

}  // namespace

extern "C" {

// ops: nops gates; gate i has k[i] targets at qubits[qoff[i]..], nc[i]
// controls at controls[coff[i]..] with values cvals[coff[i]..], and its
// 4^k matrix at mats[moff[i]..] (complex128).  Returns the number of fused
// sweeps (>= 0) or -1 on error.
}  // extern "C"

namespace {

std::vector<HostOp> host_ops(int n, int nops, const int *k, const int *qoff, const int *qubits, const int *nc,
                             const int *coff, const int *controls, const int *cvals, const long *moff,
                             const double *mats) {
  std::vector<HostOp> ops;
  for (int i = 0; i < nops; ++i) {
    std::vector<int> tb;
    for (int j = 0; j < k[i]; ++j) tb.push_back(n - 1 - qubits[qoff[i] + j]);
    uint64_t cm = 0, cv = 0;
    for (int j = 0; j < nc[i]; ++j) {
      const uint64_t bit = uint64_t(1) << (n - 1 - controls[coff[i] + j]);
      cm |= bit;
      if (cvals[coff[i] + j]) cv |= bit;
    }
    const size_t d = size_t(1) << k[i];
    std::vector<cplx> mm(d * d);
    std::memcpy(mm.data(), mats + 2 * moff[i], d * d * sizeof(cplx));
    HostOp h;
    if (analyse_op(mm, tb, cm, cv, h)) ops.push_back(h);
  }
  return ops;
}

PlanOptions emu_options(int tile_bits, int reorder, int low_bits) {
  PlanOptions opt;
  opt.tile_bits = uint32_t(tile_bits);
  opt.reorder = reorder != 0;
  // reorder: 0 off, 1 on (tile selection automatic), 2 on + selection, 3 on, no selection,
  // 4 on + selection + qubit remapping
  opt.select = (reorder == 2 || reorder == 4) ? 1 : reorder == 3 ? 0 : -1;
  opt.remap = reorder == 4;
  opt.low_bits = uint32_t(low_bits);
  return opt;
}

int emulate_plan(double *state, int n, const std::vector<PlannedLaunch> &plan, int *unfused_out) {
  int sweeps = 0, unfused = 0;
  cplx *psi = reinterpret_cast<cplx *>(state);
  for (const auto &pl : plan) {
    if (pl.is_sweep) {
      emulate_sweep(psi, pl.sweep);
      ++sweeps;
    } else {
      emulate_gate(psi, uint32_t(n), pl.gate);
      ++unfused;
    }
  }
  if (unfused_out) *unfused_out = unfused;
  return sweeps;
}

}  // namespace

extern "C" {

// Plans the gates with the matrices mats_a, then re-emits that plan with
// mats_b (same gates, other values) by rebuild_plan and emulates it on
// `state`.  *rebuilt = 1 when the rebuild took (equal op signatures and
// equal sweep structure), else 0 and the gates with mats_b were planned
// anew.  Returns the number of sweeps or -1.
int emu_rebuild(double *state, int n, int nops, const int *k, const int *qoff, const int *qubits, const int *nc,
                const int *coff, const int *controls, const int *cvals, const long *moff, const double *mats_a,
                const double *mats_b, int tile_bits, int reorder, int low_bits, int *rebuilt) {
  try {
    const auto a = host_ops(n, nops, k, qoff, qubits, nc, coff, controls, cvals, moff, mats_a);
    const auto b = host_ops(n, nops, k, qoff, qubits, nc, coff, controls, cvals, moff, mats_b);
    const PlanOptions opt = emu_options(tile_bits, reorder, low_bits);
    auto plan = plan_sweeps(a, uint32_t(n), opt);
    *rebuilt = op_signature(a) == op_signature(b) && rebuild_plan(plan, b, uint32_t(n)) ? 1 : 0;
    if (!*rebuilt) plan = plan_sweeps(b, uint32_t(n), opt);
    return emulate_plan(state, n, plan, nullptr);
  } catch (const std::exception &) {
    return -1;
  }
}

int emu_run(double *state, int n, int nops, const int *k, const int *qoff, const int *qubits,
            const int *nc, const int *coff, const int *controls, const int *cvals,
            const long *moff, const double *mats, int tile_bits, int reorder,
            int low_bits, int *unfused_out) {
  try {
    const auto ops = host_ops(n, nops, k, qoff, qubits, nc, coff, controls, cvals, moff, mats);
    const PlanOptions opt = emu_options(tile_bits, reorder, low_bits);
    auto plan = plan_sweeps(ops, uint32_t(n), opt);
    return emulate_plan(state, n, plan, unfused_out);
  } catch (const std::exception &) {
    return -1;
  }
}

}  // extern "C"

extern "C" {
// Plan statistics for a gate list (same arguments as emu_run): writes
// [sweeps, phases, ops, ops by kind 1..6, unfused] into out[0..9].
int emu_plan_stats(int n, int nops, const int *k, const int *qoff, const int *qubits,
                   const int *nc, const int *coff, const int *controls, const int *cvals,
                   const long *moff, const double *mats, int tile_bits, int reorder,
                   int low_bits, long *out) {
  try {
    std::vector<HostOp> ops;
    for (int i = 0; i < nops; ++i) {
      std::vector<int> tb;
      for (int j = 0; j < k[i]; ++j) tb.push_back(n - 1 - qubits[qoff[i] + j]);
      uint64_t cm = 0, cv = 0;
      for (int j = 0; j < nc[i]; ++j) {
        const uint64_t bit = uint64_t(1) << (n - 1 - controls[coff[i] + j]);
        cm |= bit;
        if (cvals[coff[i] + j]) cv |= bit;
      }
      const size_t d = size_t(1) << k[i];
      std::vector<cplx> mm(d * d);
      std::memcpy(mm.data(), mats + 2 * moff[i], d * d * sizeof(cplx));
      HostOp h;
      if (analyse_op(mm, tb, cm, cv, h)) ops.push_back(h);
    }
    PlanOptions opt;
    opt.tile_bits = uint32_t(tile_bits);
    opt.reorder = reorder != 0;
    // reorder: 0 off, 1 on (tile selection automatic), 2 on + selection, 3 on, no selection,
    // 4 on + selection + qubit remapping
    opt.select = (reorder == 2 || reorder == 4) ? 1 : reorder == 3 ? 0 : -1;
    opt.remap = reorder == 4;
    opt.low_bits = uint32_t(low_bits);
    auto plan = plan_sweeps(ops, uint32_t(n), opt);
    for (int i = 0; i < 12; ++i) out[i] = 0;
    for (const auto &pl : plan) {
      if (!pl.is_sweep) {
        out[9]++;
        continue;
      }
      out[0]++;
      if (pl.sweep.h.flags & kDirectLoad) out[10]++;
      if (pl.sweep.h.flags & kDirectStore) out[11]++;
      out[1] += pl.sweep.h.nphases;
      out[2] += long(pl.sweep.op.size());
      for (const auto &o : pl.sweep.op) out[2 + o.kind]++;
    }
    return 0;
  } catch (const std::exception &) {
    return -1;
  }
}
}

extern "C" {
// Adjoint gradient on the host with the engine's reverse plan (3 register bits,
// two-state sweeps).  Returns the number of reverse sweeps, -1 on error.
int emu_adjoint(int n, const sq_circuit_op *ops, uint32_t nops, const char *paulis,
                const double *weights, uint32_t nterms, uint32_t nparams, int tile_bits,
                int select, double *energy, double *grad) {
  try {
    AdjointPlan ap;
    build_adjoint(ops, nops, uint32_t(n), ap);
    const size_t N = size_t(1) << n;
    std::vector<cplx> psi(N, cplx(0, 0)), lam(N, cplx(0, 0));
    psi[0] = 1.0;
    for (const auto &op : ap.forward) emulate_gate(psi.data(), uint32_t(n), op);
    // lambda = H psi
    for (uint32_t t = 0; t < nterms; ++t) {
      for (size_t i = 0; i < N; ++i) {
        size_t j = i;
        cplx ph(1, 0);
        for (int q = 0; q < n; ++q) {
          const size_t bit = size_t(1) << (n - 1 - q);
          const int b = (i & bit) ? 1 : 0;
          switch (paulis[size_t(t) * n + q]) {
            case 'X': j ^= bit; break;
            case 'Y': j ^= bit; ph *= b ? cplx(0, 1) : cplx(0, -1); break;
            case 'Z': if (b) ph = -ph; break;
            default: break;
          }
        }
        lam[i] += weights[t] * ph * psi[j];
      }
    }
    double e = 0;
    for (size_t i = 0; i < N; ++i) e += (std::conj(psi[i]) * lam[i]).real();
    *energy = e;
    PlanOptions opt;
    opt.tile_bits = uint32_t(tile_bits);
    opt.reg_bits = 3;
    opt.max_dense_k = 3;
    opt.select = select;
    auto plan = plan_sweeps(ap.reverse, uint32_t(n), opt);
    std::vector<cplx> ip(ap.occurrences.size(), cplx(0, 0));
    int sweeps = 0;
    for (const auto &pl : plan) {
      if (pl.is_sweep) {
        emulate_sweep_n(psi.data(), lam.data(), pl.sweep, 3, &ip);
        ++sweeps;
      } else {
        emulate_gate(psi.data(), uint32_t(n), pl.gate);
        emulate_gate(lam.data(), uint32_t(n), pl.gate);
      }
    }
    for (uint32_t p = 0; p < nparams; ++p) grad[p] = 0;
    for (size_t s = 0; s < ip.size(); ++s) {
      const auto &oc = ap.occurrences[s];
      if (oc.first >= 0 && uint32_t(oc.first) < nparams) grad[oc.first] += 2.0 * ip[s].real() * oc.second;
    }
    return sweeps;
  } catch (const std::exception &) {
    return -1;
  }
}
}

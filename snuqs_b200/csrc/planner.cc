// Fusion planner: packs queued gates into fused tile sweeps.
//
// The reference applies every gate as its own full-state kernel
// (src/braket/snuqs/simulation.py:280-284 -> gate_operations_impl_cuda.cu).
// Here a sweep carries as many gates as fit its tile: a gate fits when its
// non-diagonal targets lie in the sweep's tile bit set S (|S| = m, the l
// lowest index bits always included); controls and diagonal gates fit
// anywhere.  With reordering on, a gate that does not fit is skipped and later
// gates that commute with every skipped gate may still join (gates commute
// when neither acts non-diagonally on a bit the other touches).  Inside a
// sweep, gates are cut into phases of at most 4 distinct target bits (the
// register bits).
#include <algorithm>
#include <cassert>
#include <cstring>
#include <stdexcept>

#include "host_ops.h"

namespace sq {

namespace {

int popc64(uint64_t x) { return __builtin_popcountll(x); }

struct SweepBuilder {
  uint32_t n, m, l, max_dense_k = 3, reg_bits = kRegBits, max_ops = kMaxOps;
  uint64_t S;  // tile bits (global index bits)
  std::vector<const HostOp *> ops;
  std::vector<uint64_t> phase_regs;  // register bits (global) of each phase
  std::vector<uint32_t> phase_first; // first op index of each phase
  uint32_t ncoef = 0, ninner = 0;
  // Remap: output global bit of the content of every global bit (size n;
  // empty = the identity).  Only tile bits move.
  std::vector<int> outmap;

  SweepBuilder(uint32_t n_, uint32_t m_, uint32_t l_) : n(n_), m(m_), l(l_) {
    S = (l >= 64) ? ~uint64_t(0) : ((uint64_t(1) << l) - 1);
  }

  static bool is_diag(const HostOp &op) {
    return op.kind == kOpDiag || (op.kind == kOpInner && op.inner_diag);
  }
  static uint32_t coef_count(const HostOp &op) {
    return is_diag(op) ? (1u << op.tbits.size()) : (1u << (2 * op.tbits.size()));
  }

  // Would `op` fit (tile, register, budget)?  If so, add it.
  bool try_add(const HostOp &op) {
    if (ops.size() >= size_t(max_ops)) return false;
    if (ncoef + coef_count(op) > uint32_t(kMaxCoef)) return false;
    if (op.kind == kOpInner && ninner >= uint32_t(kMaxInner)) return false;
    if (is_diag(op)) {
      if (op.tbits.size() > size_t(kMaxDiagK)) return false;
      if (phase_regs.empty()) {
        phase_regs.push_back(0);
        phase_first.push_back(uint32_t(ops.size()));
      }
      ops.push_back(&op);
      ncoef += coef_count(op);
      if (op.kind == kOpInner) ++ninner;
      return true;
    }
    const uint32_t kmax = op.kind == kOpInner ? reg_bits : max_dense_k;
    if (op.tbits.size() > size_t(kmax)) return false;
    const uint64_t T = op.target_mask();
    if (uint32_t(popc64(S | T)) > m) return false;
    const bool new_phase = phase_regs.empty() || popc64(phase_regs.back() | T) > int(reg_bits);
    if (new_phase && phase_regs.size() >= size_t(kMaxPhases)) return false;
    S |= T;
    if (new_phase) {
      phase_regs.push_back(T);
      phase_first.push_back(uint32_t(ops.size()));
    } else {
      phase_regs.back() |= T;
    }
    ops.push_back(&op);
    ncoef += coef_count(op);
    if (op.kind == kOpInner) ++ninner;
    return true;
  }

  PlannedSweep finish() const;
};

// Position of global bit b within the ascending bit list of mask.
int rank_in(uint64_t mask, int b) { return popc64(mask & ((uint64_t(1) << b) - 1)); }

// Pauli form of an inner-product op's K (canonical local order): K = alpha P
// with P_(r, r^x) = (-1)^popc(r & z) times K's row-0 entry in column x and
// every other entry zero, each to within 1e-14 |alpha| (rotation generators
// computed as dU/da U^dagger carry rounding of that size).  d: dimension;
// diag: K holds only the d diagonal entries.
bool pauli_form(const cplx *K, int d, bool diag, uint32_t &x, uint32_t &z) {
  x = 0;
  if (!diag)
    for (int c = 1; c < d; ++c)
      if (std::abs(K[c]) > std::abs(K[x])) x = uint32_t(c);
  const cplx a = diag ? K[0] : K[x];
  const double tol = 1e-14 * std::abs(a);
  if (std::abs(a) == 0.0) return false;
  auto at = [&](int r, int c) { return diag ? (r == c ? K[r] : cplx(0, 0)) : K[size_t(r) * d + c]; };
  z = 0;
  for (int j = 0; (1 << j) < d; ++j)
    if (std::abs(at(1 << j, (1 << j) ^ int(x)) + a) <= tol) z |= 1u << j;
  for (int r = 0; r < d; ++r)
    for (int c = 0; c < d; ++c) {
      const cplx want = c == (r ^ int(x)) ? ((__builtin_popcount(uint32_t(r) & z) & 1) ? -a : a) : cplx(0, 0);
      if (std::abs(at(r, c) - want) > tol) return false;
    }
  return true;
}

// Picks the cheapest sweep-op kind for a dense k-qubit matrix in canonical
// order and appends its coefficients.
void encode_dense(SweepOp &so, const std::vector<cplx> &cm, int k, std::vector<cplx> &coef) {
  const int d = 1 << k;
  auto M = [&](int r, int c) { return cm[size_t(r) * d + c]; };
  const cplx zero(0, 0), one(1, 0);
  if (k == 1 && M(0, 0) == zero && M(1, 1) == zero) {
    so.kind = kSwAnti1;
    if (M(0, 1) == one && M(1, 0) == one) so.aux |= kAuxPure;
    coef.push_back(M(0, 1));
    coef.push_back(M(1, 0));
    return;
  }
  if (k == 2) {
    bool swap2 = M(0, 0) == one && M(3, 3) == one && M(1, 2) != zero && M(2, 1) != zero;
    for (int r = 0; r < 4 && swap2; ++r)
      for (int c = 0; c < 4; ++c) {
        const bool keep = (r == c && (r == 0 || r == 3)) || (r == 1 && c == 2) || (r == 2 && c == 1);
        if (!keep && M(r, c) != zero) swap2 = false;
      }
    if (swap2) {
      so.kind = kSwSwap2;
      if (M(1, 2) == one && M(2, 1) == one) so.aux |= kAuxPure;
      coef.push_back(M(1, 2));
      coef.push_back(M(2, 1));
      return;
    }
  }
  if (k <= 2) {
    // c_r a_r + f s_r a_(r^x): real diagonal, one partner column per row, all
    // partner entries real or all imaginary.
    int x = 0;
    bool ok = true;
    for (int r = 0; r < d && ok; ++r) {
      if (M(r, r).imag() != 0) ok = false;
      for (int c = 0; c < d && ok; ++c)
        if (c != r && M(r, c) != zero) {
          if (x == 0) x = r ^ c;
          else if ((r ^ c) != x) ok = false;
        }
    }
    if (ok && x != 0) {
      bool all_re = true, all_im = true;
      for (int r = 0; r < d; ++r) {
        const cplx v = M(r, r ^ x);
        if (v.imag() != 0) all_re = false;
        if (v.real() != 0) all_im = false;
      }
      if (all_re || all_im) {
        so.kind = kSwXRot;
        so.aux |= uint8_t(x);
        if (!all_re) so.aux |= kAuxImag;
        for (int r = 0; r < d; ++r) {
          const cplx v = M(r, r ^ x);
          coef.push_back(cplx(M(r, r).real(), all_re ? v.real() : v.imag()));
        }
        return;
      }
    }
  }
  so.kind = kSwDense;
  coef.insert(coef.end(), cm.begin(), cm.end());
}

PlannedSweep SweepBuilder::finish() const {
  PlannedSweep ps;
  // Pad the tile to exactly m bits with the lowest unused bits.
  uint64_t tile = S;
  for (uint32_t b = 0; b < n && uint32_t(popc64(tile)) < m; ++b) tile |= uint64_t(1) << b;
  SweepHeader &h = ps.h;
  std::memset(&h, 0, sizeof(h));
  h.n = n;
  h.m = m;
  h.l = l;
  h.num_tiles = uint64_t(1) << (n - m);
  {
    int i = 0;
    for (uint32_t b = l; b < n; ++b)
      if ((tile >> b) & 1) h.hi[i++] = uint8_t(b);
  }
  // Phases: register bits as tile positions, padded from the top of the tile
  // so lanes keep the low positions (coalesced global access, no bank
  // conflicts).
  const int np = int(phase_regs.size());
  for (int p = 0; p < np; ++p) {
    uint32_t regpos = 0;  // bitmask of tile positions
    for (int b = 0; b < 64; ++b)
      if ((phase_regs[p] >> b) & 1) regpos |= 1u << rank_in(tile, b);
    for (int pos = int(m) - 1; pos >= 0 && __builtin_popcount(regpos) < int(reg_bits); --pos)
      regpos |= 1u << pos;
    SweepPhase ph{};
    int r = 0;
    for (uint32_t pos = 0; pos < m; ++pos)
      if ((regpos >> pos) & 1) ph.reg[r++] = uint8_t(pos);
    ph.op_begin = uint16_t(phase_first[p]);
    ph.op_end = uint16_t(p + 1 < np ? phase_first[p + 1] : ops.size());
    ps.ph.push_back(ph);
  }
  h.nphases = uint32_t(np);
  const uint32_t lowpos = (1u << std::min<uint32_t>(l, 5)) - 1;
  // Positions stored to the low global bits (where a direct store needs the
  // lanes): the low positions themselves, or their images under the remap.
  uint32_t lowpos_out = lowpos;
  if (!outmap.empty()) {
    h.flags |= kRemap;
    lowpos_out = 0;
    for (uint32_t p = 0; p < m; ++p) {
      const int in = p < l ? int(p) : int(h.hi[p - l]);
      h.out[p] = uint8_t(outmap[size_t(in)]);
      if (h.out[p] < std::min<uint32_t>(l, 5)) lowpos_out |= 1u << p;
    }
  }
  auto regmask = [&](const SweepPhase &ph) {
    uint32_t x = 0;
    for (uint32_t b = 0; b < reg_bits; ++b) x |= 1u << ph.reg[b];
    return x;
  };
  if ((regmask(ps.ph.front()) & lowpos) == 0) h.flags |= kDirectLoad;
  if ((regmask(ps.ph.back()) & lowpos_out) == 0) h.flags |= kDirectStore;

  // Ops.
  for (int p = 0; p < np; ++p) {
    const SweepPhase &ph = ps.ph[p];
    auto regof = [&](int gbit) -> int {  // register position of a global bit, or -1
      if (!((tile >> gbit) & 1)) return -1;
      const int pos = rank_in(tile, gbit);
      for (uint32_t r = 0; r < reg_bits; ++r)
        if (ph.reg[r] == pos) return int(r);
      return -1;
    };
    // Route a condition bit (global bit b must equal v) to the register,
    // tile-local or global masks.
    auto add_cond = [&](SweepOp &so, int b, uint64_t v) {
      const int r = regof(b);
      if (r >= 0) {
        so.rmask |= uint8_t(1u << r);
        if (v) so.rval |= uint8_t(1u << r);
      } else if ((tile >> b) & 1) {
        const int pos = rank_in(tile, b);
        so.lmask |= 1u << pos;
        if (v) so.lval |= 1u << pos;
      } else {
        so.gmask |= uint64_t(1) << b;
        if (v) so.gval |= uint64_t(1) << b;
      }
    };
    for (uint32_t oi = ph.op_begin; oi < ph.op_end; ++oi) {
      const HostOp &op = *ops[oi];
      SweepOp so;
      std::memset(&so, 0, sizeof(so));
      so.k = uint8_t(op.tbits.size());
      so.coef = uint32_t(ps.coef.size());
      const int k = int(op.tbits.size());
      if (is_diag(op)) {
        int nonone = 0, e = -1;
        for (size_t x = 0; x < op.m.size(); ++x)
          if (op.m[x] != cplx(1, 0)) ++nonone, e = int(x);
        if (op.kind == kOpDiag && nonone == 1) {
          so.kind = kSwPhase;
          for (int t = 0; t < k; ++t) add_cond(so, op.tbits[t], (e >> (k - 1 - t)) & 1);
          if (op.m[e] == cplx(-1, 0)) so.aux |= kAuxPure;
          ps.coef.push_back(op.m[e]);
        } else {
          so.kind = op.kind == kOpInner ? kSwInnerDiag : kSwDiag;
          if (op.kind == kOpInner) {
            so.slot = uint32_t(ps.inner_global.size());
            ps.inner_global.push_back(op.slot);
          }
          // Register targets -> canonical low index bits; the rest -> high
          // bits, most significant first.
          uint32_t vmask = 0;
          for (int t = 0; t < k; ++t) {
            const int r = regof(op.tbits[t]);
            if (r >= 0) vmask |= 1u << r;
          }
          const int nreg = __builtin_popcount(vmask);
          int newbit[kMaxDiagK];
          int nd = 0;
          for (int t = 0; t < k; ++t) {
            const int b = op.tbits[t];
            const int r = regof(b);
            if (r >= 0) {
              newbit[t] = __builtin_popcount(vmask & ((1u << r) - 1));
            } else {
              so.dsrc[nd] = ((tile >> b) & 1) ? kSrcLocal : kSrcGlobal;
              so.dpos[nd] = uint8_t(((tile >> b) & 1) ? rank_in(tile, b) : b);
              newbit[t] = -1 - nd;  // placeholder: fixed below
              ++nd;
            }
          }
          for (int t = 0; t < k; ++t)
            if (newbit[t] < 0) newbit[t] = nreg + (nd - 1 - (-1 - newbit[t]));
          so.ndt = uint8_t(nd);
          so.vmask = uint8_t(vmask);
          std::vector<cplx> cd(op.m.size());
          for (size_t x = 0; x < op.m.size(); ++x) {
            size_t y = 0;
            for (int t = 0; t < k; ++t)
              if ((x >> (k - 1 - t)) & 1) y |= size_t(1) << newbit[t];
            cd[y] = op.m[x];
          }
          uint32_t px = 0, pz = 0;
          if (op.kind == kOpInner && k <= 3 && pauli_form(cd.data(), int(cd.size()), true, px, pz))
            so.aux = uint8_t(kAuxPauli | pz);
          ps.coef.insert(ps.coef.end(), cd.begin(), cd.end());
        }
      } else {
        // Target j (matrix bit k-1-j) sits at register position rp[j]; the
        // kernel's canonical order has matrix bit i <-> i-th set bit of vmask.
        int rp[kRegBits];
        uint32_t vmask = 0;
        for (int j = 0; j < k; ++j) {
          rp[j] = regof(op.tbits[j]);
          assert(rp[j] >= 0);
          vmask |= 1u << rp[j];
        }
        so.vmask = uint8_t(vmask);
        int newbit[kRegBits];  // old matrix bit (k-1-j) -> canonical bit
        for (int j = 0; j < k; ++j) newbit[k - 1 - j] = __builtin_popcount(vmask & ((1u << rp[j]) - 1));
        const int d = 1 << k;
        std::vector<cplx> cm(size_t(d) * d);
        auto remap = [&](int x) {
          int y = 0;
          for (int b = 0; b < k; ++b)
            if ((x >> b) & 1) y |= 1 << newbit[b];
          return y;
        };
        for (int r = 0; r < d; ++r)
          for (int c = 0; c < d; ++c) cm[size_t(remap(r)) * d + remap(c)] = op.m[size_t(r) * d + c];
        for (int b = 0; b < 64; ++b)
          if ((op.cmask >> b) & 1) add_cond(so, b, (op.cval >> b) & 1);
        if (op.kind == kOpInner) {
          so.kind = kSwInnerDense;
          so.slot = uint32_t(ps.inner_global.size());
          ps.inner_global.push_back(op.slot);
          uint32_t px = 0, pz = 0;
          if (k <= 3 && pauli_form(cm.data(), d, false, px, pz)) so.aux = uint8_t(kAuxPauli | px | (pz << 3));
          ps.coef.insert(ps.coef.end(), cm.begin(), cm.end());
        } else {
          encode_dense(so, cm, k, ps.coef);
        }
      }
      so.code = uint8_t(sq_op_code(so.kind, so.vmask, so.aux));
      ps.op.push_back(so);
    }
  }
  h.ncoef = uint32_t(ps.coef.size());
  ps.ngates = uint32_t(ops.size());
  return ps;
}

// ---------------------------------------------------------------------------
// Tile selection and phase scheduling.
// ---------------------------------------------------------------------------
bool fusable_size(const HostOp &op, const PlanOptions &opt) {
  if (SweepBuilder::is_diag(op)) return op.tbits.size() <= size_t(kMaxDiagK);
  const uint32_t kmax = op.kind == kOpInner ? opt.reg_bits : std::min(opt.max_dense_k, opt.reg_bits);
  return op.tbits.size() <= size_t(kmax);
}

// Op budget of one sweep: opt.max_ops, capped by what SweepParams holds.
uint32_t op_budget(const PlanOptions &opt) {
  return opt.max_ops ? std::min<uint32_t>(opt.max_ops, kMaxOps) : uint32_t(kMaxOps);
}

// Per-op facts the tile selection reads many times (masks, coefficient
// count, fusability), computed once per op of the planner's working copy
// and looked up by address (every op pointer the planner holds points into
// that copy).
struct OpInfo {
  uint64_t T, A, tm;  // non-diagonal, touched and target bits
  uint32_t coef;
  bool diag, fits, inner;
};

struct OpTable {
  const HostOp *base = nullptr;
  std::vector<OpInfo> v;
  const OpInfo &operator()(const HostOp *p) const { return v[size_t(p - base)]; }
  void set(const HostOp &op, const PlanOptions &opt) {
    OpInfo &f = v[size_t(&op - base)];
    f.T = op.nondiag_mask();
    f.A = op.touched_mask();
    f.tm = op.target_mask();
    f.coef = SweepBuilder::coef_count(op);
    f.diag = SweepBuilder::is_diag(op);
    f.fits = fusable_size(op, opt);
    f.inner = op.kind == kOpInner;
  }
};

// Gates from rem[head..] that a sweep with tile bits S takes (same rules as
// the collection below, without growing S).
uint32_t absorbed(const std::vector<const HostOp *> &rem, size_t head, uint64_t S, uint32_t n,
                  const PlanOptions &opt, size_t window, const OpTable &tab) {
  uint32_t cnt = 0, ncoef = 0, ninner = 0;
  const uint32_t max_ops = op_budget(opt);
  uint64_t blockT = 0, blockA = 0;
  size_t skipped = 0;
  for (size_t i = head; i < rem.size(); ++i) {
    const OpInfo &f = tab(rem[i]);
    const uint64_t T = f.T, A = f.A;
    const bool commutes = (T & blockA) == 0 && (A & blockT) == 0;
    const bool diag = f.diag;
    const uint32_t c = f.coef;
    const bool fits = f.fits && (diag || (f.tm & ~S) == 0) && cnt < max_ops &&
                      ncoef + c <= uint32_t(kMaxCoef) && !(f.inner && ninner >= uint32_t(kMaxInner));
    if (commutes && fits) {
      ++cnt;
      ncoef += c;
      if (f.inner) ++ninner;
      if (cnt >= max_ops) break;
      continue;
    }
    blockT |= T;
    blockA |= A;
    if (++skipped >= window || popc64(blockT) >= int(n)) break;
  }
  return cnt;
}

// Tile bits (the l low bits plus up to m - l more) that maximise the gates
// the sweep absorbs: grown one bit, or one pair of a two-target gate's
// bits, at a time by the best gain per added bit.
uint64_t select_tile(const std::vector<const HostOp *> &rem, size_t head, uint32_t n, uint32_t m,
                     uint64_t start, const PlanOptions &opt, size_t window, const OpTable &tab) {
  uint64_t S = start;
  uint32_t cur = absorbed(rem, head, S, n, opt, window, tab);
  while (uint32_t(popc64(S)) < m) {
    // Candidate bits: targets of the next gates outside S.
    uint64_t cand = 0;
    std::vector<uint64_t> pairs;
    for (size_t i = head, seen = 0; i < rem.size() && seen < 2 * window; ++i, ++seen) {
      const OpInfo &f = tab(rem[i]);
      if (f.diag || !f.fits) continue;
      const uint64_t out = f.tm & ~S;
      cand |= out;
      if (popc64(out) == 2 && std::find(pairs.begin(), pairs.end(), out) == pairs.end() &&
          pairs.size() < 48)
        pairs.push_back(out);
    }
    if (!cand) break;
    double best = 0.0;
    uint64_t best_add = 0;
    for (uint32_t b = 0; b < n; ++b) {
      if (!((cand >> b) & 1)) continue;
      const uint64_t add = uint64_t(1) << b;
      const double g = double(absorbed(rem, head, S | add, n, opt, window, tab)) - cur;
      if (g > best) best = g, best_add = add;
    }
    if (uint32_t(popc64(S)) + 2 <= m)
      for (uint64_t pr : pairs) {
        const double g = (double(absorbed(rem, head, S | pr, n, opt, window, tab)) - cur) / 2.0;
        if (g > best) best = g, best_add = pr;
      }
    if (!best_add) break;
    S |= best_add;
    cur = absorbed(rem, head, S, n, opt, window, tab);
  }
  return S;
}

// Orders the ops of one sweep (circuit order, at most 64) into phases: a
// phase opens with the ready op that adds the fewest new register bits and
// takes every ready op that fits its register set (diagonal ops fit any
// phase).  Op j depends on an earlier op i when they do not commute.
// Returns the new order and the first index of each phase.
// `low`: the tile's lowest bits; `low_out`: the bits stored to the lowest
// bits (the same unless the sweep remaps).  A first phase whose register set
// avoids `low` can load from HBM straight into registers, and a last phase
// that avoids `low_out` can store straight back (the lanes then cover
// contiguous amplitudes), so the first phase prefers ops off `low` and
// later phases take the ops on `low_out` as early as they can.
void schedule_phases(const std::vector<const HostOp *> &ops, uint32_t reg_bits, uint64_t low,
                     uint64_t low_out, std::vector<const HostOp *> &order,
                     std::vector<uint64_t> &phase_regs, std::vector<uint32_t> &phase_first) {
  const size_t N = ops.size();
  std::vector<uint64_t> pred(N, 0), Tm(N), Am(N), tgt(N);
  std::vector<char> dg(N);
  for (size_t j = 0; j < N; ++j) {
    Tm[j] = ops[j]->nondiag_mask();
    Am[j] = ops[j]->touched_mask();
    tgt[j] = ops[j]->target_mask();
    dg[j] = SweepBuilder::is_diag(*ops[j]);
  }
  for (size_t j = 0; j < N; ++j)
    for (size_t i = 0; i < j; ++i)
      if ((Tm[i] & Am[j]) || (Am[i] & Tm[j])) pred[j] |= uint64_t(1) << i;
  const uint64_t all = N == 64 ? ~uint64_t(0) : ((uint64_t(1) << N) - 1);
  uint64_t placed = 0;
  order.clear();
  phase_regs.clear();
  phase_first.clear();
  while (placed != all) {
    uint64_t R = 0;
    phase_first.push_back(uint32_t(order.size()));
    for (;;) {
      bool progress = false;
      for (size_t x = 0; x < N; ++x) {
        const uint64_t bit = uint64_t(1) << x;
        if ((placed & bit) || (pred[x] & ~placed)) continue;
        const bool fits = dg[x] || (tgt[x] & ~R) == 0;
        if (!fits) continue;
        placed |= bit;
        order.push_back(ops[x]);
        progress = true;
      }
      if (progress) continue;
      // Open the register set to the ready op that adds the fewest bits
      // (low-bit ops last in the first phase, first in the others).
      const bool first_phase = phase_first.size() == 1;
      int best = -1, best_key = 1 << 20;
      for (size_t x = 0; x < N; ++x) {
        const uint64_t bit = uint64_t(1) << x;
        if ((placed & bit) || (pred[x] & ~placed)) continue;
        const uint64_t T = tgt[x];
        if (popc64(R | T) > int(reg_bits)) continue;
        const bool on_low = (T & (first_phase ? low : low_out)) != 0;
        const int key = (on_low == first_phase ? 16 : 0) + popc64(T & ~R);
        if (key < best_key) best_key = key, best = int(x);
      }
      if (best < 0) break;
      R |= tgt[size_t(best)];
    }
    phase_regs.push_back(R);
  }
}

// Moves op `op` through a bit permutation: the content of global bit b is
// now at bit perm[b].
void relabel(HostOp &op, const std::vector<int> &perm) {
  for (int &b : op.tbits) b = perm[size_t(b)];
  uint64_t cm = 0, cv = 0;
  for (size_t b = 0; b < perm.size(); ++b) {
    if ((op.cmask >> b) & 1) cm |= uint64_t(1) << perm[b];
    if ((op.cval >> b) & 1) cv |= uint64_t(1) << perm[b];
  }
  op.cmask = cm;
  op.cval = cv;
}

// The remap of one sweep with tile bits S, given the ops that follow it: a
// permutation of the tile's bits applied on the way out.  Low bits the next
// sweep would not choose get tile bits it would (earliest used first); every
// other bit away from home (virt_at[p] != p) goes home when its home is in
// the tile and free; the rest stay or fill the remaining places.  The bits
// away from home must still fit one tile with the low bits, so that one
// permutation sweep can always restore the order.  With no ops left, only
// homing happens.  Returns the output map (content of bit b goes to bit
// out[b]; empty: store in place) and the bits stored to the low bits.
std::vector<int> choose_remap(const std::vector<const HostOp *> &after, uint64_t S,
                              const std::vector<int> &virt_at, uint32_t n, uint32_t m, uint32_t l,
                              const PlanOptions &opt, size_t window, uint64_t &low_out,
                              const OpTable &tab) {
  const uint64_t low = (uint64_t(1) << l) - 1;
  S |= low;
  std::vector<std::pair<int, int>> swaps;  // (low slot, tile bit moved there)
  if (!after.empty()) {
    const uint64_t wish = select_tile(after, 0, n, m, 0, opt, window, tab);
    uint64_t slots = low & ~wish;
    std::vector<std::pair<size_t, int>> cands;  // (first use, bit)
    for (uint32_t b = l; b < n; ++b) {
      if (!((wish >> b) & 1) || !((S >> b) & 1)) continue;
      size_t first = after.size();
      for (size_t i = 0; i < after.size() && i < window; ++i)
        if ((tab(after[i]).tm >> b) & 1) {
          first = i;
          break;
        }
      cands.emplace_back(first, int(b));
    }
    std::sort(cands.begin(), cands.end());
    for (const auto &cb : cands) {
      if (!slots) break;
      swaps.emplace_back(__builtin_ctzll(slots), cb.second);
      slots &= slots - 1;
    }
  }
  // Builds the permutation for the first `k` swaps; returns the bits away
  // from home afterwards.
  std::vector<int> out;
  auto build = [&](size_t k) {
    out.assign(n, -1);
    uint64_t taken = 0;
    for (size_t i = 0; i < k; ++i) {
      out[size_t(swaps[i].second)] = swaps[i].first;
      taken |= uint64_t(1) << swaps[i].first;
    }
    // Homing.
    for (uint32_t p = 0; p < n; ++p) {
      if (!((S >> p) & 1) || out[p] >= 0) continue;
      const int v = virt_at[p];
      if (v != int(p) && ((S >> v) & 1) && !((taken >> v) & 1)) {
        out[p] = v;
        taken |= uint64_t(1) << v;
      }
    }
    // The rest: in place when free, else any free place in the tile.
    std::vector<int> free_pos;
    for (uint32_t p = 0; p < n; ++p) {
      if (!((S >> p) & 1) || out[p] >= 0) continue;
      if (!((taken >> p) & 1)) {
        out[p] = int(p);
        taken |= uint64_t(1) << p;
      }
    }
    for (uint32_t p = 0; p < n; ++p)
      if (((S >> p) & 1) && !((taken >> p) & 1)) free_pos.push_back(int(p));
    size_t f = 0;
    for (uint32_t p = 0; p < n; ++p) {
      if (!((S >> p) & 1)) out[p] = int(p);
      else if (out[p] < 0) out[p] = free_pos[f++];
    }
    uint64_t moved = 0;
    for (uint32_t p = 0; p < n; ++p) {
      // After the store, bit out[p] holds virtual bit virt_at[p].
      if (virt_at[p] != out[p]) moved |= uint64_t(1) << out[p];
    }
    return moved;
  };
  size_t k = swaps.size();
  uint64_t moved = build(k);
  while (k > 0 && uint32_t(popc64(moved | low)) > m) moved = build(--k);
  bool identity = true;
  for (uint32_t p = 0; p < n; ++p) identity = identity && out[p] == int(p);
  low_out = 0;
  for (uint32_t p = 0; p < n; ++p)
    if (out[p] < int(l)) low_out |= uint64_t(1) << p;
  if (identity) {
    low_out = low;
    return {};
  }
  return out;
}

}  // namespace

std::vector<PlannedLaunch> plan_sweeps(const std::vector<HostOp> &ops, uint32_t n,
                                       const PlanOptions &opt) {
  std::vector<PlannedLaunch> out;
  if (n < uint32_t(kRegBits)) throw std::invalid_argument("fused sweeps need n >= 4");
  // The tile size is the compiled kernel's (opt.tile_bits <= n); the low
  // contiguous bits leave at least one full register set free.
  const uint32_t m = std::min<uint32_t>(opt.tile_bits, n);
  if (m < uint32_t(kRegBits) || m > uint32_t(kMaxTileBits))
    throw std::invalid_argument("tile bits out of range");
  const uint32_t l = opt.low_bits ? opt.low_bits : uint32_t(sweep_low_bits(int(m)));
  if (l + opt.reg_bits > m) throw std::invalid_argument("low bits leave no register set free");
  const size_t kWindow = 256;  // lookahead when reordering
  const bool select =
      opt.reorder && (opt.select == 1 || (opt.select < 0 && n >= kSelectMinQubits && n > m));

  // The ops in the current bit order (a remapping sweep moves the bits of
  // every op after it); virt_at[p]: the original bit whose content is at p.
  std::vector<HostOp> work(ops);
  std::vector<int> virt_at(n);
  for (uint32_t b = 0; b < n; ++b) virt_at[b] = int(b);
  const bool remap = opt.remap && select;
  std::vector<const HostOp *> rem;
  for (const auto &o : work) rem.push_back(&o);
  OpTable tab;
  tab.base = work.data();
  tab.v.resize(work.size());
  for (const auto &o : work) tab.set(o, opt);
  // Recipe of a finished sweep (none when the plan remaps: its later ops are
  // relabelled copies).
  auto recipe = [&](const SweepBuilder &sb) {
    SweepRecipe r;
    if (remap) return r;
    r.S = sb.S;
    r.phase_regs = sb.phase_regs;
    r.phase_first = sb.phase_first;
    r.reg_bits = sb.reg_bits;
    r.max_dense_k = sb.max_dense_k;
    for (const HostOp *op : sb.ops) r.src.push_back(uint32_t(op - work.data()));
    return r;
  };
  size_t head = 0;  // rem[head..] still to place
  while (head < rem.size()) {
    const HostOp &first = *rem[head];
    const bool first_fusable =
        !(first.kind == kOpDense &&
          first.tbits.size() > size_t(std::min<uint32_t>(opt.max_dense_k, opt.reg_bits))) &&
        !(first.kind == kOpDiag && first.tbits.size() > size_t(kMaxDiagK));
    if (!first_fusable && first.kind == kOpInner)
      throw std::logic_error("planner: inner-product op too wide for a sweep");
    if (!first_fusable) {
      PlannedLaunch pl;
      pl.is_sweep = false;
      pl.gate = first;
      pl.gate_src = uint32_t(&first - work.data());
      out.push_back(std::move(pl));
      ++head;
      continue;
    }
    SweepBuilder sb(n, m, l);
    sb.max_ops = op_budget(opt);
    sb.reg_bits = opt.reg_bits;
    sb.max_dense_k = std::min<uint32_t>(opt.max_dense_k, opt.reg_bits);
    if (select) {
      // Tile bits chosen up front; gates that fit them (or grow them while
      // there is room) are collected in circuit order, then scheduled.
      uint64_t S = select_tile(rem, head, n, m, (uint64_t(1) << l) - 1, opt, kWindow, tab);
      if (absorbed(rem, head, S, n, opt, kWindow, tab) == 0) S = ((uint64_t(1) << l) - 1) | first.target_mask();
      std::vector<const HostOp *> chosen;
      std::vector<size_t> chosen_idx, skipped_idx;
      uint64_t blockT = 0, blockAll = 0;
      uint32_t ncoef = 0, ninner = 0;
      size_t i = head;
      for (; i < rem.size(); ++i) {
        const HostOp &op = *rem[i];
        const OpInfo &f = tab(&op);
        const uint64_t T = f.T, A = f.A;
        const bool commutes = (T & blockAll) == 0 && (A & blockT) == 0;
        const bool diag = f.diag;
        const uint32_t c = f.coef;
        const bool fits = f.fits && (diag || uint32_t(popc64(S | f.tm)) <= m) &&
                          chosen.size() < size_t(sb.max_ops) && ncoef + c <= uint32_t(kMaxCoef) &&
                          !(f.inner && ninner >= uint32_t(kMaxInner));
        if (commutes && fits) {
          if (!diag) S |= f.tm;
          chosen.push_back(&op);
          chosen_idx.push_back(i);
          ncoef += c;
          if (f.inner) ++ninner;
          if (chosen.size() >= size_t(sb.max_ops)) {
            ++i;
            break;
          }
          continue;
        }
        skipped_idx.push_back(i);
        blockT |= T;
        blockAll |= A;
        if (skipped_idx.size() >= kWindow || popc64(blockT) >= int(n)) {
          ++i;
          break;
        }
      }
      if (chosen.empty()) throw std::logic_error("planner: empty sweep");
      const uint64_t low_in = (uint64_t(1) << std::min<uint32_t>(l, 5)) - 1;
      uint64_t low_out = low_in;
      if (remap) {
        std::vector<const HostOp *> after;
        for (size_t x : skipped_idx) after.push_back(rem[x]);
        for (size_t x = i; x < rem.size(); ++x) after.push_back(rem[x]);
        uint64_t lo = 0;
        sb.outmap = choose_remap(after, S, virt_at, n, m, l, opt, kWindow, lo, tab);
        if (!sb.outmap.empty()) {
          low_out = lo;
          for (uint32_t b = 0; b < n; ++b)  // every bit the remap moves is a tile bit
            if (sb.outmap[b] != int(b)) S |= uint64_t(1) << b;
        }
      }
      std::vector<const HostOp *> order;
      schedule_phases(chosen, sb.reg_bits, low_in, low_out, order, sb.phase_regs, sb.phase_first);
      // More phases than a sweep holds: the ops of the excess phases go back
      // to the queue (every op they precede is among them).
      std::vector<size_t> back_idx;
      if (sb.phase_regs.size() > size_t(kMaxPhases)) {
        const size_t keep = sb.phase_first[kMaxPhases];
        for (size_t x = keep; x < order.size(); ++x) {
          const size_t pos = size_t(std::find(chosen.begin(), chosen.end(), order[x]) - chosen.begin());
          back_idx.push_back(chosen_idx[pos]);
        }
        order.resize(keep);
        sb.phase_regs.resize(kMaxPhases);
        sb.phase_first.resize(kMaxPhases);
      }
      sb.S = S;
      sb.ops = order;
      for (const HostOp *op : order) {
        sb.ncoef += SweepBuilder::coef_count(*op);
        if (op->kind == kOpInner) ++sb.ninner;
      }
      PlannedLaunch pl;
      pl.is_sweep = true;
      pl.sweep = sb.finish();
      pl.sweep.recipe = recipe(sb);
      out.push_back(std::move(pl));
      std::vector<size_t> again(skipped_idx);
      again.insert(again.end(), back_idx.begin(), back_idx.end());
      std::sort(again.begin(), again.end());
      std::vector<const HostOp *> next;
      for (size_t x : again) next.push_back(rem[x]);
      next.insert(next.end(), rem.begin() + i, rem.end());
      if (!sb.outmap.empty()) {
        // Ops after the sweep see its stored bit order.
        for (const HostOp *op : next) {
          relabel(const_cast<HostOp &>(*op), sb.outmap);
          tab.set(*op, opt);
        }
        std::vector<int> va(n);
        for (uint32_t b = 0; b < n; ++b) va[size_t(sb.outmap[b])] = virt_at[b];
        virt_at.swap(va);
      }
      rem.swap(next);
      head = 0;
      continue;
    }
    std::vector<const HostOp *> skipped;
    uint64_t blockT = 0, blockAll = 0;  // non-diagonal / all bits of skipped gates
    size_t i = head;
    for (; i < rem.size(); ++i) {
      const HostOp &op = *rem[i];
      const uint64_t T = op.nondiag_mask(), A = op.touched_mask();
      const bool commutes = (T & blockAll) == 0 && (A & blockT) == 0;
      if (commutes && sb.try_add(op)) continue;
      if (!opt.reorder) break;
      skipped.push_back(&op);
      blockT |= T;
      blockAll |= A;
      if (skipped.size() >= kWindow || popc64(blockT) >= int(n)) {
        ++i;
        break;
      }
    }
    if (sb.ops.empty()) throw std::logic_error("planner: first gate does not fit an empty sweep");
    PlannedLaunch pl;
    pl.is_sweep = true;
    pl.sweep = sb.finish();
    pl.sweep.recipe = recipe(sb);
    out.push_back(std::move(pl));
    // Remaining = skipped (in order) + everything after i.
    std::vector<const HostOp *> next(skipped.begin(), skipped.end());
    next.insert(next.end(), rem.begin() + i, rem.end());
    rem.swap(next);
    head = 0;
  }
  if (remap) {
    // Bits still away from home: one sweep of no gates whose tile holds them
    // (and the low bits) stores each at home.
    uint64_t moved = 0;
    for (uint32_t p = 0; p < n; ++p)
      if (virt_at[p] != int(p)) moved |= uint64_t(1) << p;
    if (moved) {
      SweepBuilder sb(n, m, l);
      sb.S |= moved;
      if (uint32_t(popc64(sb.S)) > m) throw std::logic_error("planner: restoration exceeds a tile");
      sb.outmap.resize(n);
      for (uint32_t p = 0; p < n; ++p) sb.outmap[p] = virt_at[p];
      // One phase without gates: its register bits avoid the bits loaded
      // from and stored to the low bits where the tile allows.
      uint64_t tile = sb.S;
      for (uint32_t b = 0; b < n && uint32_t(popc64(tile)) < m; ++b) tile |= uint64_t(1) << b;
      uint64_t avoid = (uint64_t(1) << std::min<uint32_t>(l, 5)) - 1;
      for (uint32_t p = 0; p < n; ++p)
        if (sb.outmap[p] < int(std::min<uint32_t>(l, 5))) avoid |= uint64_t(1) << p;
      uint64_t regs = 0;
      for (int b = int(n) - 1; b >= 0 && popc64(regs) < int(opt.reg_bits); --b)
        if (((tile >> b) & 1) && !((avoid >> b) & 1)) regs |= uint64_t(1) << b;
      sb.reg_bits = opt.reg_bits;
      sb.phase_regs.push_back(regs);
      sb.phase_first.push_back(0);
      PlannedLaunch pl;
      pl.is_sweep = true;
      pl.sweep = sb.finish();
      out.push_back(std::move(pl));
    }
  }
  return out;
}

std::vector<uint64_t> op_signature(const std::vector<HostOp> &ops) {
  std::vector<uint64_t> sig;
  sig.reserve(ops.size() * 4);
  for (const HostOp &op : ops) {
    sig.push_back(uint64_t(op.kind) | (uint64_t(op.inner_diag) << 8) | (uint64_t(op.tbits.size()) << 16) |
                  (uint64_t(op.slot) << 32));
    uint64_t t = 0;
    for (size_t j = 0; j < op.tbits.size(); ++j) t = (t << 7) | uint64_t(op.tbits[j] & 127);
    sig.push_back(t);
    sig.push_back(op.cmask);
    sig.push_back(op.cval);
  }
  return sig;
}

std::pair<uint64_t, uint64_t> op_signature_hash(const std::vector<HostOp> &ops) {
  const std::vector<uint64_t> sig = op_signature(ops);
  uint64_t a = 1469598103934665603ull, b = 0x9ae16a3b2f90404full;
  for (uint64_t w : sig)
    for (int k = 0; k < 8; ++k) {
      const uint8_t x = uint8_t(w >> (8 * k));
      a = (a ^ x) * 1099511628211ull;
      b = (b ^ x) * 0x100000001b3ull + 0x9e3779b97f4a7c15ull;
    }
  return {a, b ^ sig.size()};
}

bool rebuild_sweep(const SweepRecipe &r, const std::vector<HostOp> &ops, uint32_t n, uint32_t m, uint32_t l,
                   PlannedSweep &out) {
  if (r.src.empty()) return false;
  SweepBuilder sb(n, m, l);
  sb.S = r.S;
  sb.phase_regs = r.phase_regs;
  sb.phase_first = r.phase_first;
  sb.reg_bits = r.reg_bits;
  sb.max_dense_k = r.max_dense_k;
  for (uint32_t i : r.src) {
    if (i >= ops.size()) return false;
    sb.ops.push_back(&ops[i]);
    sb.ncoef += SweepBuilder::coef_count(ops[i]);
    if (ops[i].kind == kOpInner) ++sb.ninner;
  }
  out = sb.finish();
  out.recipe = r;
  return true;
}

bool rebuild_plan(std::vector<PlannedLaunch> &plan, const std::vector<HostOp> &ops, uint32_t n) {
  for (PlannedLaunch &pl : plan) {
    if (!pl.is_sweep) {
      if (pl.gate_src >= ops.size()) return false;
      pl.gate = ops[pl.gate_src];
      continue;
    }
    PlannedSweep &old = pl.sweep;
    PlannedSweep ns;
    if (!rebuild_sweep(old.recipe, ops, n, old.h.m, old.h.l, ns)) return false;
    if (std::memcmp(&ns.h, &old.h, sizeof(SweepHeader)) != 0 || ns.ph.size() != old.ph.size() ||
        ns.op.size() != old.op.size() || ns.inner_global != old.inner_global ||
        (!ns.ph.empty() && std::memcmp(ns.ph.data(), old.ph.data(), ns.ph.size() * sizeof(SweepPhase)) != 0) ||
        (!ns.op.empty() && std::memcmp(ns.op.data(), old.op.data(), ns.op.size() * sizeof(SweepOp)) != 0))
      return false;
    old.coef.swap(ns.coef);
  }
  return true;
}

}  // namespace sq

// Gate-matrix factory and structure analysis.
//
// Matrices follow the reference constructors
// (src/braket/snuqs/csrc/operation/gate_operations.cc:9-734): same entries,
// same formulas (cos/sin of half angles, e^{i x} as (cos x, sin x)), so the
// engine applies the reference's numbers.  ECR, CV and PRx, which the
// reference removed (src/braket/snuqs/gate_operations.py:238), follow their
// Amazon Braket definitions.
#include <cmath>

#include "../../include/snuqs_b200.h"
#include "host_ops.h"

namespace sq {

static cplx cis(double x) { return cplx(std::cos(x), std::sin(x)); }

int gate_qubits(int g) {
  switch (g) {
    case SQ_GATE_GPHASE: return 0;
    case SQ_GATE_CX: case SQ_GATE_CY: case SQ_GATE_CZ: case SQ_GATE_CPHASE_SHIFT:
    case SQ_GATE_CPHASE_SHIFT00: case SQ_GATE_CPHASE_SHIFT01: case SQ_GATE_CPHASE_SHIFT10:
    case SQ_GATE_SWAP: case SQ_GATE_ISWAP: case SQ_GATE_PSWAP: case SQ_GATE_XY:
    case SQ_GATE_XX: case SQ_GATE_YY: case SQ_GATE_ZZ: case SQ_GATE_SWAP_A2A:
    case SQ_GATE_ECR: case SQ_GATE_CV:
      return 2;
    case SQ_GATE_CCNOT: case SQ_GATE_CSWAP: return 3;
    default: return (g >= 0 && g < SQ_GATE_COUNT) ? 1 : -1;
  }
}

int gate_num_angles(int g) {
  switch (g) {
    case SQ_GATE_PHASE_SHIFT: case SQ_GATE_CPHASE_SHIFT: case SQ_GATE_CPHASE_SHIFT00:
    case SQ_GATE_CPHASE_SHIFT01: case SQ_GATE_CPHASE_SHIFT10: case SQ_GATE_ROT_X:
    case SQ_GATE_ROT_Y: case SQ_GATE_ROT_Z: case SQ_GATE_PSWAP: case SQ_GATE_XY:
    case SQ_GATE_XX: case SQ_GATE_YY: case SQ_GATE_ZZ: case SQ_GATE_GPHASE:
      return 1;
    case SQ_GATE_PRX: return 2;
    case SQ_GATE_U: return 3;
    default: return g >= 0 && g < SQ_GATE_COUNT ? 0 : -1;
  }
}

int gate_matrix(int g, const double *a, uint32_t na, std::vector<cplx> &out) {
  const int k = gate_qubits(g);
  if (k < 0 || int(na) < gate_num_angles(g)) return -1;
  const int d = 1 << k;
  out.assign(size_t(d) * d, cplx(0, 0));
  auto M = [&](int r, int c) -> cplx & { return out[size_t(r) * d + c]; };
  const cplx one(1, 0), I(0, 1);
  switch (g) {
    case SQ_GATE_IDENTITY: M(0, 0) = one; M(1, 1) = one; break;
    case SQ_GATE_HADAMARD:
      M(0, 0) = M(0, 1) = M(1, 0) = M_SQRT1_2; M(1, 1) = -M_SQRT1_2; break;
    case SQ_GATE_PAULI_X: M(0, 1) = one; M(1, 0) = one; break;
    case SQ_GATE_PAULI_Y: M(0, 1) = -I; M(1, 0) = I; break;
    case SQ_GATE_PAULI_Z: M(0, 0) = one; M(1, 1) = -1.0; break;
    case SQ_GATE_S: M(0, 0) = one; M(1, 1) = I; break;
    case SQ_GATE_SI: M(0, 0) = one; M(1, 1) = -I; break;
    case SQ_GATE_T: M(0, 0) = one; M(1, 1) = cis(M_PI / 4.); break;
    case SQ_GATE_TI: M(0, 0) = one; M(1, 1) = cis(-M_PI / 4.); break;
    case SQ_GATE_V:
      M(0, 0) = M(1, 1) = cplx(.5, .5); M(0, 1) = M(1, 0) = cplx(.5, -.5); break;
    case SQ_GATE_VI:
      M(0, 0) = M(1, 1) = cplx(.5, -.5); M(0, 1) = M(1, 0) = cplx(.5, .5); break;
    case SQ_GATE_PHASE_SHIFT: M(0, 0) = one; M(1, 1) = cis(a[0]); break;
    case SQ_GATE_ROT_X: {
      const double c = std::cos(a[0] / 2), s = std::sin(a[0] / 2);
      M(0, 0) = M(1, 1) = c; M(0, 1) = M(1, 0) = cplx(0, -s);
    } break;
    case SQ_GATE_ROT_Y: {
      const double c = std::cos(a[0] / 2), s = std::sin(a[0] / 2);
      M(0, 0) = M(1, 1) = c; M(0, 1) = -s; M(1, 0) = s;
    } break;
    case SQ_GATE_ROT_Z: M(0, 0) = cis(-a[0] / 2.); M(1, 1) = cis(a[0] / 2.); break;
    case SQ_GATE_U: {
      const double c = std::cos(a[0] / 2), s = std::sin(a[0] / 2);
      const cplx el = cis(a[2]), ep = cis(a[1]), epl = cis(a[1] + a[2]);
      M(0, 0) = c;
      M(0, 1) = cplx(-el.real() * s, -el.imag() * s);
      M(1, 0) = cplx(ep.real() * s, ep.imag() * s);
      M(1, 1) = cplx(epl.real() * c, epl.imag() * c);
    } break;
    case SQ_GATE_PRX: {
      const double c = std::cos(a[0] / 2), s = std::sin(a[0] / 2);
      const cplx em = cis(-a[1]), ep = cis(a[1]);
      M(0, 0) = M(1, 1) = c;
      M(0, 1) = -I * cplx(em.real() * s, em.imag() * s);
      M(1, 0) = -I * cplx(ep.real() * s, ep.imag() * s);
    } break;
    case SQ_GATE_CX: M(0, 0) = M(1, 1) = M(2, 3) = M(3, 2) = one; break;
    case SQ_GATE_CY: M(0, 0) = M(1, 1) = one; M(2, 3) = -I; M(3, 2) = I; break;
    case SQ_GATE_CZ: M(0, 0) = M(1, 1) = M(2, 2) = one; M(3, 3) = -1.0; break;
    case SQ_GATE_CV:
      M(0, 0) = M(1, 1) = one;
      M(2, 2) = M(3, 3) = cplx(.5, .5); M(2, 3) = M(3, 2) = cplx(.5, -.5); break;
    case SQ_GATE_CPHASE_SHIFT: M(0, 0) = M(1, 1) = M(2, 2) = one; M(3, 3) = cis(a[0]); break;
    case SQ_GATE_CPHASE_SHIFT00: M(0, 0) = cis(a[0]); M(1, 1) = M(2, 2) = M(3, 3) = one; break;
    case SQ_GATE_CPHASE_SHIFT01: M(1, 1) = cis(a[0]); M(0, 0) = M(2, 2) = M(3, 3) = one; break;
    case SQ_GATE_CPHASE_SHIFT10: M(2, 2) = cis(a[0]); M(0, 0) = M(1, 1) = M(3, 3) = one; break;
    case SQ_GATE_SWAP: case SQ_GATE_SWAP_A2A: M(0, 0) = M(1, 2) = M(2, 1) = M(3, 3) = one; break;
    case SQ_GATE_ISWAP: M(0, 0) = M(3, 3) = one; M(1, 2) = M(2, 1) = I; break;
    case SQ_GATE_PSWAP: M(0, 0) = M(3, 3) = one; M(1, 2) = M(2, 1) = cis(a[0]); break;
    case SQ_GATE_XY: {
      const double c = std::cos(a[0] / 2), s = std::sin(a[0] / 2);
      M(0, 0) = M(3, 3) = one; M(1, 1) = M(2, 2) = c; M(1, 2) = M(2, 1) = cplx(0, s);
    } break;
    case SQ_GATE_XX: {
      const double c = std::cos(a[0] / 2), s = std::sin(a[0] / 2);
      M(0, 0) = M(1, 1) = M(2, 2) = M(3, 3) = c;
      M(0, 3) = M(1, 2) = M(2, 1) = M(3, 0) = cplx(0, -s);
    } break;
    case SQ_GATE_YY: {
      const double c = std::cos(a[0] / 2), s = std::sin(a[0] / 2);
      M(0, 0) = M(1, 1) = M(2, 2) = M(3, 3) = c;
      M(0, 3) = M(3, 0) = cplx(0, s); M(1, 2) = M(2, 1) = cplx(0, -s);
    } break;
    case SQ_GATE_ZZ: {
      const cplx p = cis(a[0] / 2.), q = cis(-a[0] / 2.);
      M(0, 0) = M(3, 3) = q; M(1, 1) = M(2, 2) = p;
    } break;
    case SQ_GATE_ECR: {
      const double r = M_SQRT1_2;
      M(0, 2) = M(1, 3) = M(2, 0) = M(3, 1) = r;
      M(0, 3) = M(1, 2) = cplx(0, r); M(2, 1) = M(3, 0) = cplx(0, -r);
    } break;
    case SQ_GATE_CCNOT:
      for (int i = 0; i < 6; ++i) M(i, i) = one;
      M(6, 7) = M(7, 6) = one;
      break;
    case SQ_GATE_CSWAP:
      for (int i = 0; i < 8; ++i) M(i, i) = one;
      M(5, 5) = M(6, 6) = 0.0; M(5, 6) = M(6, 5) = one;
      break;
    case SQ_GATE_GPHASE: M(0, 0) = cis(a[0]); break;
    default: return -1;
  }
  return k;
}

int gate_matrix_derivative(int g, const double *a, uint32_t na, int param, std::vector<cplx> &out) {
  const int k = gate_qubits(g);
  const int nang = gate_num_angles(g);
  if (k < 0 || int(na) < nang || param < 0 || param >= nang) return -1;
  const int d = 1 << k;
  out.assign(size_t(d) * d, cplx(0, 0));
  auto M = [&](int r, int c) -> cplx & { return out[size_t(r) * d + c]; };
  const cplx I(0, 1);
  const double th = a[0];
  const double c = std::cos(th / 2), s = std::sin(th / 2);
  switch (g) {
    case SQ_GATE_PHASE_SHIFT: M(1, 1) = I * cis(th); break;
    case SQ_GATE_CPHASE_SHIFT: M(3, 3) = I * cis(th); break;
    case SQ_GATE_CPHASE_SHIFT00: M(0, 0) = I * cis(th); break;
    case SQ_GATE_CPHASE_SHIFT01: M(1, 1) = I * cis(th); break;
    case SQ_GATE_CPHASE_SHIFT10: M(2, 2) = I * cis(th); break;
    case SQ_GATE_GPHASE: M(0, 0) = I * cis(th); break;
    case SQ_GATE_ROT_X:
      M(0, 0) = M(1, 1) = -s / 2;
      M(0, 1) = M(1, 0) = cplx(0, -c / 2);
      break;
    case SQ_GATE_ROT_Y:
      M(0, 0) = M(1, 1) = -s / 2;
      M(0, 1) = -c / 2;
      M(1, 0) = c / 2;
      break;
    case SQ_GATE_ROT_Z:
      M(0, 0) = -I / 2.0 * cis(-th / 2.);
      M(1, 1) = I / 2.0 * cis(th / 2.);
      break;
    case SQ_GATE_PSWAP: M(1, 2) = M(2, 1) = I * cis(th); break;
    case SQ_GATE_XY:
      M(1, 1) = M(2, 2) = -s / 2;
      M(1, 2) = M(2, 1) = cplx(0, c / 2);
      break;
    case SQ_GATE_XX:
      M(0, 0) = M(1, 1) = M(2, 2) = M(3, 3) = -s / 2;
      M(0, 3) = M(1, 2) = M(2, 1) = M(3, 0) = cplx(0, -c / 2);
      break;
    case SQ_GATE_YY:
      M(0, 0) = M(1, 1) = M(2, 2) = M(3, 3) = -s / 2;
      M(0, 3) = M(3, 0) = cplx(0, c / 2);
      M(1, 2) = M(2, 1) = cplx(0, -c / 2);
      break;
    case SQ_GATE_ZZ:
      M(0, 0) = M(3, 3) = -I / 2.0 * cis(-th / 2.);
      M(1, 1) = M(2, 2) = I / 2.0 * cis(th / 2.);
      break;
    case SQ_GATE_U: {
      const cplx el = cis(a[2]), ep = cis(a[1]), epl = cis(a[1] + a[2]);
      if (param == 0) {
        M(0, 0) = -s / 2;
        M(0, 1) = -el * (c / 2);
        M(1, 0) = ep * (c / 2);
        M(1, 1) = -epl * (s / 2);
      } else if (param == 1) {
        M(1, 0) = I * ep * s;
        M(1, 1) = I * epl * c;
      } else {
        M(0, 1) = -I * el * s;
        M(1, 1) = I * epl * c;
      }
    } break;
    case SQ_GATE_PRX: {
      const cplx em = cis(-a[1]), ep = cis(a[1]);
      if (param == 0) {
        M(0, 0) = M(1, 1) = -s / 2;
        M(0, 1) = -I * em * (c / 2);
        M(1, 0) = -I * ep * (c / 2);
      } else {
        M(0, 1) = -em * s;
        M(1, 0) = ep * s;
      }
    } break;
    default: return -1;
  }
  return k;
}

uint64_t HostOp::target_mask() const {
  uint64_t r = 0;
  for (int b : tbits) r |= uint64_t(1) << b;
  return r;
}
uint64_t HostOp::touched_mask() const { return target_mask() | cmask; }
uint64_t HostOp::nondiag_mask() const {
  if (kind == kOpDiag || (kind == kOpInner && inner_diag)) return 0;
  return target_mask();
}

namespace {

bool is_diagonal(const std::vector<cplx> &m, int d) {
  for (int r = 0; r < d; ++r)
    for (int c = 0; c < d; ++c)
      if (r != c && m[size_t(r) * d + c] != cplx(0, 0)) return false;
  return true;
}

// Is local bit `b` of a d x d matrix a control with value v?  That is: the
// matrix never couples b=0 with b=1 and is the exact identity on b = !v.
bool is_control(const std::vector<cplx> &m, int d, int b, int v) {
  for (int r = 0; r < d; ++r)
    for (int c = 0; c < d; ++c) {
      const cplx x = m[size_t(r) * d + c];
      const int rb = (r >> b) & 1, cb = (c >> b) & 1;
      if (rb != cb) {
        if (x != cplx(0, 0)) return false;
      } else if (rb != v) {
        if (x != (r == c ? cplx(1, 0) : cplx(0, 0))) return false;
      }
    }
  return true;
}

// Block of m where local bit b equals v, as a (d/2) x (d/2) matrix.
std::vector<cplx> take_block(const std::vector<cplx> &m, int d, int b, int v) {
  const int h = d / 2;
  std::vector<cplx> out(size_t(h) * h);
  auto expand = [&](int x) {
    const int lo = x & ((1 << b) - 1);
    return ((x >> b) << (b + 1)) | (v << b) | lo;
  };
  for (int r = 0; r < h; ++r)
    for (int c = 0; c < h; ++c) out[size_t(r) * h + c] = m[size_t(expand(r)) * d + expand(c)];
  return out;
}

}  // namespace

bool analyse_op(const std::vector<cplx> &m0, const std::vector<int> &tb0, uint64_t cmask,
                uint64_t cval, HostOp &out) {
  std::vector<cplx> m = m0;
  std::vector<int> tb = tb0;
  int k = int(tb.size());
  int d = 1 << k;
  // Peel exact controls off the target list.
  bool changed = true;
  while (changed && k > 0 && !is_diagonal(m, d)) {
    changed = false;
    for (int j = 0; j < k; ++j) {
      const int b = k - 1 - j;  // local bit of target j
      for (int v = 1; v >= 0; --v) {
        if (is_control(m, d, b, v)) {
          m = take_block(m, d, b, v);
          cmask |= uint64_t(1) << tb[j];
          if (v) cval |= uint64_t(1) << tb[j];
          tb.erase(tb.begin() + j);
          --k;
          d >>= 1;
          changed = true;
          break;
        }
      }
      if (changed) break;
    }
  }
  out = HostOp();
  if (is_diagonal(m, d)) {
    // Diagonal: fold the controls into the diagonal (identity where they fail).
    std::vector<int> bits;
    for (int b = 63; b >= 0; --b)
      if ((cmask >> b) & 1) bits.push_back(b);
    const int nc = int(bits.size());
    bits.insert(bits.end(), tb.begin(), tb.end());
    const int kk = int(bits.size());
    std::vector<cplx> diag(size_t(1) << kk, cplx(1, 0));
    bool identity = true;
    for (int x = 0; x < (1 << kk); ++x) {
      bool ok = true;
      for (int c = 0; c < nc; ++c) {
        const int bitv = (x >> (kk - 1 - c)) & 1;
        if (bitv != int((cval >> bits[c]) & 1)) ok = false;
      }
      if (ok) diag[x] = m[size_t(x & (d - 1)) * d + (x & (d - 1))];
      if (diag[x] != cplx(1, 0)) identity = false;
    }
    if (identity) return false;
    // Drop controls again if the folded diagonal is too wide for one op; the
    // caller then treats it as a dense gate.
    if (kk > kMaxDiagK) {
      out.kind = kOpDense;
      out.tbits = tb;
      out.cmask = cmask;
      out.cval = cval;
      out.m = m;
      return true;
    }
    out.kind = kOpDiag;
    out.tbits = bits;
    out.m = diag;
    return true;
  }
  out.kind = kOpDense;
  out.tbits = tb;
  out.cmask = cmask;
  out.cval = cval;
  out.m = m;
  return true;
}

}  // namespace sq

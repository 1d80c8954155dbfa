/*
 * TEST ORACLE ONLY -- a plain-C restatement of the reference's CPU gate path.
 * Only tests/, the smoke check and bench.py's CPU-baseline leg may load it,
 * and only as the checker; the product never links it.
 *
 * Restated from (paths within the reference project):
 *   - gate matrices        src/braket/snuqs/csrc/operation/gate_operations.cc:9-734
 *   - cpu::applyGate       src/braket/snuqs/csrc/operation/gate_operations_impl_cpu.cc:10-148
 *   - initializeBasis_Z    src/braket/snuqs/csrc/operation/initialization_impl_cpu.cc:15-22
 * Gates the reference lacks (ECR, CV, PRx; gate_operations.py:238 lists them as
 * removed) follow their published Amazon Braket definitions.
 *
 * Arithmetic contract (so the restatement is bit-exact with the compiled
 * reference): complex products are (ac-bd, ad+bc) with no FMA contraction
 * (compile with -ffp-contract=off), and each output row is accumulated left
 * to right, g[r][0]*a0 + g[r][1]*a1 + ..., exactly as the reference's
 * unrolled expressions do (gate_operations_impl_cpu.cc:34-35, 58-65, 95-126).
 * Pinned against oracle/_ref (the reference compiled from its sources) and
 * the fixtures under tests/golden/.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

/* GateOperationType order of operation.h:17-52, then the gates this engine
 * adds. */
enum {
  OG_I = 0, OG_H, OG_X, OG_Y, OG_Z, OG_CX, OG_CY, OG_CZ, OG_S, OG_SI, OG_T,
  OG_TI, OG_V, OG_VI, OG_PHASESHIFT, OG_CPHASESHIFT, OG_CPHASESHIFT00,
  OG_CPHASESHIFT01, OG_CPHASESHIFT10, OG_RX, OG_RY, OG_RZ, OG_SWAP, OG_ISWAP,
  OG_PSWAP, OG_XY, OG_XX, OG_YY, OG_ZZ, OG_CCNOT, OG_CSWAP, OG_U, OG_GPHASE,
  OG_SWAPA2A, OG_ECR, OG_CV, OG_PRX, OG_COUNT
};

typedef struct { double re, im; } cplx;

static cplx C(double re, double im) { cplx z = {re, im}; return z; }
static cplx cmul(cplx a, cplx b) { return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static cplx cadd(cplx a, cplx b) { return C(a.re + b.re, a.im + b.im); }
/* std::exp(i*x) for real x: exp(0) * (cos x, sin x). */
static cplx cis(double x) { return C(cos(x), sin(x)); }

int oracle_gate_qubits(int type) {
  switch (type) {
    case OG_GPHASE: return 0;
    case OG_CX: case OG_CY: case OG_CZ: case OG_CPHASESHIFT: case OG_CPHASESHIFT00:
    case OG_CPHASESHIFT01: case OG_CPHASESHIFT10: case OG_SWAP: case OG_ISWAP:
    case OG_PSWAP: case OG_XY: case OG_XX: case OG_YY: case OG_ZZ: case OG_SWAPA2A:
    case OG_ECR: case OG_CV:
      return 2;
    case OG_CCNOT: case OG_CSWAP: return 3;
    default:
      return (type >= 0 && type < OG_COUNT) ? 1 : -1;
  }
}

int oracle_gate_num_angles(int type) {
  switch (type) {
    case OG_PHASESHIFT: case OG_CPHASESHIFT: case OG_CPHASESHIFT00: case OG_CPHASESHIFT01:
    case OG_CPHASESHIFT10: case OG_RX: case OG_RY: case OG_RZ: case OG_PSWAP: case OG_XY:
    case OG_XX: case OG_YY: case OG_ZZ: case OG_GPHASE:
      return 1;
    case OG_PRX: return 2;
    case OG_U: return 3;
    default: return 0;
  }
}

/* Writes the 2^k x 2^k row-major matrix of `type` into out (interleaved
 * re/im).  Returns k, or -1 for an unknown type. */
int oracle_gate_matrix(int type, const double *a, double *out) {
  int k = oracle_gate_qubits(type);
  if (k < 0) return -1;
  int d = 1 << k;
  cplx m[64];
  for (int i = 0; i < d * d; ++i) m[i] = C(0, 0);
#define M(r, c) m[(r) * d + (c)]
  switch (type) {
    case OG_I: M(0, 0) = C(1, 0); M(1, 1) = C(1, 0); break;
    case OG_H: M(0, 0) = C(M_SQRT1_2, 0); M(0, 1) = C(M_SQRT1_2, 0);
               M(1, 0) = C(M_SQRT1_2, 0); M(1, 1) = C(-M_SQRT1_2, 0); break;
    case OG_X: M(0, 1) = C(1, 0); M(1, 0) = C(1, 0); break;
    case OG_Y: M(0, 1) = C(0, -1); M(1, 0) = C(0, 1); break;
    case OG_Z: M(0, 0) = C(1, 0); M(1, 1) = C(-1, 0); break;
    case OG_S: M(0, 0) = C(1, 0); M(1, 1) = C(0, 1); break;
    case OG_SI: M(0, 0) = C(1, 0); M(1, 1) = C(0, -1); break;
    case OG_T: M(0, 0) = C(1, 0); M(1, 1) = cis(M_PI / 4.); break;
    case OG_TI: M(0, 0) = C(1, 0); M(1, 1) = cis(-M_PI / 4.); break;
    case OG_V: M(0, 0) = C(.5, .5); M(0, 1) = C(.5, -.5); M(1, 0) = C(.5, -.5); M(1, 1) = C(.5, .5); break;
    case OG_VI: M(0, 0) = C(.5, -.5); M(0, 1) = C(.5, .5); M(1, 0) = C(.5, .5); M(1, 1) = C(.5, -.5); break;
    case OG_PHASESHIFT: M(0, 0) = C(1, 0); M(1, 1) = cis(a[0]); break;
    case OG_RX: {
      double c = cos(a[0] / 2), s = sin(a[0] / 2);
      M(0, 0) = C(c, 0); M(0, 1) = C(0, -s); M(1, 0) = C(0, -s); M(1, 1) = C(c, 0);
    } break;
    case OG_RY: {
      double c = cos(a[0] / 2), s = sin(a[0] / 2);
      M(0, 0) = C(c, 0); M(0, 1) = C(-s, 0); M(1, 0) = C(s, 0); M(1, 1) = C(c, 0);
    } break;
    case OG_RZ: M(0, 0) = cis(-a[0] / 2.); M(1, 1) = cis(a[0] / 2.); break;
    case OG_U: {
      double c = cos(a[0] / 2), s = sin(a[0] / 2);
      cplx el = cis(a[2]), ep = cis(a[1]), epl = cis(a[1] + a[2]);
      M(0, 0) = C(c, 0);
      M(0, 1) = C(-el.re * s, -el.im * s);
      M(1, 0) = C(ep.re * s, ep.im * s);
      M(1, 1) = C(epl.re * c, epl.im * c);
    } break;
    case OG_PRX: {  /* Braket PRx(theta, phi) */
      double c = cos(a[0] / 2), s = sin(a[0] / 2);
      cplx em = cis(-a[1]), ep = cis(a[1]);
      M(0, 0) = C(c, 0);
      M(0, 1) = cmul(C(0, -1), C(em.re * s, em.im * s));
      M(1, 0) = cmul(C(0, -1), C(ep.re * s, ep.im * s));
      M(1, 1) = C(c, 0);
    } break;
    case OG_CX: M(0, 0) = C(1, 0); M(1, 1) = C(1, 0); M(2, 3) = C(1, 0); M(3, 2) = C(1, 0); break;
    case OG_CY: M(0, 0) = C(1, 0); M(1, 1) = C(1, 0); M(2, 3) = C(0, -1); M(3, 2) = C(0, 1); break;
    case OG_CZ: M(0, 0) = C(1, 0); M(1, 1) = C(1, 0); M(2, 2) = C(1, 0); M(3, 3) = C(-1, 0); break;
    case OG_CV:
      M(0, 0) = C(1, 0); M(1, 1) = C(1, 0);
      M(2, 2) = C(.5, .5); M(2, 3) = C(.5, -.5); M(3, 2) = C(.5, -.5); M(3, 3) = C(.5, .5);
      break;
    case OG_CPHASESHIFT: M(0, 0) = C(1, 0); M(1, 1) = C(1, 0); M(2, 2) = C(1, 0); M(3, 3) = cis(a[0]); break;
    case OG_CPHASESHIFT00: M(0, 0) = cis(a[0]); M(1, 1) = C(1, 0); M(2, 2) = C(1, 0); M(3, 3) = C(1, 0); break;
    case OG_CPHASESHIFT01: M(0, 0) = C(1, 0); M(1, 1) = cis(a[0]); M(2, 2) = C(1, 0); M(3, 3) = C(1, 0); break;
    case OG_CPHASESHIFT10: M(0, 0) = C(1, 0); M(1, 1) = C(1, 0); M(2, 2) = cis(a[0]); M(3, 3) = C(1, 0); break;
    case OG_SWAP: case OG_SWAPA2A:
      M(0, 0) = C(1, 0); M(1, 2) = C(1, 0); M(2, 1) = C(1, 0); M(3, 3) = C(1, 0); break;
    case OG_ISWAP: M(0, 0) = C(1, 0); M(1, 2) = C(0, 1); M(2, 1) = C(0, 1); M(3, 3) = C(1, 0); break;
    case OG_PSWAP: M(0, 0) = C(1, 0); M(1, 2) = cis(a[0]); M(2, 1) = cis(a[0]); M(3, 3) = C(1, 0); break;
    case OG_XY: {  /* +i sin off-diagonals, gate_operations.cc:441-453 */
      double c = cos(a[0] / 2), s = sin(a[0] / 2);
      M(0, 0) = C(1, 0); M(1, 1) = C(c, 0); M(1, 2) = C(0, s);
      M(2, 1) = C(0, s); M(2, 2) = C(c, 0); M(3, 3) = C(1, 0);
    } break;
    case OG_XX: {
      double c = cos(a[0] / 2), s = sin(a[0] / 2);
      M(0, 0) = C(c, 0); M(0, 3) = C(0, -s); M(1, 1) = C(c, 0); M(1, 2) = C(0, -s);
      M(2, 1) = C(0, -s); M(2, 2) = C(c, 0); M(3, 0) = C(0, -s); M(3, 3) = C(c, 0);
    } break;
    case OG_YY: {  /* +i sin on the anti-corners, gate_operations.cc:500,509 */
      double c = cos(a[0] / 2), s = sin(a[0] / 2);
      M(0, 0) = C(c, 0); M(0, 3) = C(0, s); M(1, 1) = C(c, 0); M(1, 2) = C(0, -s);
      M(2, 1) = C(0, -s); M(2, 2) = C(c, 0); M(3, 0) = C(0, s); M(3, 3) = C(c, 0);
    } break;
    case OG_ZZ: {
      cplx p = cis(a[0] / 2.), q = cis(-a[0] / 2.);
      M(0, 0) = q; M(1, 1) = p; M(2, 2) = p; M(3, 3) = q;
    } break;
    case OG_ECR: {  /* Braket ECR: (1/sqrt2) [[0,0,1,i],[0,0,i,1],[1,-i,0,0],[-i,1,0,0]] */
      double r = M_SQRT1_2;
      M(0, 2) = C(r, 0); M(0, 3) = C(0, r); M(1, 2) = C(0, r); M(1, 3) = C(r, 0);
      M(2, 0) = C(r, 0); M(2, 1) = C(0, -r); M(3, 0) = C(0, -r); M(3, 1) = C(r, 0);
    } break;
    case OG_CCNOT:
      for (int i = 0; i < 6; ++i) M(i, i) = C(1, 0);
      M(6, 7) = C(1, 0); M(7, 6) = C(1, 0);
      break;
    case OG_CSWAP:
      for (int i = 0; i < 8; ++i) M(i, i) = C(1, 0);
      M(5, 5) = C(0, 0); M(6, 6) = C(0, 0); M(5, 6) = C(1, 0); M(6, 5) = C(1, 0);
      break;
    case OG_GPHASE: M(0, 0) = cis(a[0]); break;
    default: return -1;
  }
#undef M
  memcpy(out, m, sizeof(cplx) * (size_t)d * (size_t)d);
  return k;
}

/* cpu::applyGate restated for any k (the reference covers k = 0..3).
 * Local row/column index bit (k-1-j) corresponds to targets[j]
 * (targets[0] is the most significant), and qubit q is index bit nq-1-q. */
int oracle_apply(double *state, int nq, const double *matrix,
                 const int *targets, int k) {
  if (k < 0 || k > 10 || k > nq) return -1;
  cplx *psi = (cplx *)state;
  const cplx *g = (const cplx *)matrix;
  uint64_t n = (uint64_t)1 << nq;
  if (k == 0) {
    for (uint64_t i = 0; i < n; ++i) psi[i] = cmul(psi[i], g[0]);
    return 0;
  }
  int d = 1 << k;
  uint64_t off[1024];
  uint64_t tmask = 0;
  for (int c = 0; c < d; ++c) {
    uint64_t o = 0;
    for (int j = 0; j < k; ++j)
      if ((c >> (k - 1 - j)) & 1) o |= (uint64_t)1 << (nq - 1 - targets[j]);
    off[c] = o;
  }
  for (int j = 0; j < k; ++j) tmask |= (uint64_t)1 << (nq - 1 - targets[j]);
  cplx a[1024];
  for (uint64_t i = 0; i < n; ++i) {
    if (i & tmask) continue;
    for (int c = 0; c < d; ++c) a[c] = psi[i + off[c]];
    for (int r = 0; r < d; ++r) {
      cplx acc = cmul(g[r * d], a[0]);
      for (int c = 1; c < d; ++c) acc = cadd(acc, cmul(g[r * d + c], a[c]));
      psi[i + off[r]] = acc;
    }
  }
  return 0;
}

/* Builds the gate matrix and applies it: functionals::apply's CPU branch. */
int oracle_apply_gate(double *state, int nq, int type, const int *targets,
                      int k, const double *angles) {
  double m[128];
  int kk = oracle_gate_matrix(type, angles, m);
  if (kk < 0 || kk != k) return -1;
  return oracle_apply(state, nq, m, targets, k);
}

void oracle_initialize_basis_z(double *state, int nq) {
  uint64_t n = (uint64_t)1 << nq;
  memset(state, 0, sizeof(cplx) * n);
  state[0] = 1.0;
}

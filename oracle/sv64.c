/*
 * sv64.c — FP64 CPU statevector ORACLE (test infrastructure only).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * this library, as the checker or the timed CPU baseline; the product never
 * does.  It restates, in double precision, the semantics of the reference
 * kernels for the ops of include/qsim.h:
 *   - 1Q gate on target t: pairs (i, i | 1<<t), new0 = g00 a0 + g01 a1,
 *     new1 = g10 a0 + g11 a1          (bwk/csrc/apply_gate_sm120.cu:10-14)
 *   - 4x4 gate: index (b1 b0) over (i00, i01, i10, i11), new_r = sum_c G[r][c] a_c
 *                                     (bwk/csrc/apply_gate2q_sm120.cu:11-20);
 *     here bit 0 is the op's first listed target (include/qsim.h)
 *   - controls: insert zeros at the sorted qubit positions, then OR the
 *     control mask                     (bwk/csrc/apply_mcgate_sm120.cu:62-98,
 *                                       bwk/csrc/apply_mc2qgate_sm120.cu:76-123)
 *   - diagonals: state[i] *= d[bits of i] (bwk/csrc/apply_diagonal_sm120.cu:43-105)
 *   - |0..0> init                      (apply_diagonal_sm120.cu:109-113)
 * Rotation ops use exp(-i theta P / 2) (blackwell_backend/simulator.py:147-158).
 *
 * Build: cc -O2 -fopenmp -shared -fPIC sv64.c -o _build/libsv64.so (oracle/build_oracle.py)
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "../include/qsim.h"

typedef double complex cplx;

static uint64_t insert_zero(uint64_t x, int q) {
  uint64_t lo = x & ((1ull << q) - 1ull);
  return ((x ^ lo) << 1) | lo;
}

static void sort_ints(int* a, int k) {
  for (int i = 1; i < k; ++i) {
    int v = a[i], j = i - 1;
    while (j >= 0 && a[j] > v) { a[j + 1] = a[j]; --j; }
    a[j + 1] = v;
  }
}

static uint64_t deposit(uint64_t x, const int* sorted, int k) {
  for (int j = 0; j < k; ++j) x = insert_zero(x, sorted[j]);
  return x;
}

static cplx M(const qs_op* o, int i) { return o->m[2 * i] + I * o->m[2 * i + 1]; }

void sv64_init(cplx* psi, int n) {
  uint64_t N = 1ull << n;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)N; ++i) psi[i] = 0;
  psi[0] = 1;
}

/* controlled 2x2: controls c[0..nc-1], target t */
static void apply_c1(cplx* psi, int n, const int* c, int nc, int t, cplx g00, cplx g01, cplx g10, cplx g11) {
  int all[10];
  uint64_t cm = 0;
  for (int i = 0; i < nc; ++i) { all[i] = c[i]; cm |= 1ull << c[i]; }
  all[nc] = t;
  sort_ints(all, nc + 1);
  const uint64_t items = 1ull << (n - nc - 1), st = 1ull << t;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)items; ++p) {
    uint64_t i0 = deposit((uint64_t)p, all, nc + 1) | cm, i1 = i0 | st;
    cplx a0 = psi[i0], a1 = psi[i1];
    psi[i0] = g00 * a0 + g01 * a1;
    psi[i1] = g10 * a0 + g11 * a1;
  }
}

/* controlled 4x4 on (t0 = bit0, t1 = bit1) */
static void apply_c2(cplx* psi, int n, const int* c, int nc, int t0, int t1, const cplx* G) {
  int all[10];
  uint64_t cm = 0;
  for (int i = 0; i < nc; ++i) { all[i] = c[i]; cm |= 1ull << c[i]; }
  all[nc] = t0;
  all[nc + 1] = t1;
  sort_ints(all, nc + 2);
  const uint64_t items = 1ull << (n - nc - 2), s0 = 1ull << t0, s1 = 1ull << t1;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)items; ++p) {
    uint64_t i = deposit((uint64_t)p, all, nc + 2) | cm;
    uint64_t idx[4] = {i, i | s0, i | s1, i | s0 | s1};
    cplx a[4], o[4];
    for (int k = 0; k < 4; ++k) a[k] = psi[idx[k]];
    for (int r = 0; r < 4; ++r) o[r] = G[4 * r] * a[0] + G[4 * r + 1] * a[1] + G[4 * r + 2] * a[2] + G[4 * r + 3] * a[3];
    for (int k = 0; k < 4; ++k) psi[idx[k]] = o[k];
  }
}

static void apply_phase_all(cplx* psi, int n, const int* q, int k, cplx ph) {
  int s[10];
  uint64_t m = 0;
  for (int i = 0; i < k; ++i) { s[i] = q[i]; m |= 1ull << q[i]; }
  sort_ints(s, k);
  const uint64_t items = 1ull << (n - k);
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)items; ++p) {
    uint64_t i = deposit((uint64_t)p, s, k) | m;
    psi[i] *= ph;
  }
}

static void apply_diag(cplx* psi, int n, const int* q, int k, const cplx* d) {
  const uint64_t N = 1ull << n;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)N; ++i) {
    int sel = 0;
    for (int j = 0; j < k; ++j) sel |= (int)((((uint64_t)i) >> q[j]) & 1ull) << j;
    psi[i] *= d[sel];
  }
}

/* Returns 0 on success, -1 on an unsupported op. */
int sv64_apply_ops(cplx* psi, int n, const qs_op* ops, int nops) {
  for (int k = 0; k < nops; ++k) {
    const qs_op* o = &ops[k];
    const int nq = o->nq;
    const int* q = o->q;
    switch (o->kind) {
      case QS_OP_U1: apply_c1(psi, n, q, 0, q[0], M(o, 0), M(o, 1), M(o, 2), M(o, 3)); break;
      case QS_OP_MCU1: apply_c1(psi, n, q, nq - 1, q[nq - 1], M(o, 0), M(o, 1), M(o, 2), M(o, 3)); break;
      case QS_OP_MCX: apply_c1(psi, n, q, nq - 1, q[nq - 1], 0, 1, 1, 0); break;
      case QS_OP_Y: apply_c1(psi, n, q, 0, q[0], 0, -I, I, 0); break;
      case QS_OP_RX: case QS_OP_RY: case QS_OP_RZ: {
        const double th = o->m[0], c = cos(th / 2), s = sin(th / 2);
        if (o->kind == QS_OP_RX) apply_c1(psi, n, q, 0, q[0], c, -I * s, -I * s, c);
        else if (o->kind == QS_OP_RY) apply_c1(psi, n, q, 0, q[0], c, -s, s, c);
        else apply_c1(psi, n, q, 0, q[0], cexp(-I * th / 2), 0, 0, cexp(I * th / 2));
        break;
      }
      case QS_OP_U2: case QS_OP_MCU2: {
        cplx G[16];
        for (int i = 0; i < 16; ++i) G[i] = M(o, i);
        apply_c2(psi, n, q, nq - 2, q[nq - 2], q[nq - 1], G);
        break;
      }
      case QS_OP_MCSWAP: {
        cplx G[16] = {0};
        G[0] = 1; G[4 * 1 + 2] = 1; G[4 * 2 + 1] = 1; G[15] = 1;
        apply_c2(psi, n, q, nq - 2, q[nq - 2], q[nq - 1], G);
        break;
      }
      case QS_OP_MCPHASE: apply_phase_all(psi, n, q, nq, M(o, 0)); break;
      case QS_OP_DIAG1: { cplx d[2] = {M(o, 0), M(o, 1)}; apply_diag(psi, n, q, 1, d); break; }
      case QS_OP_DIAG2: { cplx d[4] = {M(o, 0), M(o, 1), M(o, 2), M(o, 3)}; apply_diag(psi, n, q, 2, d); break; }
      default: return -1;
    }
  }
  return 0;
}

/* |<a|b>|^2 / (|a|^2 |b|^2) with a complex64 (float pairs) and b complex128. */
double sv64_fidelity_c64(const float* a, const cplx* b, int n) {
  const uint64_t N = 1ull << n;
  double re = 0, im = 0, na = 0, nb = 0;
#pragma omp parallel for reduction(+ : re, im, na, nb) schedule(static)
  for (int64_t i = 0; i < (int64_t)N; ++i) {
    double ar = a[2 * i], ai = a[2 * i + 1];
    double br = creal(b[i]), bi = cimag(b[i]);
    re += ar * br + ai * bi;
    im += ar * bi - ai * br;
    na += ar * ar + ai * ai;
    nb += br * br + bi * bi;
  }
  return (re * re + im * im) / (na * nb);
}

/* max_i |a_i - b_i| */
double sv64_max_abs_err_c64(const float* a, const cplx* b, int n) {
  const uint64_t N = 1ull << n;
  double m = 0;
#pragma omp parallel for reduction(max : m) schedule(static)
  for (int64_t i = 0; i < (int64_t)N; ++i) {
    double dr = a[2 * i] - creal(b[i]), di = a[2 * i + 1] - cimag(b[i]);
    double e = sqrt(dr * dr + di * di);
    if (e > m) m = e;
  }
  return m;
}

/* sum_t c_t <psi|P_t|psi> with P = i^{|x&z|} X^x Z^z, in FP64: the same
 * definition as the numpy restatement sv_oracle.pauli_expectation (and the
 * reference's expectation_pauli, bwk/csrc/expectation_sm120.cu:100-163,
 * generalised to any X/Y/Z string). */
double sv64_expect_pauli(const cplx* psi, int n, const uint64_t* x, const uint64_t* z, const double* c,
                         int nterms) {
  const uint64_t N = 1ull << n;
  double tot = 0.0;
  for (int t = 0; t < nterms; ++t) {
    const int ny = __builtin_popcountll(x[t] & z[t]) & 3;
    const cplx ph = ny == 0 ? 1.0 : ny == 1 ? I : ny == 2 ? -1.0 : -I;
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
    for (int64_t i = 0; i < (int64_t)N; ++i) {
      const uint64_t j = (uint64_t)i ^ x[t];
      const double sg = (__builtin_popcountll(j & z[t]) & 1) ? -1.0 : 1.0;
      acc += creal(conj(psi[i]) * ph * sg * psi[j]);
    }
    tot += c[t] * acc;
  }
  return tot;
}

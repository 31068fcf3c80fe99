// qs_plan.cpp — host-side circuit planner (FP64) and plan execution.
//
// Replaces the reference's Python compile step
// (blackwell_backend/simulator.py:247-434, the 6-phase fusion) and dispatcher
// (simulator.py:439-468).  Differences by design:
//   * all matrix products run in FP64 on the host (the reference multiplies
//     complex64 tensors on the GPU, simulator.py:339-377);
//   * instead of one launch per fused op, the circuit is cut into tile passes
//     (qs_pass.cu): each pass streams the state through shared memory once and
//     applies every gate it holds in registers;
//   * diagonal gates, phases and controls never constrain a pass: they are
//     evaluated from the amplitude index wherever their qubits live.
#include "qs_api.h"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <array>
#include <map>
#include <set>
#include <tuple>

namespace {

using cd = std::complex<double>;

enum IKind { I_U1, I_U2, I_X, I_SWAP, I_Y, I_NEG, I_PHASE, I_DIAG1, I_DIAG2, I_RY, I_XRY };

inline bool is_diag_kind(int k) { return k == I_NEG || k == I_PHASE || k == I_DIAG1 || k == I_DIAG2; }

struct IOp {
  int kind;
  int tq[2] = {-1, -1};   // non-diagonal targets (bit0, bit1)
  int ntq = 0;
  std::vector<int> cq;    // controls (all must be 1); for PHASE/NEG: the qubits
  int dq[2] = {-1, -1};   // diagonal qubits (DIAG1/DIAG2)
  int ndq = 0;
  cd m[16];
};

// ------------------------------------------------------------ normalise --
void mat_from(const double* m, cd* out, int count) {
  for (int i = 0; i < count; ++i) out[i] = cd(m[2 * i], m[2 * i + 1]);
}

void check_q(int q, int n) {
  if (q < 0 || q >= n) throw qs_error(QS_ERR_INVALID, "op qubit index out of range");
}

std::vector<IOp> normalise(int n, const qs_op* ops, int nops) {
  std::vector<IOp> out;
  out.reserve(nops);
  for (int i = 0; i < nops; ++i) {
    const qs_op& o = ops[i];
    QS_CHECK_ARG(o.nq >= 0 && o.nq <= 8, "op nq out of range");
    for (int k = 0; k < o.nq; ++k) check_q(o.q[k], n);
    {
      std::set<int> u(o.q, o.q + o.nq);
      QS_CHECK_ARG((int)u.size() == o.nq, "op has a repeated qubit");
    }
    IOp p;
    switch (o.kind) {
      case QS_OP_U1:
        QS_CHECK_ARG(o.nq == 1, "U1 needs 1 qubit");
        p.kind = I_U1; p.tq[0] = o.q[0]; p.ntq = 1; mat_from(o.m, p.m, 4);
        break;
      case QS_OP_U2:
        QS_CHECK_ARG(o.nq == 2, "U2 needs 2 qubits");
        p.kind = I_U2; p.tq[0] = o.q[0]; p.tq[1] = o.q[1]; p.ntq = 2; mat_from(o.m, p.m, 16);
        break;
      case QS_OP_DIAG1:
        QS_CHECK_ARG(o.nq == 1, "DIAG1 needs 1 qubit");
        p.kind = I_DIAG1; p.dq[0] = o.q[0]; p.ndq = 1; mat_from(o.m, p.m, 2);
        break;
      case QS_OP_DIAG2:
        QS_CHECK_ARG(o.nq == 2, "DIAG2 needs 2 qubits");
        p.kind = I_DIAG2; p.dq[0] = o.q[0]; p.dq[1] = o.q[1]; p.ndq = 2; mat_from(o.m, p.m, 4);
        break;
      case QS_OP_MCU1:
        QS_CHECK_ARG(o.nq >= 1, "MCU1 needs a target");
        p.kind = I_U1; p.tq[0] = o.q[o.nq - 1]; p.ntq = 1;
        p.cq.assign(o.q, o.q + o.nq - 1); mat_from(o.m, p.m, 4);
        break;
      case QS_OP_MCU2:
        QS_CHECK_ARG(o.nq >= 2, "MCU2 needs two targets");
        p.kind = I_U2; p.tq[0] = o.q[o.nq - 2]; p.tq[1] = o.q[o.nq - 1]; p.ntq = 2;
        p.cq.assign(o.q, o.q + o.nq - 2); mat_from(o.m, p.m, 16);
        break;
      case QS_OP_MCX:
        QS_CHECK_ARG(o.nq >= 1, "MCX needs a target");
        p.kind = I_X; p.tq[0] = o.q[o.nq - 1]; p.ntq = 1; p.cq.assign(o.q, o.q + o.nq - 1);
        break;
      case QS_OP_MCSWAP:
        QS_CHECK_ARG(o.nq >= 2, "MCSWAP needs two targets");
        p.kind = I_SWAP; p.tq[0] = o.q[o.nq - 2]; p.tq[1] = o.q[o.nq - 1]; p.ntq = 2;
        p.cq.assign(o.q, o.q + o.nq - 2);
        break;
      case QS_OP_MCPHASE: {
        QS_CHECK_ARG(o.nq >= 1, "MCPHASE needs a qubit");
        cd ph(o.m[0], o.m[1]);
        p.kind = (ph == cd(-1.0, 0.0)) ? I_NEG : I_PHASE;
        p.cq.assign(o.q, o.q + o.nq);
        p.m[0] = ph;
        break;
      }
      case QS_OP_Y:
        QS_CHECK_ARG(o.nq == 1, "Y needs 1 qubit");
        p.kind = I_Y; p.tq[0] = o.q[0]; p.ntq = 1;
        break;
      case QS_OP_RX: case QS_OP_RY: case QS_OP_RZ: {
        QS_CHECK_ARG(o.nq == 1, "rotation needs 1 qubit");
        const double th = o.m[0], c = std::cos(th / 2), s = std::sin(th / 2);
        if (o.kind == QS_OP_RZ) {
          p.kind = I_DIAG1; p.dq[0] = o.q[0]; p.ndq = 1;
          p.m[0] = std::polar(1.0, -th / 2); p.m[1] = std::polar(1.0, th / 2);
        } else {
          p.kind = I_U1; p.tq[0] = o.q[0]; p.ntq = 1;
          if (o.kind == QS_OP_RX) { p.m[0] = c; p.m[1] = cd(0, -s); p.m[2] = cd(0, -s); p.m[3] = c; }
          else { p.m[0] = c; p.m[1] = -s; p.m[2] = s; p.m[3] = c; }
        }
        break;
      }
      case QS_OP_DEPOLARIZE: case QS_OP_AMP_DAMP: case QS_OP_DEPHASE:
        throw qs_error(QS_ERR_INVALID, "noise channel op in a unitary program (use qs_noise_trajectories)");
      default:
        throw qs_error(QS_ERR_INVALID, "unknown op kind " + std::to_string(o.kind));
    }
    if (p.kind == I_U1 && !p.cq.empty() && p.m[1] == 0.0 && p.m[2] == 0.0) {
      // controlled diagonal: phase d0 where the controls are set, times
      // d1/d0 where controls and target are set
      IOp a, b;
      a.kind = I_PHASE; a.cq = p.cq; a.m[0] = p.m[0];
      b.kind = I_PHASE; b.cq = p.cq; b.cq.push_back(p.tq[0]); b.m[0] = p.m[3] / p.m[0];
      if (a.m[0] != 1.0) out.push_back(a);
      if (b.m[0] != 1.0) out.push_back(b);
      continue;
    }
    out.push_back(std::move(p));
  }
  return out;
}

// --------------------------------------- two-qubit Cartan split (FP64) --
// A dense U(4) costs 16 FMA per amplitude.  Its Cartan (KAK) form
//   U = (A1 (x) A0) . N . (B1 (x) B0),   N = exp(i(a XX + b YY + c ZZ))
// replaces it by four single-qubit gates, which fuse with their neighbours,
// and N, which only mixes |00> with |11> and |01> with |10>: a real rotation
// in each of the two subspaces (one FMA per amplitude component in scaled
// form) between two-qubit diagonals that merge into the diagonal tables.
// Method (Kraus & Cirac, PRA 63, 062309; Vatan & Williams, PRA 69, 032315):
// in the magic basis Q local gates are real orthogonal and N is diagonal,
// so with V = Q^dag U' Q (U' = U / det(U)^(1/4)) the symmetric unitary
// V^T V = O D O^T has a real orthogonal eigenbasis O, V = K1 D^(1/2) O^T with
// K1 real orthogonal, and A = Q K1 Q^dag, N = Q D^(1/2) Q^dag, B = Q O^T Q^dag.
// Every result is recomposed and compared with U; any failure keeps U dense.
namespace kak {

using C4 = std::array<cd, 16>;  // row-major 4x4, index = bit0 + 2 bit1

C4 mul(const C4& A, const C4& B) {
  C4 R{};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      cd s = 0;
      for (int k = 0; k < 4; ++k) s += A[4 * i + k] * B[4 * k + j];
      R[4 * i + j] = s;
    }
  return R;
}
C4 dag(const C4& A) {
  C4 R{};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) R[4 * i + j] = std::conj(A[4 * j + i]);
  return R;
}
C4 transpose(const C4& A) {
  C4 R{};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) R[4 * i + j] = A[4 * j + i];
  return R;
}
double dist(const C4& A, const C4& B) {
  double m = 0;
  for (int i = 0; i < 16; ++i) m = std::max(m, std::abs(A[i] - B[i]));
  return m;
}

// Magic basis: columns (|00>+|11>)/sqrt2, i(|00>-|11>)/sqrt2,
// i(|01>+|10>)/sqrt2, (|01>-|10>)/sqrt2.
const C4& magic() {
  static const C4 Q = [] {
    const double r = 1.0 / std::sqrt(2.0);
    const cd I(0, 1);
    C4 q{};
    q[4 * 0 + 0] = r;  q[4 * 3 + 0] = r;
    q[4 * 0 + 1] = I * r; q[4 * 3 + 1] = -I * r;
    q[4 * 1 + 2] = I * r; q[4 * 2 + 2] = I * r;
    q[4 * 1 + 3] = r;  q[4 * 2 + 3] = -r;
    return q;
  }();
  return Q;
}

// Cyclic Jacobi eigen-decomposition of a real symmetric 4x4 (A = V diag V^T).
void jacobi4(double A[4][4], double V[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) V[i][j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0;
    for (int p = 0; p < 4; ++p)
      for (int q = p + 1; q < 4; ++q) off += A[p][q] * A[p][q];
    if (off < 1e-30) return;
    for (int p = 0; p < 4; ++p)
      for (int q = p + 1; q < 4; ++q) {
        if (std::abs(A[p][q]) < 1e-300) continue;
        const double th = (A[q][q] - A[p][p]) / (2 * A[p][q]);
        const double t = (th >= 0 ? 1.0 : -1.0) / (std::abs(th) + std::sqrt(th * th + 1));
        const double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < 4; ++k) {  // A <- J^T A J
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 4; ++k) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 4; ++k) {
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
}

// L = X (x) Y (X on bit 1, Y on bit 0) -> X, Y; false if L is not a product.
bool split_local(const C4& L, cd X[4], cd Y[4]) {
  int bi = 0, bj = 0;
  double best = -1;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      double nrm = 0;
      for (int k = 0; k < 2; ++k)
        for (int l = 0; l < 2; ++l) nrm += std::norm(L[4 * (2 * i + k) + (2 * j + l)]);
      if (nrm > best) { best = nrm; bi = i; bj = j; }
    }
  // Y = block (bi, bj) scaled to a unitary; X[i][j] = <block(i,j), Y>/2
  const double sc = std::sqrt(best / 2.0);
  if (sc < 1e-6) return false;
  for (int k = 0; k < 2; ++k)
    for (int l = 0; l < 2; ++l) Y[2 * k + l] = L[4 * (2 * bi + k) + (2 * bj + l)] / sc;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      cd s = 0;
      for (int k = 0; k < 2; ++k)
        for (int l = 0; l < 2; ++l) s += std::conj(Y[2 * k + l]) * L[4 * (2 * i + k) + (2 * j + l)];
      X[2 * i + j] = s / 2.0;
    }
  C4 R{};
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int k = 0; k < 2; ++k)
        for (int l = 0; l < 2; ++l) R[4 * (2 * i + k) + (2 * j + l)] = X[2 * i + j] * Y[2 * k + l];
  return dist(R, L) < 1e-10;
}

C4 kron(const cd X[4], const cd Y[4]) {
  C4 R{};
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int k = 0; k < 2; ++k)
        for (int l = 0; l < 2; ++l) R[4 * (2 * i + k) + (2 * j + l)] = X[2 * i + j] * Y[2 * k + l];
  return R;
}

// U = (A1 (x) A0) N (B1 (x) B0) with N in span{I, XX, YY, ZZ}; false when the
// split does not reproduce U to 1e-10.
bool decompose(const cd* Uin, cd A0[4], cd A1[4], cd B0[4], cd B1[4], C4& N) {
  C4 U;
  for (int i = 0; i < 16; ++i) U[i] = Uin[i];
  // det(U) by Gaussian elimination with partial pivoting
  C4 T = U;
  cd det = 1;
  for (int c = 0; c < 4; ++c) {
    int p = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::abs(T[4 * r + c]) > std::abs(T[4 * p + c])) p = r;
    if (std::abs(T[4 * p + c]) < 1e-12) return false;
    if (p != c) {
      for (int k = 0; k < 4; ++k) std::swap(T[4 * p + k], T[4 * c + k]);
      det = -det;
    }
    det *= T[4 * c + c];
    for (int r = c + 1; r < 4; ++r) {
      const cd f = T[4 * r + c] / T[4 * c + c];
      for (int k = c; k < 4; ++k) T[4 * r + k] -= f * T[4 * c + k];
    }
  }
  const cd root = std::pow(det, 0.25);
  C4 Us;
  for (int i = 0; i < 16; ++i) Us[i] = U[i] / root;
  const C4& Q = magic();
  const C4 V = mul(dag(Q), mul(Us, Q));
  const C4 P = mul(transpose(V), V);
  double O[4][4];
  bool ok = false;
  for (double r : {0.5772156649015329, 1.4142135623730951, 2.718281828459045, 0.3183098861837907}) {
    double A[4][4];
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) A[i][j] = P[4 * i + j].real() + r * P[4 * i + j].imag();
    jacobi4(A, O);
    // O^T P O must be diagonal
    ok = true;
    for (int i = 0; i < 4 && ok; ++i)
      for (int j = 0; j < 4 && ok; ++j) {
        if (i == j) continue;
        cd s = 0;
        for (int k = 0; k < 4; ++k)
          for (int l = 0; l < 4; ++l) s += O[k][i] * P[4 * k + l] * O[l][j];
        if (std::abs(s) > 1e-9) ok = false;
      }
    if (ok) break;
  }
  if (!ok) return false;
  // det(O) = +1
  {
    double M[4][4];
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) M[i][j] = O[i][j];
    double d = 1;
    for (int c = 0; c < 4; ++c) {
      int p = c;
      for (int r = c + 1; r < 4; ++r)
        if (std::abs(M[r][c]) > std::abs(M[p][c])) p = r;
      if (p != c) { for (int k = 0; k < 4; ++k) std::swap(M[p][k], M[c][k]); d = -d; }
      d *= M[c][c];
      if (std::abs(M[c][c]) < 1e-300) return false;
      for (int r = c + 1; r < 4; ++r) {
        const double f = M[r][c] / M[c][c];
        for (int k = c; k < 4; ++k) M[r][k] -= f * M[c][k];
      }
    }
    if (d < 0)
      for (int i = 0; i < 4; ++i) O[i][0] = -O[i][0];
  }
  cd dh[4];  // square roots of the eigenvalues of P
  for (int i = 0; i < 4; ++i) {
    cd s = 0;
    for (int k = 0; k < 4; ++k)
      for (int l = 0; l < 4; ++l) s += O[k][i] * P[4 * k + l] * O[l][i];
    dh[i] = std::sqrt(s);
  }
  auto build_k1 = [&](C4& K1) {
    C4 VO{};
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        cd s = 0;
        for (int k = 0; k < 4; ++k) s += V[4 * i + k] * O[k][j];
        VO[4 * i + j] = s / dh[j];
      }
    K1 = VO;
  };
  C4 K1;
  build_k1(K1);
  // K1 is real orthogonal; make det(K1) = +1 by flipping one square root
  {
    double M[4][4];
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) M[i][j] = K1[4 * i + j].real();
    double d = 1;
    for (int c = 0; c < 4; ++c) {
      int p = c;
      for (int r = c + 1; r < 4; ++r)
        if (std::abs(M[r][c]) > std::abs(M[p][c])) p = r;
      if (p != c) { for (int k = 0; k < 4; ++k) std::swap(M[p][k], M[c][k]); d = -d; }
      d *= M[c][c];
      if (std::abs(M[c][c]) < 1e-300) return false;
      for (int r = c + 1; r < 4; ++r) {
        const double f = M[r][c] / M[c][c];
        for (int k = c; k < 4; ++k) M[r][k] -= f * M[c][k];
      }
    }
    if (d < 0) {
      dh[0] = -dh[0];
      build_k1(K1);
    }
  }
  C4 Dh{}, OT{};
  for (int i = 0; i < 4; ++i) Dh[4 * i + i] = dh[i];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) OT[4 * i + j] = O[j][i];
  const C4 La = mul(Q, mul(K1, dag(Q)));
  const C4 Lb = mul(Q, mul(OT, dag(Q)));
  N = mul(Q, mul(Dh, dag(Q)));
  if (!split_local(La, A1, A0) || !split_local(Lb, B1, B0)) return false;
  // N only couples |00>-|11> and |01>-|10>
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      const bool coupled = (i == j) || (i ^ j) == 3;
      if (!coupled && std::abs(N[4 * i + j]) > 1e-10) return false;
    }
  // global phase onto A0, then check the recomposition
  C4 R = mul(kron(A1, A0), mul(N, kron(B1, B0)));
  cd z = 0;
  for (int i = 0; i < 16; ++i) z += std::conj(R[i]) * U[i];
  z /= 4.0;
  if (std::abs(std::abs(z) - 1.0) > 1e-9) return false;
  for (int i = 0; i < 4; ++i) A0[i] *= z;
  R = mul(kron(A1, A0), mul(N, kron(B1, B0)));
  return dist(R, U) < 1e-10;
}

}  // namespace kak

// The Cartan split trades one dense op for several cheap ones: a win in
// specialised passes, a loss in the generic kernel, whose cost is per op.  The
// caller says whether the plan will be specialised; QSIM_KAK=0/1 overrides.
bool kak_enabled(bool specialised) {
  const char* e = std::getenv("QSIM_KAK");
  const int env = (e && *e) ? (e[0] == '0' ? 0 : 1) : -1;
  return env < 0 ? specialised : env == 1;
}

// 2x2 unitary V on (x, y) = diag(l0, l1) . [[c, -s], [s, c]] . diag(1, r1)
// with c, s >= 0 (the single-qubit factorisation of emit_1q).
void split_2x2(const cd V[4], cd& l0, cd& l1, double& c, double& s, cd& r1) {
  c = std::abs(V[0]);
  s = std::abs(V[2]);
  const double nrm = std::sqrt(c * c + s * s);
  if (s <= 1e-12 * nrm) {         // diagonal
    l0 = V[0]; l1 = V[3]; c = 1; s = 0; r1 = 1;
  } else if (c <= 1e-12 * nrm) {  // anti-diagonal
    l0 = 1; l1 = V[2]; c = 0; s = 1; r1 = -V[1];
  } else {
    l0 = V[0] / c; l1 = V[2] / s; r1 = -V[1] / (l0 * s);
    c /= nrm; s /= nrm;
  }
}

void permute_u2_bits(cd* m);

// Replaces uncontrolled dense two-qubit gates by their Cartan form (see
// namespace kak): B0, B1, diag, parity rotation (I_XRY), diag, A0, A1.
std::vector<IOp> kak_expand(const std::vector<IOp>& in, bool specialised) {
  if (!kak_enabled(specialised)) return in;
  std::vector<IOp> out;
  out.reserve(in.size() * 4);
  for (const IOp& o : in) {
    if (o.kind != I_U2 || !o.cq.empty()) { out.push_back(o); continue; }
    IOp u = o;
    if (u.tq[0] > u.tq[1]) {  // bit0 = the lower qubit
      std::swap(u.tq[0], u.tq[1]);
      permute_u2_bits(u.m);
    }
    cd A0[4], A1[4], B0[4], B1[4];
    kak::C4 N;
    if (!kak::decompose(u.m, A0, A1, B0, B1, N)) { out.push_back(o); continue; }
    const int qa = u.tq[0], qb = u.tq[1];
    // subspaces of N: even (x, y) = (|00>, |11>) = indices (0, 3);
    // odd (x, y) = (qa=0 qb=1, qa=1 qb=0) = indices (2, 1)
    const cd Ve[4] = {N[0], N[3], N[12], N[15]};
    const cd Vo[4] = {N[10], N[9], N[6], N[5]};
    cd le0, le1, re1, lo0, lo1, ro1;
    double ce, se, co, so;
    split_2x2(Ve, le0, le1, ce, se, re1);
    split_2x2(Vo, lo0, lo1, co, so, ro1);
    auto one = [&](int q, const cd* M) {
      IOp g;
      g.kind = I_U1; g.tq[0] = q; g.ntq = 1;
      for (int i = 0; i < 4; ++i) g.m[i] = M[i];
      out.push_back(g);
    };
    auto diag2 = [&](cd d0, cd d1, cd d2, cd d3) {  // index = bit(qa) + 2 bit(qb)
      IOp g;
      g.kind = I_DIAG2; g.dq[0] = qa; g.dq[1] = qb; g.ndq = 2;
      g.m[0] = d0; g.m[1] = d1; g.m[2] = d2; g.m[3] = d3;
      out.push_back(g);
    };
    one(qa, B0);
    one(qb, B1);
    if (se == 0.0 && so == 0.0) {  // N is diagonal
      diag2(le0, lo1 * ro1, lo0, le1 * re1);
    } else {
      diag2(1.0, ro1, 1.0, re1);
      // scaled rotation per subspace: (t, form) and the dropped factor
      auto scaled = [](double c, double s, double& t, double& form, double& f) {
        if (c >= s) { t = s / c; form = 0; f = c; } else { t = c / s; form = 1; f = s; }
      };
      double te, fe_form, fe, to, fo_form, fo;
      scaled(ce, se, te, fe_form, fe);
      scaled(co, so, to, fo_form, fo);
      IOp x;
      x.kind = I_XRY; x.tq[0] = qa; x.tq[1] = qb; x.ntq = 2;
      x.m[0] = cd(te, fe_form);
      x.m[1] = cd(to, fo_form);
      out.push_back(x);
      diag2(le0 * fe, lo1 * fo, lo0 * fo, le1 * fe);
    }
    one(qa, A0);
    one(qb, A1);
  }
  return out;
}

// ----------------------------------------------------- 1Q fusion (FP64) --
struct M2 { cd a[4]; };
M2 mul(const M2& A, const M2& B) {  // A*B
  M2 C;
  C.a[0] = A.a[0] * B.a[0] + A.a[1] * B.a[2];
  C.a[1] = A.a[0] * B.a[1] + A.a[1] * B.a[3];
  C.a[2] = A.a[2] * B.a[0] + A.a[3] * B.a[2];
  C.a[3] = A.a[2] * B.a[1] + A.a[3] * B.a[3];
  return C;
}

// Is `o` an uncontrolled single-qubit op?  Then return its 2x2 matrix.
bool as_1q(const IOp& o, int& q, M2& M) {
  switch (o.kind) {
    case I_U1:
      if (!o.cq.empty()) return false;
      q = o.tq[0]; for (int i = 0; i < 4; ++i) M.a[i] = o.m[i]; return true;
    case I_X:
      if (!o.cq.empty()) return false;
      q = o.tq[0]; M.a[0] = 0; M.a[1] = 1; M.a[2] = 1; M.a[3] = 0; return true;
    case I_Y:
      q = o.tq[0]; M.a[0] = 0; M.a[1] = cd(0, -1); M.a[2] = cd(0, 1); M.a[3] = 0; return true;
    case I_DIAG1:
      q = o.dq[0]; M.a[0] = o.m[0]; M.a[1] = 0; M.a[2] = 0; M.a[3] = o.m[1]; return true;
    case I_NEG: case I_PHASE:
      if (o.cq.size() != 1) return false;
      q = o.cq[0]; M.a[0] = 1; M.a[1] = 0; M.a[2] = 0; M.a[3] = o.m[0];
      if (o.kind == I_NEG) M.a[3] = -1.0;
      return true;
    default:
      return false;
  }
}

IOp diag_op(int q, cd d0, cd d1) {
  IOp p;
  if (d0 == 1.0) {
    p.kind = (d1 == -1.0) ? I_NEG : I_PHASE;
    p.cq = {q};
    p.m[0] = d1;
    return p;
  }
  p.kind = I_DIAG1; p.dq[0] = q; p.ndq = 1; p.m[0] = d0; p.m[1] = d1;
  return p;
}

// Emits the fused single-qubit matrix M on q.  Dense matrices become
// D_L * R(c, s) * D_R with R = [[c, -s], [s, c]] real (4 FMA per amplitude
// instead of 8) and D_L, D_R diagonal; the diagonals are later merged with
// neighbouring diagonal gates into one table op per register block.
//   c = |M00|, s = |M10|, D_R = diag(1, r1), D_L = diag(M00/c, M10/s),
//   r1 = -M01 / (l0 s)            (exact factorisation of a unitary M)
void emit_1q(int q, const M2& M, std::vector<IOp>& out, bool decompose) {
  const bool diag = (M.a[1] == 0.0 && M.a[2] == 0.0);
  if (diag) {
    if (M.a[0] == 1.0 && M.a[3] == 1.0) return;
    out.push_back(diag_op(q, M.a[0], M.a[3]));
    return;
  }
  if (M.a[0] == 0.0 && M.a[3] == 0.0 && M.a[1] == 1.0 && M.a[2] == 1.0) {
    IOp p;
    p.kind = I_X; p.tq[0] = q; p.ntq = 1;
    out.push_back(p);
    return;
  }
  const double c = std::abs(M.a[0]), sn = std::abs(M.a[2]);
  if (decompose && c > 1e-9 && sn > 1e-9) {
    const cd l0 = M.a[0] / c, l1 = M.a[2] / sn, r1 = -M.a[1] / (l0 * sn);
    if (r1 != 1.0) out.push_back(diag_op(q, 1.0, r1));
    IOp r;
    r.kind = I_RY; r.tq[0] = q; r.ntq = 1;
    const double nrm = std::sqrt(c * c + sn * sn);
    r.m[0] = cd(c / nrm, sn / nrm);
    out.push_back(r);
    if (!(l0 == 1.0 && l1 == 1.0)) out.push_back(diag_op(q, l0, l1));
    return;
  }
  IOp p;
  p.kind = I_U1; p.tq[0] = q; p.ntq = 1;
  for (int i = 0; i < 4; ++i) p.m[i] = M.a[i];
  out.push_back(p);
}

void qubits_of(const IOp& o, std::vector<int>& qs) {
  qs.clear();
  for (int i = 0; i < o.ntq; ++i) qs.push_back(o.tq[i]);
  for (int i = 0; i < o.ndq; ++i) qs.push_back(o.dq[i]);
  for (int c : o.cq) qs.push_back(c);
}

// Reorders a register block's ops into layers: as many uncontrolled
// single-qubit rotations / dense 2x2s on distinct qubits as are ready, then
// every ready diagonal, then the next layer, and so on (two ops keep their
// order when they share a qubit and are not both diagonal).  The encoder
// turns each layer into one Kronecker op and each diagonal run into one
// table, so maximal layers mean fewer table multiplies per amplitude.  Any
// other op (two-target, controlled) is placed as soon as nothing of the
// current layer or run is ready.
void layer_block_ops(const std::vector<IOp>& ops, std::vector<int>& idx) {
  const int m = (int)idx.size();
  if (m < 3) return;
  std::vector<uint64_t> qm(m, 0);
  std::vector<char> dg(m, 0), kr(m, 0);
  std::vector<int> qs;
  for (int i = 0; i < m; ++i) {
    const IOp& o = ops[idx[i]];
    qubits_of(o, qs);
    for (int q : qs) qm[i] |= 1ull << q;
    dg[i] = is_diag_kind(o.kind);
    kr[i] = (o.kind == I_RY || o.kind == I_U1) && o.cq.empty();
  }
  std::vector<int> indeg(m, 0);
  std::vector<std::vector<int>> succ(m);
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < j; ++i)
      if ((qm[i] & qm[j]) && !(dg[i] && dg[j])) {
        succ[i].push_back(j);
        ++indeg[j];
      }
  std::vector<char> done(m, 0);
  std::vector<int> out;
  out.reserve(m);
  auto emit = [&](int i) {
    done[i] = 1;
    out.push_back(idx[i]);
    for (int s2 : succ[i]) --indeg[s2];
  };
  while ((int)out.size() < m) {
    bool any = false;
    // a layer of ready rotations on distinct qubits (taken in list order)
    uint64_t used = 0;
    for (int i = 0; i < m; ++i)
      if (!done[i] && indeg[i] == 0 && kr[i] && !(qm[i] & used)) {
        used |= qm[i];
        emit(i);
        any = true;
      }
    if (any) continue;
    // every ready diagonal
    for (int i = 0; i < m; ++i)
      if (!done[i] && indeg[i] == 0 && dg[i]) {
        emit(i);
        any = true;
      }
    if (any) continue;
    for (int i = 0; i < m; ++i)
      if (!done[i] && indeg[i] == 0) {
        emit(i);
        break;
      }
  }
  idx.swap(out);
}

std::vector<IOp> fuse_1q(int n, const std::vector<IOp>& in, bool decompose) {
  std::vector<IOp> out;
  std::vector<M2> pend(n);
  std::vector<char> has(n, 0);
  auto flush = [&](int q) {
    if (!has[q]) return;
    emit_1q(q, pend[q], out, decompose);
    has[q] = 0;
  };
  std::vector<int> qs;
  for (const IOp& o : in) {
    int q;
    M2 M;
    if (as_1q(o, q, M)) {
      pend[q] = has[q] ? mul(M, pend[q]) : M;
      has[q] = 1;
      continue;
    }
    qubits_of(o, qs);
    for (int x : qs) flush(x);
    out.push_back(o);
  }
  for (int q = 0; q < n; ++q) flush(q);
  return out;
}

// Reorders the op list into alternating runs: every dense op that is ready
// (all ops it does not commute with already emitted) goes first; when none is
// ready, every ready diagonal op is emitted as one run.  Two ops commute when
// each shared qubit is used in a diagonal role (control, phase, diagonal) by
// both.  In a layered circuit this yields: all rotations of a layer, then one
// run with every diagonal between it and the next layer, which the encoder
// merges into a single table op per register block.
std::vector<IOp> schedule_runs(int n, const std::vector<IOp>& in) {
  const int m = (int)in.size();
  std::vector<std::vector<int>> succ(m);
  std::vector<int> indeg(m, 0);
  std::vector<int> lastT(n, -1);
  std::vector<std::vector<int>> dset(n);
  auto edge = [&](int a, int b) {
    if (a < 0) return;
    succ[a].push_back(b);
    ++indeg[b];
  };
  for (int b = 0; b < m; ++b) {
    const IOp& o = in[b];
    uint64_t tm = 0;
    for (int i = 0; i < o.ntq; ++i) tm |= 1ull << o.tq[i];
    std::vector<int> qs;
    qubits_of(o, qs);
    std::sort(qs.begin(), qs.end());
    qs.erase(std::unique(qs.begin(), qs.end()), qs.end());
    for (int q : qs) {
      if ((tm >> q) & 1ull) {
        edge(lastT[q], b);
        for (int d : dset[q]) edge(d, b);
        lastT[q] = b;
        dset[q].clear();
      } else {
        edge(lastT[q], b);
        dset[q].push_back(b);
      }
    }
  }
  // duplicate edges only inflate indeg consistently (each is decremented once)
  std::vector<IOp> out;
  out.reserve(m);
  std::vector<int> ready_dense, ready_diag;
  for (int b = 0; b < m; ++b)
    if (indeg[b] == 0) (is_diag_kind(in[b].kind) ? ready_diag : ready_dense).push_back(b);
  auto release = [&](int b) {
    for (int s2 : succ[b])
      if (--indeg[s2] == 0) (is_diag_kind(in[s2].kind) ? ready_diag : ready_dense).push_back(s2);
  };
  while (!ready_dense.empty() || !ready_diag.empty()) {
    if (!ready_dense.empty()) {
      // keep program order among the ready dense ops
      std::sort(ready_dense.begin(), ready_dense.end());
      std::vector<int> batch;
      batch.swap(ready_dense);
      for (int b : batch) { out.push_back(in[b]); release(b); }
      continue;
    }
    std::sort(ready_diag.begin(), ready_diag.end());
    std::vector<int> batch;
    batch.swap(ready_diag);
    for (int b : batch) { out.push_back(in[b]); release(b); }
  }
  if ((int)out.size() != m) throw qs_error(QS_ERR_INVALID, "internal: op scheduling cycle");
  return out;
}

// --------------------------------------------------------- pass split ----
struct PassPlan {
  int T;
  std::vector<int> S;        // tile qubits ascending
  std::vector<int> ops;      // indices into the fused op list, in order
};

std::vector<PassPlan> split_passes(int n, int T, const std::vector<IOp>& ops) {
  std::vector<PassPlan> passes;
  std::vector<int> remaining(ops.size());
  for (size_t i = 0; i < ops.size(); ++i) remaining[i] = (int)i;
  const int Lc = std::min(T, 4);  // low qubits always in the tile (coalescing)
  if (T >= n) {
    PassPlan p;
    p.T = n;
    for (int q = 0; q < n; ++q) p.S.push_back(q);
    p.ops = remaining;
    passes.push_back(std::move(p));
    return passes;
  }
  std::vector<char> inS(n), bT(n), bD(n);
  while (!remaining.empty()) {
    std::fill(inS.begin(), inS.end(), 0);
    std::fill(bT.begin(), bT.end(), 0);
    std::fill(bD.begin(), bD.end(), 0);
    int sz = 0;
    for (int q = 0; q < Lc; ++q) { inS[q] = 1; ++sz; }
    PassPlan p;
    p.T = T;
    std::vector<int> left;
    for (int idx : remaining) {
      const IOp& o = ops[idx];
      bool blocked = false;
      for (int i = 0; i < o.ntq && !blocked; ++i) blocked = bT[o.tq[i]] || bD[o.tq[i]];
      for (int i = 0; i < o.ndq && !blocked; ++i) blocked = bT[o.dq[i]];
      for (size_t i = 0; i < o.cq.size() && !blocked; ++i) blocked = bT[o.cq[i]];
      if (!blocked) {
        int need = 0;
        for (int i = 0; i < o.ntq; ++i) need += !inS[o.tq[i]];
        if (sz + need <= T) {
          for (int i = 0; i < o.ntq; ++i) if (!inS[o.tq[i]]) { inS[o.tq[i]] = 1; ++sz; }
          p.ops.push_back(idx);
          continue;
        }
        blocked = true;
      }
      for (int i = 0; i < o.ntq; ++i) bT[o.tq[i]] = 1;
      for (int i = 0; i < o.ndq; ++i) bD[o.dq[i]] = 1;
      for (int c : o.cq) bD[c] = 1;
      left.push_back(idx);
    }
    QS_CHECK_ARG(!p.ops.empty(), "planner made no progress (op wider than the tile?)");
    for (int q = 0; q < n && sz < T; ++q) if (!inS[q]) { inS[q] = 1; ++sz; }
    for (int q = 0; q < n; ++q) if (inS[q]) p.S.push_back(q);
    passes.push_back(std::move(p));
    remaining.swap(left);
  }
  return passes;
}

// ---------------------------------------------------------- encoding -----
inline size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

void permute_u2_bits(cd* m) {
  static const int perm[4] = {0, 2, 1, 3};
  cd r[16];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) r[4 * a + b] = m[4 * perm[a] + perm[b]];
  for (int i = 0; i < 16; ++i) m[i] = r[i];
}

// A diagonal op as a product of "all set" terms: multiply by w where every
// qubit of `mask` is 1 (mask 0: a constant).  DIAG1(q; d0, d1) = d0 * (d1/d0
// on q); DIAG2 likewise with the pair term d11 d00 / (d01 d10).
struct DTerm { uint64_t mask; cd w; };
thread_local int64_t g_dtab_stats[4] = {0, 0, 0, 0};  // tables, group, sign, cross terms

void diag_terms(const IOp& o, std::vector<DTerm>& t) {
  switch (o.kind) {
    case I_NEG: case I_PHASE: {
      uint64_t m = 0;
      for (int c : o.cq) m |= 1ull << c;
      t.push_back({m, o.kind == I_NEG ? cd(-1.0, 0.0) : o.m[0]});
      break;
    }
    case I_DIAG1: {
      const uint64_t a = 1ull << o.dq[0];
      t.push_back({0, o.m[0]});
      t.push_back({a, o.m[1] / o.m[0]});
      break;
    }
    case I_DIAG2: {
      const uint64_t a = 1ull << o.dq[0], b = 1ull << o.dq[1];
      t.push_back({0, o.m[0]});
      t.push_back({a, o.m[1] / o.m[0]});
      t.push_back({b, o.m[2] / o.m[0]});
      t.push_back({a | b, o.m[3] * o.m[0] / (o.m[1] * o.m[2])});
      break;
    }
    default:
      throw qs_error(QS_ERR_INVALID, "internal: not a diagonal op");
  }
}

// One DK_DTAB op (kernel layout, qs_pass.cu):
//   pool: [2^R table entries (if rc & 1)]
//         [t0 group terms:  (gmask lo, gmask hi) as raw bits, w]        2 float2 each
//         [t1 sign terms:   (regmask lo, hi), (gmask lo, gmask hi)]     2 float2 each
//         [d0 cross terms:  (regmask lo, hi), (gmask lo, gmask hi), w]  3 float2 each
// (regmask: bit j = register index j is affected; the high word is only
// non-zero for 6-qubit register blocks, which only specialised passes use)
// amplitude j of a group with global index gidx is multiplied by
//   T[j] * prod_{group terms, gidx has gmask} w * prod_{cross, j in regmask, gidx has gmask} w
// and negated where the XOR of the active sign terms' regmasks has bit j.
// `scale` is the pass's pending real factor (dropped by scaled rotations); it
// is folded into the table when the op has one (FP64, rounded once).
void encode_dtab(const std::vector<DTerm>& terms, const std::vector<int>& regq, int R,
                 std::vector<DevOp>& dops, std::vector<float>& coef, bool& need_g, double& scale) {
  uint64_t rmask_all = 0;
  for (int k = 0; k < R; ++k) rmask_all |= 1ull << regq[k];
  const int J = 1 << R;
  std::vector<cd> T(J, cd(1.0, 0.0));
  std::map<uint64_t, cd> gterm;
  std::vector<std::pair<uint64_t, uint64_t>> sterm;
  std::vector<std::tuple<uint64_t, uint64_t, cd>> xterm;
  auto regmask = [&](uint64_t m) {
    uint64_t rm = 0;
    for (int j = 0; j < J; ++j) {
      bool all = true;
      for (int k = 0; k < R; ++k)
        if (((m >> regq[k]) & 1ull) && !((j >> k) & 1)) all = false;
      if (all) rm |= 1ull << j;
    }
    return rm;
  };
  for (const DTerm& d : terms) {
    if (d.w == 1.0) continue;
    const uint64_t mr = d.mask & rmask_all, mg = d.mask & ~rmask_all;
    if (mg == 0) {
      const uint64_t rm = regmask(mr);
      for (int j = 0; j < J; ++j)
        if ((rm >> j) & 1ull) T[j] *= d.w;
    } else if (mr == 0) {
      auto it = gterm.find(mg);
      if (it == gterm.end()) gterm[mg] = d.w; else it->second *= d.w;
    } else if (d.w == -1.0) {
      sterm.push_back({regmask(mr), mg});
    } else {
      xterm.emplace_back(regmask(mr), mg, d.w);
    }
  }
  std::vector<std::pair<uint64_t, cd>> gl;
  for (auto& kv : gterm)
    if (kv.second != 1.0) gl.push_back(kv);
  bool table = false;
  for (int j = 0; j < J; ++j) table |= (T[j] != 1.0);
  if (!table && gl.empty() && sterm.empty() && xterm.empty()) return;  // identity
  if (table && scale != 1.0) {
    for (int j = 0; j < J; ++j) T[j] *= scale;
    scale = 1.0;
  }
  // split into several ops if a count would overflow its 8-bit field
  size_t gi = 0, si = 0, xi = 0;
  bool first = true;
  do {
    DevOp d;
    std::memset(&d, 0, sizeof(d));
    d.kind = DK_DTAB;
    const size_t ng = std::min<size_t>(gl.size() - gi, 255), ns = std::min<size_t>(sterm.size() - si, 255),
                 nx = std::min<size_t>(xterm.size() - xi, 255);
    d.t0 = (uint8_t)ng;
    d.t1 = (uint8_t)ns;
    d.d0 = (uint8_t)nx;
    d.rc = (first && table) ? 1 : 0;
    d.coef = (uint32_t)(coef.size() / 2);
    auto put = [&](cd v) { coef.push_back((float)v.real()); coef.push_back((float)v.imag()); };
    auto put_bits = [&](uint32_t a, uint32_t b) {
      float fa, fb;
      std::memcpy(&fa, &a, 4);
      std::memcpy(&fb, &b, 4);
      coef.push_back(fa);
      coef.push_back(fb);
    };
    if (d.rc)
      for (int j = 0; j < J; ++j) put(T[j]);
    for (size_t k = 0; k < ng; ++k, ++gi) {
      put_bits((uint32_t)gl[gi].first, (uint32_t)(gl[gi].first >> 32));
      put(gl[gi].second);
    }
    for (size_t k = 0; k < ns; ++k, ++si) {
      put_bits((uint32_t)sterm[si].first, (uint32_t)(sterm[si].first >> 32));
      put_bits((uint32_t)sterm[si].second, (uint32_t)(sterm[si].second >> 32));
    }
    for (size_t k = 0; k < nx; ++k, ++xi) {
      put_bits((uint32_t)std::get<0>(xterm[xi]), (uint32_t)(std::get<0>(xterm[xi]) >> 32));
      put_bits((uint32_t)std::get<1>(xterm[xi]), (uint32_t)(std::get<1>(xterm[xi]) >> 32));
      put(std::get<2>(xterm[xi]));
    }
    d.ncoef = 0;
    if (ng || ns || nx) need_g = true;
    g_dtab_stats[0] += 1; g_dtab_stats[1] += (int64_t)ng; g_dtab_stats[2] += (int64_t)ns; g_dtab_stats[3] += (int64_t)nx;
    dops.push_back(d);
    first = false;
  } while (gi < gl.size() || si < sterm.size() || xi < xterm.size());
}

thread_local int g_last_devops = 0;

void encode_pass(int n, const PassPlan& pp, const std::vector<IOp>& ops, std::vector<char>& blob,
                 uint32_t& pass_off, int& R_out, int& nblocks_out, int& has2_out, int& ncoef_out, int block_bits) {
  // QSIM_LAYER_BLOCKS=0 keeps each block's ops in the order they were taken
  static const bool layer_blocks = [] {
    const char* e = std::getenv("QSIM_LAYER_BLOCKS");
    return !(e && e[0] == '0');
  }();
  const int T = pp.T;
  const int R = std::min(block_bits, T);
  std::vector<int> tpos(n, -1);  // global qubit -> tile position
  for (int k = 0; k < T; ++k) tpos[pp.S[k]] = k;

  // Register blocks.  The pass's ops form a dependency graph (two ops depend
  // on each other when they share a qubit, unless both are diagonal).  Each
  // block starts empty and repeatedly takes, in circuit order, every ready
  // op that fits: diagonal ops always (they need no register position),
  // others when their targets fit in R tile positions with the block's.  A
  // block thus follows the light cone of its qubits instead of cutting the
  // op list into consecutive runs.
  struct Blk { std::vector<int> regs; std::vector<int> ops; };
  std::vector<Blk> blks;
  {
    const int m = (int)pp.ops.size();
    std::vector<std::vector<int>> succ(m);
    std::vector<int> indeg(m, 0);
    std::vector<uint64_t> qmask(m, 0);
    std::vector<char> diag(m, 0);
    std::vector<int> qs;
    for (int i = 0; i < m; ++i) {
      const IOp& o = ops[pp.ops[i]];
      qubits_of(o, qs);
      for (int q : qs) qmask[i] |= 1ull << q;
      diag[i] = is_diag_kind(o.kind);
      for (int k = 0; k < o.ntq; ++k)
        if (tpos[o.tq[k]] < 0) throw qs_error(QS_ERR_INVALID, "internal: pass target outside tile");
    }
    // last op seen on each qubit, split into the trailing diagonal group and
    // the last non-diagonal op, so edges stay O(ops * qubits)
    std::vector<int> last_nd(64, -1);
    std::vector<std::vector<int>> diag_since(64);
    for (int i = 0; i < m; ++i) {
      std::vector<int> preds;
      for (int q = 0; q < 64; ++q) {
        if (!((qmask[i] >> q) & 1ull)) continue;
        if (diag[i]) {
          if (last_nd[q] >= 0) preds.push_back(last_nd[q]);
        } else {
          if (last_nd[q] >= 0) preds.push_back(last_nd[q]);
          for (int d : diag_since[q]) preds.push_back(d);
        }
      }
      std::sort(preds.begin(), preds.end());
      preds.erase(std::unique(preds.begin(), preds.end()), preds.end());
      for (int pi : preds) { succ[pi].push_back(i); ++indeg[i]; }
      for (int q = 0; q < 64; ++q) {
        if (!((qmask[i] >> q) & 1ull)) continue;
        if (diag[i]) diag_since[q].push_back(i);
        else { last_nd[q] = i; diag_since[q].clear(); }
      }
    }
    std::set<int> ready;
    for (int i = 0; i < m; ++i)
      if (indeg[i] == 0) ready.insert(i);
    int placed = 0;
    while (placed < m) {
      Blk cur;
      bool took = true;
      while (took) {
        took = false;
        for (auto it = ready.begin(); it != ready.end(); ++it) {
          const int i = *it;
          const IOp& o = ops[pp.ops[i]];
          std::vector<int> need;
          for (int k = 0; k < o.ntq; ++k) {
            const int p = tpos[o.tq[k]];
            if (std::find(cur.regs.begin(), cur.regs.end(), p) == cur.regs.end()) need.push_back(p);
          }
          if ((int)(cur.regs.size() + need.size()) > R) continue;
          for (int p : need) cur.regs.push_back(p);
          cur.ops.push_back(pp.ops[i]);
          ready.erase(it);
          ++placed;
          for (int sidx : succ[i])
            if (--indeg[sidx] == 0) ready.insert(sidx);
          took = true;
          break;  // rescan from the earliest ready op
        }
      }
      if (cur.ops.empty()) throw qs_error(QS_ERR_INVALID, "internal: no op fits an empty register block");
      if (layer_blocks) layer_block_ops(ops, cur.ops);
      blks.push_back(cur);
    }
    if (blks.empty()) blks.push_back(Blk());
  }

  std::vector<DevBlock> dblocks;
  std::vector<DevOp> dops;
  std::vector<float> coef;  // float2 pool, re/im
  int has2 = 0;
  double pend_scale = 1.0;  // product of the factors dropped by scaled rotations
  auto emit_scale = [&]() {
    DevOp d;
    std::memset(&d, 0, sizeof(d));
    d.kind = DK_SCALE;
    d.ncoef = 1;
    d.coef = (uint32_t)(coef.size() / 2);
    coef.push_back((float)pend_scale);
    coef.push_back(0.f);
    dops.push_back(d);
    pend_scale = 1.0;
  };
  for (Blk& b : blks) {
    // pad to R positions with the lowest unused tile positions
    for (int p = 0; (int)b.regs.size() < R && p < T; ++p)
      if (std::find(b.regs.begin(), b.regs.end(), p) == b.regs.end()) b.regs.push_back(p);
    std::sort(b.regs.begin(), b.regs.end());
    std::vector<int> regq(R);
    for (int k = 0; k < R; ++k) regq[k] = pp.S[b.regs[k]];
    auto regidx = [&](int q) -> int {
      int p = tpos[q];
      if (p < 0) return -1;
      auto it = std::find(b.regs.begin(), b.regs.end(), p);
      return it == b.regs.end() ? -1 : (int)(it - b.regs.begin());
    };
    DevBlock db;
    std::memset(&db, 0, sizeof(db));
    for (int k = 0; k < R; ++k) db.pos[k] = (int8_t)b.regs[k];
    db.op_begin = (int32_t)dops.size();
    bool need_g = false;
    std::vector<DTerm> run;  // pending diagonal run
    auto flush_run = [&]() {
      if (run.empty()) return;
      encode_dtab(run, regq, R, dops, coef, need_g, pend_scale);
      run.clear();
    };
    // pending Kronecker layer: uncontrolled 1Q rotations / dense gates on
    // distinct register bits (they commute), emitted as one op
    std::vector<std::pair<int, IOp>> kron;  // (register bit, op)
    auto flush_kron = [&]() {
      if (kron.empty()) return;
      // rotations -> one DK_KRY (scaled form), dense 2x2s -> one DK_KU1;
      // they act on distinct register bits, so their order is free
      unsigned rmask = 0, umask = 0;
      std::vector<cd> rslot((size_t)R, cd(0.0, 0.0)), uslot((size_t)R * 4, cd(0.0, 0.0));
      for (int k = 0; k < R; ++k) { uslot[4 * k] = 1.0; uslot[4 * k + 3] = 1.0; }
      for (auto& kv : kron) {
        const IOp& g = kv.second;
        const int k = kv.first;
        if (g.kind == I_RY) {
          const double c = g.m[0].real(), sn = g.m[0].imag();  // both > 0
          if (c >= sn) { rslot[k] = cd(sn / c, 0.0); pend_scale *= c; }
          else { rslot[k] = cd(c / sn, 1.0); pend_scale *= sn; }
          rmask |= 1u << k;
        } else {
          for (int i = 0; i < 4; ++i) uslot[4 * k + i] = g.m[i];
          umask |= 1u << k;
        }
      }
      auto put_op = [&](DevKind kind, unsigned mask, const std::vector<cd>& slots) {
        DevOp d;
        std::memset(&d, 0, sizeof(d));
        d.kind = kind;
        d.t0 = (uint8_t)mask;
        d.coef = (uint32_t)(coef.size() / 2);
        for (const cd& v : slots) { coef.push_back((float)v.real()); coef.push_back((float)v.imag()); }
        d.ncoef = (uint8_t)slots.size();
        dops.push_back(d);
      };
      if (rmask) put_op(DK_KRY, rmask, rslot);
      if (umask) put_op(DK_KU1, umask, uslot);
      // keep intermediate amplitudes far from the FP32 range limits
      if (pend_scale < 0x1p-40) emit_scale();
      kron.clear();
    };
    for (int idx : b.ops) {
      IOp o = ops[idx];
      if (is_diag_kind(o.kind)) { flush_kron(); diag_terms(o, run); continue; }
      if ((o.kind == I_RY || o.kind == I_U1) && o.cq.empty()) {
        flush_run();
        const int k = regidx(o.tq[0]);
        bool clash = false;
        for (auto& kv : kron) clash |= (kv.first == k);
        if (clash) flush_kron();
        kron.push_back({k, o});
        continue;
      }
      flush_kron();
      flush_run();
      DevOp d;
      std::memset(&d, 0, sizeof(d));
      for (int c : o.cq) {
        int r = regidx(c);
        if (r >= 0) d.rc |= (uint8_t)(1u << r); else { d.gc |= 1ull << c; need_g = true; }
      }
      int ncoef = 0;
      switch (o.kind) {
        case I_U1: d.kind = DK_U1; d.t0 = (uint8_t)regidx(o.tq[0]); ncoef = 4; break;
        case I_RY: d.kind = DK_RY; d.t0 = (uint8_t)regidx(o.tq[0]); ncoef = 1; break;
        case I_U2: {
          int a = regidx(o.tq[0]), c = regidx(o.tq[1]);
          if (a > c) { std::swap(a, c); permute_u2_bits(o.m); }
          d.kind = (d.rc || d.gc) ? DK_CU2 : DK_U2; d.t0 = (uint8_t)a; d.t1 = (uint8_t)c; ncoef = 16;
          has2 = 1;
          break;
        }
        case I_X: d.kind = DK_X; d.t0 = (uint8_t)regidx(o.tq[0]); break;
        case I_Y: d.kind = DK_Y; d.t0 = (uint8_t)regidx(o.tq[0]); break;
        case I_SWAP: {
          int a = regidx(o.tq[0]), c = regidx(o.tq[1]);
          if (a > c) std::swap(a, c);
          d.kind = DK_SWAP; d.t0 = (uint8_t)a; d.t1 = (uint8_t)c;
          has2 = 1;
          break;
        }
        case I_XRY: {  // tq[0] < tq[1], and register order follows qubit order
          const int a = regidx(o.tq[0]), c = regidx(o.tq[1]);
          if (a >= c) throw qs_error(QS_ERR_INVALID, "internal: parity rotation bits out of order");
          d.kind = DK_XRY; d.t0 = (uint8_t)a; d.t1 = (uint8_t)c; ncoef = 2;
          has2 = 1;
          break;
        }
        default: throw qs_error(QS_ERR_INVALID, "internal: unexpected op kind in block");
      }
      d.ncoef = (uint8_t)ncoef;
      d.coef = (uint32_t)(coef.size() / 2);
      for (int i = 0; i < ncoef; ++i) {
        coef.push_back((float)o.m[i].real());
        coef.push_back((float)o.m[i].imag());
      }
      dops.push_back(d);
    }
    flush_kron();
    flush_run();
    if (&b == &blks.back() && pend_scale != 1.0) emit_scale();  // every amplitude gets it once
    db.op_end = (int32_t)dops.size();
    db.pos[7] = need_g ? 1 : 0;
    dblocks.push_back(db);
  }

  DevPass hdr;
  std::memset(&hdr, 0, sizeof(hdr));
  hdr.T = T;
  hdr.R = R;
  hdr.nblocks = (int32_t)dblocks.size();
  hdr.n_qubits = n;
  for (int k = 0; k < T; ++k) hdr.S[k] = pp.S[k];
  hdr.ncoef = (uint32_t)(coef.size() / 2);
  // 2: every op is an uncontrolled dense 4x4 (the interpreter then runs a
  // dispatch-free op loop; QSIM_DENSE_ONLY=0 turns that off)
  static const bool dense_only_on = [] {
    const char* e = std::getenv("QSIM_DENSE_ONLY");
    return !(e && e[0] == '0');
  }();
  if (has2 && dense_only_on && !dops.empty() &&
      std::all_of(dops.begin(), dops.end(), [](const DevOp& d) { return d.kind == DK_U2; }))
    has2 = 2;
  hdr.has2 = (uint32_t)has2;
  size_t off = align16(sizeof(DevPass));
  hdr.block_off = (uint32_t)off;
  off = align16(off + dblocks.size() * sizeof(DevBlock));
  hdr.op_off = (uint32_t)off;
  off = align16(off + dops.size() * sizeof(DevOp));
  hdr.coef_off = (uint32_t)off;
  off = align16(off + coef.size() * sizeof(float));
  hdr.bytes = (uint32_t)off;

  pass_off = (uint32_t)blob.size();
  blob.resize(blob.size() + off, 0);
  char* base = blob.data() + pass_off;
  std::memcpy(base, &hdr, sizeof(hdr));
  if (!dblocks.empty()) std::memcpy(base + hdr.block_off, dblocks.data(), dblocks.size() * sizeof(DevBlock));
  if (!dops.empty()) std::memcpy(base + hdr.op_off, dops.data(), dops.size() * sizeof(DevOp));
  if (!coef.empty()) std::memcpy(base + hdr.coef_off, coef.data(), coef.size() * sizeof(float));
  R_out = R;
  g_last_devops = (int)dops.size();
  nblocks_out = (int)dblocks.size();
  has2_out = has2;
  ncoef_out = (int)hdr.ncoef;
}

double op_flops(const IOp& o) {
  switch (o.kind) {
    case I_U1: return 16;
    case I_U2: return 32;
    case I_XRY: return 4;
    case I_RY: return o.cq.empty() ? 4 : 8;
    case I_PHASE: case I_DIAG1: case I_DIAG2: return 8;
    default: return 0;
  }
}

}  // namespace

void qs_build_plan(int n, const qs_op* ops, int nops, int tile_bits, qs_plan_s* plan, int block_bits,
                   bool specialised) {
  QS_CHECK_ARG(n >= 1 && n <= QS_MAX_QUBITS, "n_qubits out of range [1, 34]");
  QS_CHECK_ARG(nops >= 0 && (nops == 0 || ops != nullptr), "ops pointer is null");
  // register blocks: 5 qubits for specialised passes, 4 for the generic kernel
  // (fewer registers, higher occupancy: measured faster there)
  if (tile_bits == 0) tile_bits = 13;
  if (block_bits == 0) block_bits = specialised ? 5 : 4;
  QS_CHECK_ARG(block_bits >= 2 && block_bits <= (specialised ? 6 : 5),
               "block_bits must be in [2, 5] (6 only for specialised passes)");
  std::vector<IOp> norm = kak_expand(normalise(n, ops, nops), specialised);
  std::vector<IOp> fused = schedule_runs(n, fuse_1q(n, norm, true));
  int T = n <= 14 ? n : tile_bits;
  std::vector<PassPlan> passes = split_passes(n, T, fused);
  plan->n_qubits = n;
  plan->tile_bits = T;
  plan->blob.clear();
  plan->pass_offsets.clear();
  plan->pass_T.clear();
  plan->pass_R.clear();
  plan->pass_has2.clear();
  plan->pass_ncoef.clear();
  int nblocks_total = 0;
  int64_t devops_total = 0;
  double flops = 0;
  for (auto& o : fused) flops += op_flops(o);
  for (const PassPlan& pp : passes) {
    uint32_t off;
    int R, nb, h2, nc;
    encode_pass(n, pp, fused, plan->blob, off, R, nb, h2, nc, block_bits);
    plan->pass_offsets.push_back(off);
    plan->pass_T.push_back(pp.T);
    plan->pass_R.push_back(R);
    plan->pass_has2.push_back(h2);
    plan->pass_ncoef.push_back(nc);
    nblocks_total += nb;
    devops_total += g_last_devops;
  }
  qs_plan_info& I = plan->info;
  I.n_qubits = n;
  I.tile_bits = T;
  I.n_passes = (int32_t)passes.size();
  I.n_blocks = nblocks_total;
  I.n_ops_in = nops;
  I.n_ops_fused = (int64_t)fused.size();
  I.bytes_moved = (double)passes.size() * 16.0 * std::ldexp(1.0, n);
  I.flops = flops * std::ldexp(1.0, n);
  I.n_device_ops = devops_total;
  if (std::getenv("QSIM_PLAN_STATS"))
    std::fprintf(stderr, "qsim plan: n=%d passes=%d blocks=%d devops=%lld dtab=%lld gterms=%lld sterms=%lld xterms=%lld\n",
                 n, (int)passes.size(), nblocks_total, (long long)devops_total, (long long)g_dtab_stats[0],
                 (long long)g_dtab_stats[1], (long long)g_dtab_stats[2], (long long)g_dtab_stats[3]);
  for (auto& v : g_dtab_stats) v = 0;
}

// Stream-ordered allocation: creating or destroying a plan never
// synchronises the device (a plain cudaFree would wait for every stream).
void qs_plan_upload(qs_context* h, qs_plan_s* p) {
  p->device = h->device;
  if (p->blob.empty()) return;
  // Passes for the tensor cores get their block matrices (32 KiB each, built
  // on the device by k_block_mats) after the program, in the same allocation.
  const size_t np = p->pass_offsets.size();
  p->pass_mats.assign(np, -1);
  size_t n_mats = 0;
  for (size_t i = 0; i < np; ++i)
    if (qs_tc_pass(h, p->pass_T[i], p->pass_R[i], p->pass_has2[i])) {
      p->pass_mats[i] = (int64_t)n_mats;
      n_mats += (size_t)reinterpret_cast<const DevPass*>(p->blob.data() + p->pass_offsets[i])->nblocks;
    }
  constexpr size_t kMat = 8192;  // floats per block matrix
  const size_t moff = (p->blob.size() + 255) & ~size_t(255);
  QS_CUDA(cudaMallocAsync(&p->d_blob, moff + n_mats * kMat * sizeof(float), h->stream));
  QS_CUDA(cudaMemcpyAsync(p->d_blob, p->blob.data(), p->blob.size(), cudaMemcpyHostToDevice, h->stream));
  p->d_mats = n_mats ? reinterpret_cast<float*>(static_cast<char*>(p->d_blob) + moff) : nullptr;
  std::vector<TcMatJob> jobs;  // host temporary, alive until the synchronisation below
  if (n_mats) {
    for (size_t i = 0; i < np; ++i) {
      if (p->pass_mats[i] < 0) continue;
      const auto* dP = reinterpret_cast<const DevPass*>(static_cast<const char*>(p->d_blob) + p->pass_offsets[i]);
      const int nb = reinterpret_cast<const DevPass*>(p->blob.data() + p->pass_offsets[i])->nblocks;
      for (int b = 0; b < nb; ++b)
        jobs.push_back(TcMatJob{dP, (uint64_t)b, p->d_mats + ((size_t)p->pass_mats[i] + b) * kMat});
    }
    void* d_jobs = nullptr;
    QS_CUDA(cudaMallocAsync(&d_jobs, jobs.size() * sizeof(TcMatJob), h->stream));
    QS_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(TcMatJob), cudaMemcpyHostToDevice, h->stream));
    qs_launch_block_mats(h, h->stream, static_cast<const TcMatJob*>(d_jobs), (int)jobs.size());
    QS_CUDA(cudaFreeAsync(d_jobs, h->stream));
  }
  // The plan may be executed on another stream: make the program resident
  // before returning (this waits on the handle's stream only).
  QS_CUDA(cudaStreamSynchronize(h->stream));
  p->stream = h->stream;
}

void qs_plan_free_device(void* d, cudaStream_t stream) {
  if (d) cudaFreeAsync(d, stream);
}

void qs_plan_run(qs_context* h, qs_plan_s* p, void* state, bool from_zero, uint64_t n_states) {
  const int n = p->n_qubits;
  p->stream = h->stream;
  if (p->pass_offsets.empty()) {
    if (from_zero) QS_CHECK_ARG(qs_state_init_batched(h, state, (int)n_states, n) == QS_OK, h->err.c_str());
    return;
  }
  // Pass specialisation.  Mode 2 compiles every pass before the first
  // execution.  Mode 1 (tiered, plans on >= jit_min_qubits qubits) uses
  // cached kernels from the first execution, queues a background compile at
  // the second (the plan is being reused) and switches over when it is done.
  if (h->jit_mode == 2 && !p->jit_tried) {
    p->jit_tried = true;
    std::string why;
    if (!qs_jit_compile_plan(h, p, why)) {
      p->jit.clear();
      p->jit_err = why;
    }
  } else if (h->jit_mode == 1 && n >= h->jit_min_qubits) {
    qs_jit_tiered(h, p);
  }
  if (!p->jit_err.empty() && std::getenv("QSIM_JIT_VERBOSE")) {
    std::fprintf(stderr, "qsim: pass specialisation off: %s\n", p->jit_err.c_str());
    p->jit_err.clear();
  }
  p->info.n_jit_passes = (int32_t)p->jit.size();
  const bool use_jit = h->jit_mode != 0 && p->jit.size() == p->pass_offsets.size();
  for (size_t i = 0; i < p->pass_offsets.size(); ++i) {
    const int T = p->pass_T[i];
    const uint32_t flags = (from_zero && i == 0) ? PI_FROM_ZERO : 0u;
    if (i < p->pass_mats.size() && p->pass_mats[i] >= 0) {  // tensor cores take the pass
      const DevPass* dp = reinterpret_cast<const DevPass*>(static_cast<const char*>(p->d_blob) + p->pass_offsets[i]);
      qs_launch_pass_tc_single(h, state, dp, T, n_states << (n - T), flags, p->d_mats + (size_t)p->pass_mats[i] * 8192);
      continue;
    }
    if (use_jit) {
      qs_jit_launch(h, p, i, state, n_states << (n - T), flags);
      continue;
    }
    const DevPass* dp = reinterpret_cast<const DevPass*>(static_cast<const char*>(p->d_blob) + p->pass_offsets[i]);
    qs_launch_pass_single(h, state, dp, T, p->pass_R[i], n_states << (n - T), flags, p->pass_has2[i],
                          p->pass_ncoef[i]);
  }
}

// qs_run_circuit's plan cache: entries per handle, and the largest circuit kept.
constexpr size_t kRunCacheEntries = 16;
constexpr int kRunCacheMaxOps = 4096;

static uint64_t fnv1a(const void* data, size_t bytes, uint64_t seed) {
  const unsigned char* b = static_cast<const unsigned char*>(data);
  uint64_t x = 0xcbf29ce484222325ull ^ seed;
  for (size_t i = 0; i < bytes; ++i) x = (x ^ b[i]) * 0x100000001b3ull;
  return x;
}

// A cached plan last ran on plan->stream.  While that is the handle's stream
// the program is freed stream-ordered behind the runs.  Otherwise that stream
// may since have been destroyed: wait for the device, then free it on the
// handle's stream.
static void run_cache_free(qs_context* h, qs_plan_s* p) {
  if (p->stream != h->stream) {
    cudaDeviceSynchronize();
    p->stream = h->stream;
  }
  qs_plan_destroy(p);
}

void qs_run_cache_clear(qs_context* h) {
  for (auto& e : h->run_cache) run_cache_free(h, e.plan);
  h->run_cache.clear();
}

extern "C" {

int qs_plan_create(qs_handle_t h, int n, const qs_op* ops, int nops, qs_plan_t* out) {
  QS_REQUIRE_HANDLE(h);
  qs_plan_s* p = nullptr;
  QS_API_BEGIN
  QS_CHECK_ARG(out != nullptr, "out is null");
  *out = nullptr;
  p = new qs_plan_s();
  int tb = 0, bb = 0;
  qs_circuit_shape(h, n, ops, nops, h->jit_mode == 2, tb, bb);
  qs_build_plan(n, ops, nops, tb, p, bb, h->jit_mode == 2);
  qs_plan_upload(h, p);
  *out = p;
  p = nullptr;
  return QS_OK;
  }
  catch (const qs_error& e) {
    h->err = e.what();
    if (p) { qs_plan_free_device(p->d_blob, h->stream); delete p; }
    return e.code;
  }
  catch (const std::exception& e) {
    h->err = e.what();
    if (p) { qs_plan_free_device(p->d_blob, h->stream); delete p; }
    return QS_ERR_INVALID;
  }
}

int qs_plan_analyze(int n, const qs_op* ops, int nops, int tile_bits, qs_plan_info* info) {
  qs_context* h = nullptr;
  QS_API_BEGIN
  QS_CHECK_ARG(info != nullptr, "info is null");
  if (tile_bits == 0) tile_bits = 13;
  QS_CHECK_ARG(tile_bits >= 10 && tile_bits <= 14, "tile_bits must be in [10, 14]");
  qs_plan_s p;
  qs_build_plan(n, ops, nops, tile_bits, &p);
  *info = p.info;
  QS_API_END(h)
}

int qs_plan_program(int n, const qs_op* ops, int nops, int tile_bits, int block_bits, int specialised, void* out,
                    size_t cap, size_t* needed) {
  qs_context* h = nullptr;
  QS_API_BEGIN
  QS_CHECK_ARG(needed != nullptr, "needed is null");
  if (tile_bits == 0) tile_bits = 13;
  QS_CHECK_ARG(tile_bits >= 10 && tile_bits <= 14, "tile_bits must be in [10, 14]");
  QS_CHECK_ARG(block_bits >= 0 && block_bits <= 6 && block_bits != 1, "block_bits must be 0 (auto) or in [2, 6]");
  qs_plan_s p;
  qs_build_plan(n, ops, nops, tile_bits, &p, block_bits, specialised != 0);
  *needed = p.blob.size();
  if (out && cap >= p.blob.size() && !p.blob.empty()) std::memcpy(out, p.blob.data(), p.blob.size());
  QS_API_END(h)
}

int qs_plan_jit_check(int n, const qs_op* ops, int nops, int tile_bits, int block_bits, int* n_passes) {
  qs_context* h = nullptr;
  QS_API_BEGIN
  if (tile_bits == 0) tile_bits = 13;
  QS_CHECK_ARG(tile_bits >= 10 && tile_bits <= 14, "tile_bits must be in [10, 14]");
  QS_CHECK_ARG(block_bits >= 0 && block_bits <= 6 && block_bits != 1, "block_bits must be 0 (auto) or in [2, 6]");
  qs_plan_s p;
  qs_build_plan(n, ops, nops, tile_bits, &p, block_bits, true);
  std::string err;
  if (!qs_jit_compile_only(&p, err)) throw qs_error(QS_ERR_INVALID, "pass specialisation: " + err);
  if (n_passes) *n_passes = (int)p.pass_offsets.size();
  QS_API_END(h)
}

int qs_plan_info_get(qs_plan_t plan, qs_plan_info* info) {
  if (!plan || !info) { qs_set_tls_error("null plan or info"); return QS_ERR_INVALID; }
  *info = plan->info;
  return QS_OK;
}

int qs_plan_execute(qs_handle_t h, qs_plan_t plan, void* state) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(plan != nullptr, "plan is null");
  qs_check_state(state, plan->n_qubits);
  QS_CHECK_ARG(plan->device == h->device, "plan was built for another device");
  qs_plan_run(h, plan, state, false, 1);
  QS_API_END(h)
}

int qs_plan_execute_from_zero(qs_handle_t h, qs_plan_t plan, void* state) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(plan != nullptr, "plan is null");
  qs_check_state(state, plan->n_qubits);
  QS_CHECK_ARG(plan->device == h->device, "plan was built for another device");
  qs_plan_run(h, plan, state, true, 1);
  QS_API_END(h)
}

int qs_plan_destroy(qs_plan_t plan) {
  if (!plan) return QS_OK;
  qs_plan_free_device(plan->d_blob, plan->stream);
  delete plan;
  return QS_OK;
}

int qs_run_circuit(qs_handle_t h, void* state, int n, const qs_op* ops, int nops) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  QS_CHECK_ARG(nops >= 0 && (nops == 0 || ops), "ops pointer is null");
  // A circuit run again (the same op records, width and plan shape) on the
  // same stream reuses its plan: no planning and no program upload.  Entries
  // are keyed on the full records, so a hit runs exactly the plan a fresh
  // call would build, and every run of an entry is on one stream.
  int tb = 0, bb = 0;
  const int spec = h->jit_mode == 2 ? 1 : 0;
  qs_circuit_shape(h, n, ops, nops, spec != 0, tb, bb);
  const bool cacheable = nops <= kRunCacheMaxOps;
  const uint64_t key = cacheable ? fnv1a(ops, sizeof(qs_op) * (size_t)nops, (uint64_t)n * 0x100000001b3ull) : 0;
  auto& cache = h->run_cache;
  for (size_t i = 0; cacheable && i < cache.size(); ++i) {
    qs_context::RunEntry& e = cache[i];
    if (e.hash != key || e.n != n || e.tile_bits != tb || e.block_bits != bb || e.specialised != spec ||
        e.plan->stream != h->stream || (int)e.ops.size() != nops ||
        (nops && std::memcmp(e.ops.data(), ops, sizeof(qs_op) * (size_t)nops)))
      continue;
    qs_context::RunEntry hit = std::move(e);
    cache.erase(cache.begin() + (long)i);
    const int rc = qs_plan_execute(h, hit.plan, state);
    if (rc != QS_OK) {
      qs_plan_destroy(hit.plan);
      return rc;
    }
    cache.push_back(std::move(hit));
    return QS_OK;
  }
  qs_plan_t p = nullptr;
  int rc = qs_plan_create(h, n, ops, nops, &p);
  if (rc != QS_OK) return rc;
  rc = qs_plan_execute(h, p, state);
  if (rc != QS_OK || !cacheable) {
    // No wait: qs_plan_destroy frees the device program stream-ordered after
    // the queued passes.
    qs_plan_destroy(p);
    return rc;
  }
  if (cache.size() >= kRunCacheEntries) {
    run_cache_free(h, cache.front().plan);
    cache.erase(cache.begin());
  }
  cache.push_back(qs_context::RunEntry{key, n, tb, bb, spec, std::vector<qs_op>(ops, ops + nops), p});
  return QS_OK;
  QS_API_END(h)
}

int qs_apply_gates_fused(qs_handle_t h, void* state, int n, const float* gates, const int* targets, int ngates) {
  QS_REQUIRE_HANDLE(h);
  QS_API_BEGIN
  std::vector<qs_op> ops;
  QS_CHECK_ARG(ngates >= 0, "n_gates must be >= 0");
  QS_CHECK_ARG(ngates == 0 || (gates && targets), "gates/targets pointer is null");
  ops.resize(ngates);
  for (int g = 0; g < ngates; ++g) {
    qs_op& o = ops[g];
    std::memset(&o, 0, sizeof(o));
    o.kind = QS_OP_U1;
    o.nq = 1;
    o.q[0] = targets[g];
    o.param = -1;
    for (int i = 0; i < 8; ++i) o.m[i] = gates[8 * g + i];
  }
  return qs_run_circuit(h, state, n, ops.data(), ngates);
  QS_API_END(h)
}

}  // extern "C"

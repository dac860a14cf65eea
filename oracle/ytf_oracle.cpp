// ytf_oracle.cpp -- CPU FP64 restatement of YellowThinFilms' spectral Green's-function
// path (mode solve -> S-matrix cascade -> cavity transfer map -> source projection ->
// synthesis of G), used ONLY as the checker of the CUDA implementation.
//
// TEST INFRASTRUCTURE. Nothing in the product (libytf, the Python host package) links,
// loads or calls this file. Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg load it, through oracle/ytf_oracle.py.
//
// Every routine restates one reference function; each cites the reference file:line it
// follows (paths within the YellowThinFilms project). Arithmetic is std::complex<double>
// throughout, in the reference's operation order where that order is visible.
//
// Third-party arithmetic the reference reaches and that is not in its tree:
//   * LAPACK ZGEEVX (Julia 1.12 LinearAlgebra.eigen -> LAPACK.geevx!('B','N','V','N'),
//     then sorted by (real, imag)). The oracle calls LAPACK's own ZGEEVX through a
//     function pointer installed at load time (scipy's bundled LAPACK), so the general
//     mode solve is the same routine the reference calls.
//   * Bessels.jl 0.2.8 besselj0/besselj1/besselj(2,.): the oracle uses the C library's
//     j0/j1/jn (both are correctly rounded to a few ulp on the real axis).
//   * FastGaussQuadrature 1.3.0 gausslegendre: restated as Newton iteration on the
//     Legendre three-term recurrence in long double, rounded to double.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace ytfo {

typedef std::complex<double> cd;
static const cd I1(0.0, 1.0);
static const double PI = 3.14159265358979323846;

// ---------------------------------------------------------------------------------
// Small column-major matrices (StaticArrays SMatrix stand-ins)
// ---------------------------------------------------------------------------------
template <int R, int C>
struct Mt {
  cd v[R * C];
  Mt() { for (int i = 0; i < R * C; ++i) v[i] = cd(0.0, 0.0); }
  cd& operator()(int i, int j) { return v[i + R * j]; }
  const cd& operator()(int i, int j) const { return v[i + R * j]; }
};
typedef Mt<2, 2> M2;
typedef Mt<4, 4> M4;
typedef Mt<4, 2> M42;
typedef Mt<2, 4> M24;
typedef Mt<2, 3> M23;
typedef Mt<4, 3> M43;
typedef Mt<2, 1> V2;
typedef Mt<4, 1> V4;

template <int R, int K, int C>
static Mt<R, C> mul(const Mt<R, K>& a, const Mt<K, C>& b) {
  Mt<R, C> o;
  for (int i = 0; i < R; ++i)
    for (int j = 0; j < C; ++j) {
      cd s = a(i, 0) * b(0, j);
      for (int k = 1; k < K; ++k) s += a(i, k) * b(k, j);
      o(i, j) = s;
    }
  return o;
}
template <int R, int C>
static Mt<R, C> add(const Mt<R, C>& a, const Mt<R, C>& b) {
  Mt<R, C> o;
  for (int i = 0; i < R * C; ++i) o.v[i] = a.v[i] + b.v[i];
  return o;
}
template <int R, int C>
static Mt<R, C> sub(const Mt<R, C>& a, const Mt<R, C>& b) {
  Mt<R, C> o;
  for (int i = 0; i < R * C; ++i) o.v[i] = a.v[i] - b.v[i];
  return o;
}
template <int R, int C>
static Mt<R, C> neg(const Mt<R, C>& a) {
  Mt<R, C> o;
  for (int i = 0; i < R * C; ++i) o.v[i] = -a.v[i];
  return o;
}
// conjugate transpose
template <int R, int C>
static Mt<C, R> adj(const Mt<R, C>& a) {
  Mt<C, R> o;
  for (int i = 0; i < R; ++i)
    for (int j = 0; j < C; ++j) o(j, i) = std::conj(a(i, j));
  return o;
}
static M2 eye2() { M2 o; o(0, 0) = 1.0; o(1, 1) = 1.0; return o; }
static M4 eye4() { M4 o; for (int i = 0; i < 4; ++i) o(i, i) = 1.0; return o; }
// (I - A) with the UniformScaling convention: off-diagonal -A, diagonal 1 - A
static M2 i_minus(const M2& a) {
  M2 o;
  o(0, 0) = 1.0 - a(0, 0); o(1, 0) = -a(1, 0); o(0, 1) = -a(0, 1); o(1, 1) = 1.0 - a(1, 1);
  return o;
}
// diagonal (from a 2-vector) times matrix and matrix times diagonal
template <int C>
static Mt<2, C> dmul(const V2& d, const Mt<2, C>& a) {
  Mt<2, C> o;
  for (int j = 0; j < C; ++j) { o(0, j) = d.v[0] * a(0, j); o(1, j) = d.v[1] * a(1, j); }
  return o;
}
static M2 muld(const M2& a, const V2& d) {
  M2 o;
  for (int i = 0; i < 2; ++i) { o(i, 0) = a(i, 0) * d.v[0]; o(i, 1) = a(i, 1) * d.v[1]; }
  return o;
}

static inline bool isfinc(const cd& z) { return std::isfinite(z.real()) && std::isfinite(z.imag()); }
template <int R, int C>
static bool allfinite(const Mt<R, C>& a) {
  for (int i = 0; i < R * C; ++i) if (!isfinc(a.v[i])) return false;
  return true;
}

struct Singular : std::runtime_error { Singular() : std::runtime_error("singular") {} };
// Julia's eigen(::Matrix) refuses non-finite input (LAPACK's chkfinite raises ArgumentError)
// and raises LAPACKException when zgeevx fails; the per-node try/catch of
// build_cavity_transfer_1d/2d (mod_CavityTransfer.jl:249-251) catches neither, so either ends
// the whole build with that error. EigenError carries the message; the node loops record it
// and the build raises it once the loop is done (an exception must not leave an OpenMP region).
struct EigenError : std::runtime_error { using std::runtime_error::runtime_error; };

// 2x2 solve by Cramer's rule, column by column (StaticArrays `\` for a 2x2 system).
template <int C>
static Mt<2, C> solve2(const M2& a, const Mt<2, C>& b) {
  cd det = a(0, 0) * a(1, 1) - a(0, 1) * a(1, 0);
  Mt<2, C> o;
  for (int j = 0; j < C; ++j) {
    o(0, j) = (a(1, 1) * b(0, j) - a(0, 1) * b(1, j)) / det;
    o(1, j) = (a(0, 0) * b(1, j) - a(1, 0) * b(0, j)) / det;
  }
  return o;
}
static M2 inv2(const M2& a) { return solve2<2>(a, eye2()); }

// 4x4 solve by LU with partial pivoting (largest |a|), as StaticArrays' lu for 4x4.
// Throws Singular on an exactly zero pivot.
template <int C>
static Mt<4, C> solve4(const M4& A, const Mt<4, C>& B) {
  cd a[4][4];
  cd b[4][C];
  for (int i = 0; i < 4; ++i) {
    for (int j = 0; j < 4; ++j) a[i][j] = A(i, j);
    for (int j = 0; j < C; ++j) b[i][j] = B(i, j);
  }
  for (int k = 0; k < 4; ++k) {
    int p = k;
    double best = std::abs(a[k][k]);
    for (int i = k + 1; i < 4; ++i) {
      double v = std::abs(a[i][k]);
      if (v > best) { best = v; p = i; }
    }
    if (a[p][k] == cd(0.0, 0.0)) throw Singular();
    if (p != k) {
      for (int j = 0; j < 4; ++j) std::swap(a[p][j], a[k][j]);
      for (int j = 0; j < C; ++j) std::swap(b[p][j], b[k][j]);
    }
    cd inv = 1.0 / a[k][k];
    for (int i = k + 1; i < 4; ++i) {
      cd l = a[i][k] * inv;
      a[i][k] = l;
      for (int j = k + 1; j < 4; ++j) a[i][j] -= l * a[k][j];
      for (int j = 0; j < C; ++j) b[i][j] -= l * b[k][j];
    }
  }
  Mt<4, C> x;
  for (int j = 0; j < C; ++j)
    for (int i = 3; i >= 0; --i) {
      cd s = b[i][j];
      for (int k = i + 1; k < 4; ++k) s -= a[i][k] * x(k, j);
      x(i, j) = s / a[i][i];
    }
  return x;
}

// Column-pivoted Householder QR least-squares solve (fallback of the interface
// matrix, mod_ScatteringMatrix.jl:35-44: qr(LHS, ColumnNorm()) \ RHS), rank from
// the diagonal of R against eps * |R11| * n.
static M4 qr_solve4(const M4& A, const M4& B) {
  cd a[4][4], b[4][4];
  int perm[4] = {0, 1, 2, 3};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) { a[i][j] = A(i, j); b[i][j] = B(i, j); }
  for (int k = 0; k < 4; ++k) {
    int pc = k; double best = -1;
    for (int j = k; j < 4; ++j) {
      double s = 0; for (int i = k; i < 4; ++i) s += std::norm(a[i][j]);
      if (s > best) { best = s; pc = j; }
    }
    if (pc != k) { for (int i = 0; i < 4; ++i) std::swap(a[i][pc], a[i][k]); std::swap(perm[pc], perm[k]); }
    double nrm = 0; for (int i = k; i < 4; ++i) nrm += std::norm(a[i][k]);
    nrm = std::sqrt(nrm);
    if (nrm == 0) continue;
    cd alpha = a[k][k];
    cd ph = std::abs(alpha) > 0 ? alpha / std::abs(alpha) : cd(1, 0);
    cd v[4];
    for (int i = 0; i < 4; ++i) v[i] = 0;
    v[k] = alpha + ph * nrm;
    for (int i = k + 1; i < 4; ++i) v[i] = a[i][k];
    double vn = 0; for (int i = k; i < 4; ++i) vn += std::norm(v[i]);
    if (vn == 0) continue;
    for (int j = k; j < 4; ++j) {
      cd s = 0; for (int i = k; i < 4; ++i) s += std::conj(v[i]) * a[i][j];
      s *= 2.0 / vn;
      for (int i = k; i < 4; ++i) a[i][j] -= s * v[i];
    }
    for (int j = 0; j < 4; ++j) {
      cd s = 0; for (int i = k; i < 4; ++i) s += std::conj(v[i]) * b[i][j];
      s *= 2.0 / vn;
      for (int i = k; i < 4; ++i) b[i][j] -= s * v[i];
    }
  }
  double tol = std::numeric_limits<double>::epsilon() * 4 * std::abs(a[0][0]);
  int rank = 0;
  for (int k = 0; k < 4; ++k) if (std::abs(a[k][k]) > tol) rank = k + 1;
  M4 x;
  for (int j = 0; j < 4; ++j) {
    cd y[4] = {0, 0, 0, 0};
    for (int i = rank - 1; i >= 0; --i) {
      cd s = b[i][j];
      for (int k = i + 1; k < rank; ++k) s -= a[i][k] * y[k];
      y[i] = s / a[i][i];
    }
    for (int i = 0; i < 4; ++i) x(perm[i], j) = y[i];
  }
  return x;
}

// ---------------------------------------------------------------------------------
// LAPACK hook
// ---------------------------------------------------------------------------------
typedef void (*zgeevx_t)(char*, char*, char*, char*, int*, cd*, int*, cd*, cd*, int*, cd*, int*, int*,
                         int*, double*, double*, double*, double*, cd*, int*, double*, int*);
static zgeevx_t g_zgeevx = nullptr;

// ---------------------------------------------------------------------------------
// Materials and layers (mod_ModeSolver.jl:20-80)
// ---------------------------------------------------------------------------------
enum Kind { ISO = 0, UNI = 1, BIAX = 2, GEN = 3 };

struct Layer {
  int ekind, mkind;
  cd eps[9];  // column-major 3x3: eps[(i-1) + 3*(j-1)] = ϵ[i,j]
  cd mu[9];
  double d;
  cd E(int i, int j) const { return eps[(i - 1) + 3 * (j - 1)]; }
  cd U(int i, int j) const { return mu[(i - 1) + 3 * (j - 1)]; }
};
typedef std::vector<Layer> Stack;

// ---------------------------------------------------------------------------------
// Modes (mod_ModeSolver.jl:83-92)
// ---------------------------------------------------------------------------------
struct Modes {
  M42 Vf, Vb, Wf, Wb;
  V2 Qf, Qb;
};

// _berreman_core (mod_ModeSolver.jl:122-193)
static M4 berreman_core(const Layer& L, double w, double kx, double ky) {
  cd e11 = L.E(1, 1), e12 = L.E(1, 2), e21 = L.E(2, 1), e22 = L.E(2, 2);
  cd e13 = L.E(1, 3), e23 = L.E(2, 3), e31 = L.E(3, 1), e32 = L.E(3, 2), e33 = L.E(3, 3);
  cd m11 = L.U(1, 1), m12 = L.U(1, 2), m21 = L.U(2, 1), m22 = L.U(2, 2);
  cd m13 = L.U(1, 3), m23 = L.U(2, 3), m31 = L.U(3, 1), m32 = L.U(3, 2), m33 = L.U(3, 3);
  cd k1(kx, 0.0), k2(ky, 0.0);
  cd de = cd(1.0, 0.0) / e33;
  cd dm = cd(1.0, 0.0) / m33;
  cd iw = cd(1.0, 0.0) / w;
  cd ezt1 = e31, ezt2 = e32, mzt1 = m31, mzt2 = m32;
  cd Se11 = e11 - e13 * de * ezt1, Se12 = e12 - e13 * de * ezt2;
  cd Se21 = e21 - e23 * de * ezt1, Se22 = e22 - e23 * de * ezt2;
  cd Sm11 = m11 - m13 * dm * mzt1, Sm12 = m12 - m13 * dm * mzt2;
  cd Sm21 = m21 - m23 * dm * mzt1, Sm22 = m22 - m23 * dm * mzt2;
  cd re1 = de * ezt1, re2 = de * ezt2;
  cd se1 = e13 * de, se2 = e23 * de;
  cd rm1 = dm * mzt1, rm2 = dm * mzt2;
  cd sm1 = m13 * dm, sm2 = m23 * dm;
  cd t21 = -std::conj(k2), t22 = std::conj(k1);
  cd t31 = iw * k1, t32 = iw * k2;
  cd Rsm1 = sm2, Rsm2 = -sm1, Rse1 = se2, Rse2 = -se1;
  cd B11_11 = Rsm1 * t21 - k1 * re1, B11_12 = Rsm1 * t22 - k1 * re2;
  cd B11_21 = Rsm2 * t21 - k2 * re1, B11_22 = Rsm2 * t22 - k2 * re2;
  cd a11 = w * Sm21, a12 = w * Sm22, a21 = -w * Sm11, a22 = -w * Sm12;
  cd B12_11 = a11 - t31 * de * t21, B12_12 = a12 - t31 * de * t22;
  cd B12_21 = a21 - t32 * de * t21, B12_22 = a22 - t32 * de * t22;
  cd b11 = w * Se21, b12 = w * Se22, b21 = -w * Se11, b22 = -w * Se12;
  cd B21_11 = t31 * dm * t21 - b11, B21_12 = t31 * dm * t22 - b12;
  cd B21_21 = t32 * dm * t21 - b21, B21_22 = t32 * dm * t22 - b22;
  cd B22_11 = Rse1 * t21 - k1 * rm1, B22_12 = Rse1 * t22 - k1 * rm2;
  cd B22_21 = Rse2 * t21 - k2 * rm1, B22_22 = Rse2 * t22 - k2 * rm2;
  M4 B;
  B(0, 0) = B11_11; B(1, 0) = B11_21; B(2, 0) = B21_11; B(3, 0) = B21_21;
  B(0, 1) = B11_12; B(1, 1) = B11_22; B(2, 1) = B21_12; B(3, 1) = B21_22;
  B(0, 2) = B12_11; B(1, 2) = B12_21; B(2, 2) = B22_11; B(3, 2) = B22_21;
  B(0, 3) = B12_12; B(1, 3) = B12_22; B(2, 3) = B22_12; B(3, 3) = B22_22;
  return B;
}

// Julia eigen(B) for a general complex 4x4: LAPACK zgeevx('B','N','V','N'), then
// sortperm by (real, imag) (LinearAlgebra.eigsortby).
static void eigen4(const M4& B, cd Q[4], M4& V) {
  if (!g_zgeevx) throw std::runtime_error("oracle: LAPACK zgeevx not installed");
  for (int i = 0; i < 16; ++i)
    if (!isfinc(B.v[i])) throw EigenError("ArgumentError: matrix contains Infs or NaNs");
  cd a[16];
  for (int i = 0; i < 16; ++i) a[i] = B.v[i];
  char balanc = 'B', jobvl = 'N', jobvr = 'V', sense = 'N';
  int n = 4, lda = 4, ldvl = 1, ldvr = 4, ilo = 0, ihi = 0, info = 0, lwork = -1;
  cd w[4], vl[1], vr[16], wq;
  double scale[4], abnrm, rconde[4], rcondv[4], rwork[8];
  g_zgeevx(&balanc, &jobvl, &jobvr, &sense, &n, a, &lda, w, vl, &ldvl, vr, &ldvr, &ilo, &ihi, scale,
           &abnrm, rconde, rcondv, &wq, &lwork, rwork, &info);
  lwork = std::max(8, (int)wq.real());
  std::vector<cd> work(lwork);
  for (int i = 0; i < 16; ++i) a[i] = B.v[i];
  g_zgeevx(&balanc, &jobvl, &jobvr, &sense, &n, a, &lda, w, vl, &ldvl, vr, &ldvr, &ilo, &ihi, scale,
           &abnrm, rconde, rcondv, work.data(), &lwork, rwork, &info);
  if (info != 0) throw EigenError("LAPACKException(" + std::to_string(info) + ")");
  int p[4] = {0, 1, 2, 3};
  std::stable_sort(p, p + 4, [&](int x, int y) {
    if (w[x].real() != w[y].real()) return w[x].real() < w[y].real();
    return w[x].imag() < w[y].imag();
  });
  for (int j = 0; j < 4; ++j) {
    Q[j] = w[p[j]];
    for (int i = 0; i < 4; ++i) V(i, j) = vr[i + 4 * p[j]];
  }
}

static bool closed_form_layer(const Layer& L) { return (L.ekind == ISO || L.ekind == UNI) && L.mkind == ISO; }

// _eigen_QV closed form for iso/uniaxial ε with isotropic μ (mod_ModeSolver.jl:243-265)
static void eigen_qv_closed(const Layer& L, double w, double kx, double ky, cd Q[4], M4& V) {
  cd et = L.E(1, 1), ez = L.E(3, 3), mr = L.U(1, 1);
  cd wc(w, 0.0);
  double kr = std::hypot(kx, ky);
  double phi = kr == 0 ? 0.0 : std::atan2(ky, kx);
  double c = std::cos(phi), s = std::sin(phi);
  cd kzo = std::sqrt(wc * wc * et * mr - kr * kr);
  cd kze = std::sqrt(et * (wc * wc * mr - kr * kr / ez));
  cd A = 1.0 / (wc * mr);
  cd Bn = 1.0 / (wc * et);
  cd mA = -A;
  V(0, 0) = -s; V(1, 0) = c; V(2, 0) = mA * kzo * c; V(3, 0) = mA * kzo * s;
  V(0, 1) = -s; V(1, 1) = c; V(2, 1) = A * kzo * c; V(3, 1) = A * kzo * s;
  V(0, 2) = Bn * kze * c; V(1, 2) = Bn * kze * s; V(2, 2) = -s; V(3, 2) = c;
  cd mB = -Bn;
  V(0, 3) = mB * kze * c; V(1, 3) = mB * kze * s; V(2, 3) = -s; V(3, 3) = c;
  Q[0] = kzo; Q[1] = -kzo; Q[2] = kze; Q[3] = -kze;
}

// _modes_layer (mod_ModeSolver.jl:274-326). Returns false if the sort overflows a slot
// (the reference would raise a BoundsError there).
static bool modes_layer(const Layer& L, double w, double kx, double ky, Modes& out) {
  cd Q[4];
  M4 V;
  if (closed_form_layer(L)) eigen_qv_closed(L, w, kx, ky, Q, V);
  else eigen4(berreman_core(L, w, kx, ky), Q, V);
  M4 W;  // R4s * V: rows (V4, -V3, -V2, V1)
  for (int j = 0; j < 4; ++j) {
    W(0, j) = V(3, j); W(1, j) = -V(2, j); W(2, j) = -V(1, j); W(3, j) = V(0, j);
  }
  double Pz[4];
  for (int j = 0; j < 4; ++j) {
    cd s = std::conj(V(0, j)) * W(0, j);
    for (int i = 1; i < 4; ++i) s += std::conj(V(i, j)) * W(i, j);
    Pz[j] = 0.25 * s.real();
  }
  const double tol = std::sqrt(std::numeric_limits<double>::epsilon());
  Modes m;
  int idf = 0, idb = 0, ndeg = 0, deg[4];
  auto putf = [&](int j) {
    if (idf >= 2) return false;
    for (int i = 0; i < 4; ++i) { m.Vf(i, idf) = V(i, j); m.Wf(i, idf) = W(i, j); }
    m.Qf.v[idf] = Q[j]; ++idf; return true;
  };
  auto putb = [&](int j) {
    if (idb >= 2) return false;
    for (int i = 0; i < 4; ++i) { m.Vb(i, idb) = V(i, j); m.Wb(i, idb) = W(i, j); }
    m.Qb.v[idb] = Q[j]; ++idb; return true;
  };
  for (int j = 0; j < 4; ++j) {
    if (std::fabs(Pz[j]) > tol) {
      if (Pz[j] > 0) { if (!putf(j)) return false; }
      else { if (!putb(j)) return false; }
    } else if (std::fabs(Q[j].imag()) > tol) {
      if (Q[j].imag() > tol) { if (!putf(j)) return false; }
      else if (Q[j].imag() < -tol) { if (!putb(j)) return false; }
    } else {
      deg[ndeg++] = j;
    }
  }
  for (int i = 0; i < ndeg; ++i) {
    int j = deg[i];
    if (idf < 2) putf(j);
    else if (idb < 2) putb(j);
  }
  out = m;
  return true;
}

// _match_modes (mod_ModeSolver.jl:333-349), applied to one direction (V, W, Q)
static void match_modes(const M42& Wa, M42& Vb, M42& Wb, V2& Qb) {
  M2 C = mul(adj(Wa), Vb);
  double sid = std::norm(C(0, 0)) + std::norm(C(1, 1));
  double ssw = std::norm(C(0, 1)) + std::norm(C(1, 0));
  if (ssw > sid) {
    for (int i = 0; i < 4; ++i) { std::swap(Vb(i, 0), Vb(i, 1)); std::swap(Wb(i, 0), Wb(i, 1)); }
    std::swap(Qb.v[0], Qb.v[1]);
  }
}

// _modes_stack_core (mod_ModeSolver.jl:358-392)
static bool modes_stack(const Stack& st, double w, double kx, double ky, std::vector<Modes>& out) {
  int N = (int)st.size();
  out.resize(N);
  Modes m0;
  if (!modes_layer(st[0], w, kx, ky, m0)) return false;
  out[0] = m0;
  for (int j = 1; j < N; ++j) {
    Modes mj;
    if (!modes_layer(st[j], w, kx, ky, mj)) return false;
    match_modes(out[j - 1].Wf, mj.Vf, mj.Wf, mj.Qf);
    match_modes(out[j - 1].Wb, mj.Vb, mj.Wb, mj.Qb);
    out[j] = mj;
  }
  return true;
}

// _Rot4 / _rotate_modes (mod_ModeSolver.jl:471-482)
static Modes rotate_modes(const Modes& m, double phi) {
  double c = std::cos(phi), s = std::sin(phi);
  auto rot = [&](const M42& a) {
    M42 o;
    for (int j = 0; j < 2; ++j) {
      o(0, j) = c * a(0, j) - s * a(1, j);
      o(1, j) = s * a(0, j) + c * a(1, j);
      o(2, j) = c * a(2, j) - s * a(3, j);
      o(3, j) = s * a(2, j) + c * a(3, j);
    }
    return o;
  };
  Modes r;
  r.Vf = rot(m.Vf); r.Vb = rot(m.Vb); r.Wf = rot(m.Wf); r.Wb = rot(m.Wb);
  r.Qf = m.Qf; r.Qb = m.Qb;
  return r;
}

static bool azimuthally_symmetric(const Stack& st) {
  for (auto& L : st) if (!closed_form_layer(L)) return false;
  return true;
}

// ---------------------------------------------------------------------------------
// S-matrix (mod_ScatteringMatrix.jl)
// ---------------------------------------------------------------------------------
static M4 blk4(const M42& l, const M42& r) {
  M4 o;
  for (int i = 0; i < 4; ++i) { o(i, 0) = l(i, 0); o(i, 1) = l(i, 1); o(i, 2) = r(i, 0); o(i, 3) = r(i, 1); }
  return o;
}
// _S_Interface_Matrix (:27-47)
static M4 s_interface(const Modes& A, const Modes& B) {
  M4 L = blk4(neg(B.Vf), A.Vb), R = blk4(neg(A.Vf), B.Vb);
  try { return solve4<4>(L, R); } catch (Singular&) { return qr_solve4(L, R); }
}
// _SProp (:50-62): diag(e^{iQf d}, e^{-iQb d})
static M4 s_prop(double d, const Modes& m) {
  M4 o;
  o(0, 0) = std::exp(I1 * m.Qf.v[0] * d);
  o(1, 1) = std::exp(I1 * m.Qf.v[1] * d);
  o(2, 2) = std::exp(-I1 * m.Qb.v[0] * d);
  o(3, 3) = std::exp(-I1 * m.Qb.v[1] * d);
  return o;
}
static M2 blk(const M4& S, int bi, int bj) {
  M2 o;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) o(i, j) = S(2 * bi + i, 2 * bj + j);
  return o;
}
static M4 join(const M2& a, const M2& b, const M2& c, const M2& d) {
  M4 o;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) { o(i, j) = a(i, j); o(i, j + 2) = b(i, j); o(i + 2, j) = c(i, j); o(i + 2, j + 2) = d(i, j); }
  return o;
}
// _Redheffer (:65-85)
static M4 redheffer(const M4& S1, const M4& S2) {
  M2 a11 = blk(S1, 0, 0), a12 = blk(S1, 0, 1), a21 = blk(S1, 1, 0), a22 = blk(S1, 1, 1);
  M2 b11 = blk(S2, 0, 0), b12 = blk(S2, 0, 1), b21 = blk(S2, 1, 0), b22 = blk(S2, 1, 1);
  M2 D1 = i_minus(mul(a12, b21));
  M2 D2 = i_minus(mul(b21, a12));
  M2 S11 = mul(b11, solve2<2>(D1, a11));
  M2 S12 = add(b12, mul(b11, mul(solve2<2>(D1, a12), b22)));
  M2 S21 = add(a21, mul(a22, mul(solve2<2>(D2, b21), a11)));
  M2 S22 = mul(a22, solve2<2>(D2, b22));
  return join(S11, S12, S21, S22);
}

struct SAll {
  std::vector<M4> Sint, Sprop, SLeft, SRight;
};
// S_all_ingredients (:94-109) and S_all_Matrix (:112-142)
static void s_all(const Stack& st, const std::vector<Modes>& modes, SAll& S) {
  int N = (int)st.size();
  S.Sprop.resize(N);
  S.Sint.resize(N > 0 ? N - 1 : 0);
  for (int j = 0; j < N; ++j) S.Sprop[j] = s_prop(st[j].d, modes[j]);
  for (int j = 1; j < N; ++j) S.Sint[j - 1] = s_interface(modes[j - 1], modes[j]);
  S.SLeft.assign(N, M4());
  S.SRight.assign(N, M4());
  S.SLeft[0] = eye4();
  M4 S0 = redheffer(eye4(), S.Sprop[0]);
  for (int j = 1; j < N; ++j) {
    M4 Stot = redheffer(S0, S.Sint[j - 1]);
    S.SLeft[j] = Stot;
    S0 = redheffer(Stot, S.Sprop[j]);
  }
  S.SRight[N - 1] = eye4();
  for (int k = N - 2; k >= 0; --k) {
    M4 effect = redheffer(S.Sprop[k], S.Sint[k]);
    S.SRight[k] = redheffer(effect, S.SRight[k + 1]);
  }
}

// ---------------------------------------------------------------------------------
// Field solver (mod_FieldSolver.jl)
// ---------------------------------------------------------------------------------
static const double DENORMAL_FLOOR = 1e-250;
static cd flushc(const cd& x) { return std::abs(x) < DENORMAL_FLOOR ? cd(0.0, 0.0) : x; }
template <int R, int C>
static Mt<R, C> flushm(const Mt<R, C>& a) {
  Mt<R, C> o;
  for (int i = 0; i < R * C; ++i) o.v[i] = flushc(a.v[i]);
  return o;
}
// _cond2x2 (:33-42)
static double cond2x2(const M2& A) {
  M2 G = mul(adj(A), A);
  double tr = (G(0, 0) + G(1, 1)).real();
  double det = (G(0, 0) * G(1, 1) - G(0, 1) * G(1, 0)).real();
  double disc = std::sqrt(std::max(tr * tr - 4 * det, 0.0));
  double l1 = (tr + disc) / 2, l2 = (tr - disc) / 2;
  if (l2 <= 0) return INFINITY;
  return std::sqrt(l1 / l2);
}
// _cond2x2_eq (:49-53)
static double cond2x2_eq(const M2& A) {
  double n1 = std::sqrt(std::norm(A(0, 0)) + std::norm(A(1, 0)));
  double n2 = std::sqrt(std::norm(A(0, 1)) + std::norm(A(1, 1)));
  if (!(n1 > 0 && n2 > 0 && std::isfinite(n1) && std::isfinite(n2))) return INFINITY;
  V2 dg; dg.v[0] = 1.0 / n1; dg.v[1] = 1.0 / n2;
  return cond2x2(muld(A, dg));
}
// FieldSolver._SProp(d, Q) (:56-61)
static V2 sprop2(double d, const V2& Q) {
  V2 o;
  o.v[0] = std::exp(I1 * Q.v[0] * d);
  o.v[1] = std::exp(I1 * Q.v[1] * d);
  return o;
}

struct Cav {
  M2 RL, RR;
  M4 RRright;
  bool has_rr;
  V2 Qf, Qb;
  double d;
};
// _R_cavity (:72-89); `layer` is 1-based
static Cav r_cavity(const Stack& st, int layer, const std::vector<Modes>& modes, const SAll& S) {
  int N = (int)st.size();
  Cav c;
  c.d = st[layer - 1].d;
  c.Qf = modes[layer - 1].Qf;
  c.Qb = modes[layer - 1].Qb;
  c.RL = blk(S.SLeft[layer - 1], 0, 1);
  c.has_rr = layer != N;
  if (layer == N) return c;
  V2 a = sprop2(-c.d, c.Qf), b = sprop2(c.d, c.Qb);
  M4 SPhi;
  SPhi(0, 0) = a.v[0]; SPhi(1, 1) = a.v[1]; SPhi(2, 2) = b.v[0]; SPhi(3, 3) = b.v[1];
  c.RRright = redheffer(SPhi, S.SRight[layer - 1]);
  c.RR = blk(c.RRright, 1, 0);
  return c;
}

// _cavity_resummation (:142-152), generic over the seed width C
template <int C>
static void cavity_resummation(const Mt<2, C>& Sp, const Mt<2, C>& Sm, const Cav& c, int N, int layer,
                               Mt<2, C>& Fp, Mt<2, C>& Fm) {
  if (layer == N) { Fp = Mt<2, C>(); Fm = Sm; return; }
  V2 PF = sprop2(c.d, c.Qf), PB = sprop2(-c.d, c.Qb);
  M2 M = mul(muld(dmul(PF, c.RL), PB), c.RR);
  Fp = solve2<C>(i_minus(M), add(Sp, dmul(PF, mul(c.RL, Sm))));
  Fm = add(Sm, dmul(PB, mul(c.RR, Fp)));
}

// _walk_stack (:191-290). `layers` = obs layers of interest (1-based), empty = all.
template <int C>
static void walk_stack(const Stack& st, int layer, const Mt<2, C>& Fp, const Mt<2, C>& Fm, const Cav& cv,
                       const std::vector<Modes>& modes, const SAll& S, const std::set<int>* layers,
                       std::vector<Mt<2, C>>& Ef, std::vector<Mt<2, C>>& Eb, double tol = 1e-8) {
  int N = (int)st.size();
  typedef Mt<2, C> MC;
  MC Z;
  Ef.assign(N, Z);
  Eb.assign(N, Z);
  MC Ef_left = mul(cv.RL, Fm);
  bool want_self = layers == nullptr || layers->count(layer);
  bool any_right = false, any_left = false;
  if (layers) for (int o : *layers) { if (o > layer) any_right = true; if (o < layer) any_left = true; }
  bool need_right = layers == nullptr || any_right || (want_self && layer < N);
  bool need_left = layers == nullptr || any_left;
  if (layer < N && need_right) {
    M2 S11 = blk(cv.RRright, 0, 0), S12 = blk(cv.RRright, 0, 1);
    MC cm = Z;
    MC cp = add(mul(S11, Fp), mul(S12, cm));
    Ef[N - 1] = add(Ef[N - 1], flushm(cp));
    Eb[N - 1] = add(Eb[N - 1], flushm(cm));
    for (int k = layer + 1; k <= N - 1; ++k) {
      const M4& Sk = S.SRight[k - 1];
      M2 S11k = blk(Sk, 0, 0), S12k = blk(Sk, 0, 1), S21k = blk(Sk, 1, 0), S22k = blk(Sk, 1, 1);
      MC bp = cond2x2_eq(S11k) > 1 / tol ? Z : solve2<C>(S11k, sub(cp, mul(S12k, cm)));
      MC bm = add(mul(S21k, bp), mul(S22k, cm));
      Ef[k - 1] = add(Ef[k - 1], flushm(bp));
      Eb[k - 1] = add(Eb[k - 1], flushm(bm));
    }
  }
  if (layer > 1 && need_left) {
    M2 S22 = blk(S.SLeft[layer - 1], 1, 1);
    MC ap = Z;
    MC am = mul(S22, Fm);
    Ef[0] = add(Ef[0], flushm(ap));
    Eb[0] = add(Eb[0], flushm(am));
    for (int k = layer - 1; k >= 2; --k) {
      const M4& Sk = S.SLeft[k - 1];
      M2 S11k = blk(Sk, 0, 0), S12k = blk(Sk, 0, 1), S21k = blk(Sk, 1, 0), S22k = blk(Sk, 1, 1);
      MC bm = cond2x2_eq(S22k) > 1 / tol ? Z : solve2<C>(S22k, sub(am, mul(S21k, ap)));
      MC bp = add(mul(S11k, ap), mul(S12k, bm));
      Ef[k - 1] = add(Ef[k - 1], flushm(bp));
      Eb[k - 1] = add(Eb[k - 1], flushm(bm));
    }
  }
  for (int k = 1; k <= N - 1; ++k) {
    MC Ef_far;
    if (k == layer) Ef_far = Fp;
    else Ef_far = dmul(sprop2(st[k - 1].d, modes[k - 1].Qf), Ef[k - 1]);
    MC Eb_next = k == layer - 1 ? Fm : Eb[k];
    const M4& Sk = S.Sint[k - 1];
    M2 S21k = blk(Sk, 1, 0), S22k = blk(Sk, 1, 1);
    Eb[k - 1] = flushm(add(mul(S21k, Ef_far), mul(S22k, Eb_next)));
  }
  Ef[layer - 1] = flushm(Ef_left);
  if (layer == N) Eb[N - 1] = flushm(Fm);
}

// _cavity_transfer_columns (:320-341): T^o per obs layer (1-based), in `obs` order
static void cavity_transfer_columns(const Stack& st, int layer, const std::vector<Modes>& modes, const SAll& S,
                                    const std::vector<int>& obs, std::vector<M4>& T) {
  int N = (int)st.size();
  Cav cv = r_cavity(st, layer, modes, S);
  M24 Ep, Em;
  Ep(0, 0) = 1; Ep(1, 1) = 1;
  Em(0, 2) = 1; Em(1, 3) = 1;
  M24 Sp = layer < N ? Ep : M24();
  M24 Fp, Fm;
  cavity_resummation<4>(Sp, Em, cv, N, layer, Fp, Fm);
  std::set<int> others;
  for (int o : obs) if (o != layer) others.insert(o);
  std::vector<M24> Ef, Eb;
  if (!others.empty()) walk_stack<4>(st, layer, Fp, Fm, cv, modes, S, &others, Ef, Eb);
  T.resize(obs.size());
  for (size_t i = 0; i < obs.size(); ++i) {
    int o = obs[i];
    M24 ef, eb;
    if (o == layer) { ef = mul(cv.RL, Fm); eb = mul(cv.RR, Fp); }
    else { ef = Ef[o - 1]; eb = Eb[o - 1]; }
    M4 t;
    for (int j = 0; j < 4; ++j) { t(0, j) = ef(0, j); t(1, j) = ef(1, j); t(2, j) = eb(0, j); t(3, j) = eb(1, j); }
    T[i] = t;
  }
}

// Modal_amp (:356-363) for one point seed (z, sif, sib) in `layer` (Modal_amp convention)
static void modal_amp(const Stack& st, int layer, double z, const V2& sif, const V2& sib, const std::vector<Modes>& modes,
                      const SAll& S, std::vector<V2>& Ef, std::vector<V2>& Eb) {
  int N = (int)st.size();
  Cav cv = r_cavity(st, layer, modes, S);
  double d = cv.d;
  double zpos = layer == 1 ? d - z : z;
  V2 Sp, Sm;
  if (layer < N) {
    V2 pf = sprop2(d - zpos, cv.Qf);
    Sp.v[0] = sif.v[0] * pf.v[0]; Sp.v[1] = sif.v[1] * pf.v[1];
  }
  V2 pb = sprop2(-zpos, cv.Qb);
  Sm.v[0] = sib.v[0] * pb.v[0]; Sm.v[1] = sib.v[1] * pb.v[1];
  V2 Fp, Fm;
  cavity_resummation<1>(Sp, Sm, cv, N, layer, Fp, Fm);
  walk_stack<1>(st, layer, Fp, Fm, cv, modes, S, nullptr, Ef, Eb);
}

// Modal_amp_profile (:375-406) at local zs (layer's own frame, 0..d)
static void modal_amp_profile(const Stack& st, int layer, double z, const V2& sif, const V2& sib,
                              const std::vector<Modes>& modes, const SAll& S, int nz, const double* zs, V2* Ef, V2* Eb) {
  int N = (int)st.size();
  Cav cv = r_cavity(st, layer, modes, S);
  double d = cv.d;
  double zpos = layer == 1 ? d - z : z;
  V2 Sp, Sm;
  if (layer < N) {
    V2 pf = sprop2(d - zpos, cv.Qf);
    Sp.v[0] = sif.v[0] * pf.v[0]; Sp.v[1] = sif.v[1] * pf.v[1];
  }
  V2 pb = sprop2(-zpos, cv.Qb);
  Sm.v[0] = sib.v[0] * pb.v[0]; Sm.v[1] = sib.v[1] * pb.v[1];
  V2 Fp, Fm;
  cavity_resummation<1>(Sp, Sm, cv, N, layer, Fp, Fm);
  V2 Ef0 = mul(cv.RL, Fm), Ebd = mul(cv.RR, Fp);
  for (int i = 0; i < nz; ++i) {
    double zf = zs[i];
    V2 ef = Ef0, eb = Ebd;
    if (zpos < zf) { V2 p = sprop2(-zpos, cv.Qf); ef.v[0] += sif.v[0] * p.v[0]; ef.v[1] += sif.v[1] * p.v[1]; }
    if (zpos > zf) { V2 p = sprop2(d - zpos, cv.Qb); eb.v[0] += sib.v[0] * p.v[0]; eb.v[1] += sib.v[1] * p.v[1]; }
    Ef[i] = flushm(ef);
    Eb[i] = flushm(eb);
  }
}

// ---------------------------------------------------------------------------------
// Source projection (mod_SourceProj.jl:34-60)
// ---------------------------------------------------------------------------------
static void source_projection(double kx, double ky, double w, const Layer& L, const Modes& m, M23& sif, M23& sib) {
  cd etz1 = L.E(1, 3), etz2 = L.E(2, 3), ezz = L.E(3, 3);
  cd kt1(kx, 0.0), kt2(ky, 0.0);
  cd jw(0.0, -w);  // (-1im * ω)
  // Jt_cols = jw .* [1 0 0; 0 1 0]; Jz_row = jw .* (0, 0, 1)
  cd Jz[3] = {jw * 0.0, jw * 0.0, jw * 1.0};
  M43 J;
  for (int q = 0; q < 3; ++q) {
    J(0, q) = kt1 * Jz[q] / (ezz * w);
    J(1, q) = kt2 * Jz[q] / (ezz * w);
  }
  // J_Ht = R2s * Jt_cols - (R2s * ϵtz) * transpose(Jz_row) / ϵzz ; R2s = [0 1; -1 0]
  cd Jt[2][3] = {{jw * 1.0, jw * 0.0, jw * 0.0}, {jw * 0.0, jw * 1.0, jw * 0.0}};
  cd r1 = etz2, r2 = -etz1;  // R2s * ϵtz
  for (int q = 0; q < 3; ++q) {
    J(2, q) = Jt[1][q] - r1 * Jz[q] / ezz;
    J(3, q) = -Jt[0][q] - r2 * Jz[q] / ezz;
  }
  M4 V = blk4(m.Vf, m.Vb), W = blk4(m.Wf, m.Wb);
  M4 WV = mul(adj(W), V);
  M43 WJ = mul(adj(W), J);
  M43 s = solve4<3>(WV, WJ);
  for (int q = 0; q < 3; ++q) {
    sif(0, q) = s(0, q); sif(1, q) = s(1, q);
    sib(0, q) = s(2, q); sib(1, q) = s(3, q);
  }
}

// ---------------------------------------------------------------------------------
// Transfer cache (mod_CavityTransfer.jl)
// ---------------------------------------------------------------------------------
struct Basis {  // per node, per mode m: Ex,Ey,Ez (f), Ex,Ey,Ez (b), KZf, KZb
  cd exf[2], eyf[2], ezf[2], exb[2], eyb[2], ezb[2], kzf[2], kzb[2];
};

// _mode_field_core + _fill_obs_basis! (:87-130)
static void fill_basis(const Layer& L, const Modes& m, double w, double kx, double ky, Basis& B) {
  cd ezt1 = L.E(3, 1), ezt2 = L.E(3, 2), ezz = L.E(3, 3);
  cd k1(kx, 0.0), k2(ky, 0.0);
  for (int j = 0; j < 2; ++j) {
    auto field = [&](const M42& V, cd& ex, cd& ey, cd& ez) {
      ex = V(0, j); ey = V(1, j);
      ez = -(ezt1 * V(0, j) + ezt2 * V(1, j) + (1.0 / w) * (k1 * V(3, j) - k2 * V(2, j))) / ezz;
    };
    cd exf, eyf, ezf, exb, eyb, ezb;
    field(m.Vf, exf, eyf, ezf);
    field(m.Vb, exb, eyb, ezb);
    cd kzf = m.Qf.v[j], kzb = m.Qb.v[j];
    if (!(isfinc(exf) && isfinc(eyf) && isfinc(ezf) && isfinc(exb) && isfinc(eyb) && isfinc(ezb) && isfinc(kzf) && isfinc(kzb)))
      continue;
    B.exf[j] = exf; B.eyf[j] = eyf; B.ezf[j] = ezf;
    B.exb[j] = exb; B.eyb[j] = eyb; B.ezb[j] = ezb;
    B.kzf[j] = kzf; B.kzb[j] = kzb;
  }
}

struct Cache {
  Stack st;
  double w = 0;
  int src = 1;                 // 1-based
  std::vector<int> obs;        // 1-based, sorted unique
  bool is2d = false, rotation = false;
  int Nk = 0, Np = 1;          // nodes: n = k + Nk * p
  std::vector<double> kr, wr;  // 1D: kx nodes / weights; 2D: kρ nodes / weights
  std::vector<double> phi, wphi;
  std::vector<double> kxn, kyn;  // per flat node
  std::vector<char> valid;
  std::vector<std::vector<char>> Tvalid;  // [obs index][node]
  std::vector<std::vector<M4>> T;         // [obs index][node]
  std::vector<V2> Qf, Qb;
  std::vector<M23> sf, sb;
  std::vector<std::vector<Basis>> basis;  // [obs index][node]
  std::vector<double> d_obs;
  double d_src = 0;
  mutable std::string node_error;  // set by a node that raised past the per-node catch
  int n() const { return Nk * Np; }
  int oidx(int o) const {
    for (size_t i = 0; i < obs.size(); ++i) if (obs[i] == o) return (int)i;
    return -1;
  }
};

static void alloc_cache(Cache& c) {
  int n = c.n(), no = (int)c.obs.size();
  c.valid.assign(n, 0);
  c.Tvalid.assign(no, std::vector<char>(n, 0));
  c.T.assign(no, std::vector<M4>(n));
  c.Qf.assign(n, V2()); c.Qb.assign(n, V2());
  c.sf.assign(n, M23()); c.sb.assign(n, M23());
  Basis z;
  for (int j = 0; j < 2; ++j) z.exf[j] = z.eyf[j] = z.ezf[j] = z.exb[j] = z.eyb[j] = z.ezb[j] = z.kzf[j] = z.kzb[j] = 0.0;
  c.basis.assign(no, std::vector<Basis>(n, z));
  c.d_obs.resize(no);
  for (int i = 0; i < no; ++i) c.d_obs[i] = c.st[c.obs[i] - 1].d;
  c.d_src = c.st[c.src - 1].d;
}

// Fill one node from a solved, continuity-matched mode set and its T^o
// (build_cavity_transfer_1d body :226-248, fill_node! :339-359)
static void fill_node(Cache& c, int n, double kx, double ky, const std::vector<Modes>& modes, const std::vector<M4>& Tk) {
  M23 sif, sib;
  try {
    source_projection(kx, ky, c.w, c.st[c.src - 1], modes[c.src - 1], sif, sib);
  } catch (Singular&) { return; }
  if (!(allfinite(sif) && allfinite(sib))) return;
  for (size_t i = 0; i < c.obs.size(); ++i)
    if (allfinite(Tk[i])) { c.T[i][n] = Tk[i]; c.Tvalid[i][n] = 1; }
  c.Qf[n] = modes[c.src - 1].Qf;
  c.Qb[n] = modes[c.src - 1].Qb;
  c.sf[n] = sif;
  c.sb[n] = neg(sib);
  for (size_t i = 0; i < c.obs.size(); ++i) fill_basis(c.st[c.obs[i] - 1], modes[c.obs[i] - 1], c.w, kx, ky, c.basis[i][n]);
  c.valid[n] = 1;
}

static bool solve_node(const Cache& c, double kx, double ky, std::vector<Modes>& modes, std::vector<M4>& Tk) {
  try {
    if (!modes_stack(c.st, c.w, kx, ky, modes)) return false;
    SAll S;
    s_all(c.st, modes, S);
    cavity_transfer_columns(c.st, c.src, modes, S, c.obs, Tk);
    return true;
  } catch (Singular&) {
    return false;
  } catch (EigenError& e) {
#pragma omp critical(ytfo_node_error)
    if (c.node_error.empty()) c.node_error = e.what();
    return false;
  }
}

// the error a node of the build raised past the reference's per-node catch, if any
static void raise_node_error(const Cache& c) {
  if (!c.node_error.empty()) throw std::runtime_error(c.node_error);
}

// build_cavity_transfer_1d (:196-258)
static void build_1d(Cache& c) {
  alloc_cache(c);
  int n = c.n();
  c.kxn = c.kr; c.kyn.assign(n, 0.0);
#pragma omp parallel for schedule(dynamic, 16)
  for (int k = 0; k < n; ++k) {
    std::vector<Modes> modes;
    std::vector<M4> Tk;
    if (!solve_node(c, c.kr[k], 0.0, modes, Tk)) continue;
    fill_node(c, k, c.kr[k], 0.0, modes, Tk);
  }
  raise_node_error(c);
}

// build_cavity_transfer_2d (:307-398)
static void build_2d(Cache& c) {
  alloc_cache(c);
  int Nk = c.Nk, Np = c.Np;
  c.kxn.resize(Nk * Np); c.kyn.resize(Nk * Np);
  for (int p = 0; p < Np; ++p)
    for (int k = 0; k < Nk; ++k) {
      c.kxn[k + Nk * p] = c.kr[k] * std::cos(c.phi[p]);
      c.kyn[k + Nk * p] = c.kr[k] * std::sin(c.phi[p]);
    }
  if (c.rotation) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < Nk; ++k) {
      std::vector<Modes> modes0;
      std::vector<M4> Tk;
      double kx0 = c.kr[k] * std::cos(0.0), ky0 = c.kr[k] * std::sin(0.0);
      if (!solve_node(c, kx0, ky0, modes0, Tk)) continue;
      for (int p = 0; p < Np; ++p) {
        std::vector<Modes> mr(modes0.size());
        for (size_t j = 0; j < modes0.size(); ++j) mr[j] = rotate_modes(modes0[j], c.phi[p]);
        double kr = c.kr[k], ph = c.phi[p];
        fill_node(c, k + Nk * p, kr * std::cos(ph), kr * std::sin(ph), mr, Tk);
      }
    }
  } else {
#pragma omp parallel for schedule(dynamic, 16)
    for (int idx = 0; idx < Nk * Np; ++idx) {
      int k = idx / Np, p = idx % Np;
      std::vector<Modes> modes;
      std::vector<M4> Tk;
      double kr = c.kr[k], ph = c.phi[p];
      double kx = kr * std::cos(ph), ky = kr * std::sin(ph);
      if (!solve_node(c, kx, ky, modes, Tk)) continue;
      fill_node(c, k + Nk * p, kx, ky, modes, Tk);
    }
  }
  raise_node_error(c);
}

// ---------------------------------------------------------------------------------
// Synthesis (mod_ClosedFormField.jl)
// ---------------------------------------------------------------------------------
// _phase (:59-69)
static cd phase(const cd& kz, double z) {
  double a = -kz.imag() * z, b = kz.real() * z;
  if (!std::isfinite(a) || !std::isfinite(b) || a > 700) return cd(0.0, 0.0);
  if (a < -700) return cd(0.0, 0.0);
  return std::exp(cd(a, b));
}
static cd finite_or_zero(const cd& z) { return isfinc(z) ? z : cd(0.0, 0.0); }
static double zpos_of(const Cache& c, double zsrc) { return c.src == 1 ? c.d_src - zsrc : zsrc; }

enum Terms { T_ALL = 0, T_DIRECT = 1, T_SCATTERED = 2, T_TOEPLITZ = 3, T_HANKEL = 4 };

// Amplitude arrays: [node][m][q]
struct Amp {
  std::vector<cd> f, b;  // size n*6, index (n*2 + m)*3 + q
  void init(int n) { f.assign(n * 6, 0.0); b.assign(n * 6, 0.0); }
  cd& F(int n, int m, int q) { return f[(n * 2 + m) * 3 + q]; }
  cd& B(int n, int m, int q) { return b[(n * 2 + m) * 3 + q]; }
};

// amplitude_at (1D :175-203, 2D :539-566), point source (Δz_box = 0)
static void amplitude_at(const Cache& c, int obs_layer, double zsrc, double uf, double ub, Amp& A) {
  int oi = c.oidx(obs_layer);
  if (oi < 0) throw std::runtime_error("amplitude_at: obs_layer not in this cache's obs_layers");
  double zpos = zpos_of(c, zsrc), d = c.d_src;
  double se = std::sqrt(std::numeric_limits<double>::epsilon());
  if (!(-se <= zpos && zpos <= d + se)) throw std::runtime_error("amplitude_at: zsrc_local outside [0,d]");
  int n = c.n();
  A.init(n);
  for (int k = 0; k < n; ++k) {
    if (!(c.valid[k] && c.Tvalid[oi][k])) continue;
    const V2 &Qf = c.Qf[k], &Qb = c.Qb[k];
    cd Pf[2] = {std::exp(I1 * Qf.v[0] * (d - zpos)), std::exp(I1 * Qf.v[1] * (d - zpos))};
    cd Pb[2] = {std::exp(-I1 * Qb.v[0] * zpos), std::exp(-I1 * Qb.v[1] * zpos)};
    for (int q = 0; q < 3; ++q) {
      V4 u;
      u.v[0] = uf * c.sf[k](0, q) * Pf[0];
      u.v[1] = uf * c.sf[k](1, q) * Pf[1];
      u.v[2] = ub * c.sb[k](0, q) * Pb[0];
      u.v[3] = ub * c.sb[k](1, q) * Pb[1];
      V4 v = mul(c.T[oi][k], u);
      A.F(k, 0, q) = v.v[0]; A.F(k, 1, q) = v.v[1];
      A.B(k, 0, q) = v.v[2]; A.B(k, 1, q) = v.v[3];
    }
  }
}

// direct_amplitude (1D :232-259, 2D :577-602), point source
static void direct_amplitude(const Cache& c, double zsrc, double zobs, Amp& A) {
  double zpos = zpos_of(c, zsrc);
  double zeta = zobs - zpos;
  int n = c.n();
  A.init(n);
  bool fwd = zeta > 0, bwd = zeta < 0;
  if (!(fwd || bwd)) return;
  for (int k = 0; k < n; ++k) {
    if (!c.valid[k]) continue;
    if (fwd) {
      cd e[2] = {phase(c.Qf[k].v[0], zeta), phase(c.Qf[k].v[1], zeta)};
      for (int q = 0; q < 3; ++q)
        for (int m = 0; m < 2; ++m) A.F(k, m, q) = c.sf[k](m, q) * e[m];
    } else {
      cd e[2] = {phase(c.Qb[k].v[0], zeta), phase(c.Qb[k].v[1], zeta)};
      for (int q = 0; q < 3; ++q)
        for (int m = 0; m < 2; ++m) A.B(k, m, q) = c.sb[k](m, q) * e[m];
    }
  }
}

// _term_amplitudes (:143-160) -> (Af_r, Ab_r, with_direct)
static bool term_amplitudes(const Cache& c, int obs_layer, double zsrc, int terms, Amp& R) {
  bool same = obs_layer == c.src;
  if ((terms == T_TOEPLITZ || terms == T_HANKEL || terms == T_DIRECT) && !same)
    throw std::runtime_error("closed_form_G: terms needs obs_layer == source_layer");
  if (terms == T_ALL || terms == T_SCATTERED) {
    amplitude_at(c, obs_layer, zsrc, 1.0, 1.0, R);
    return same && terms == T_ALL;
  }
  if (terms == T_DIRECT) {
    amplitude_at(c, obs_layer, zsrc, 1.0, 0.0, R);
    std::fill(R.f.begin(), R.f.end(), cd(0.0, 0.0));
    std::fill(R.b.begin(), R.b.end(), cd(0.0, 0.0));
    return true;
  }
  if (terms == T_TOEPLITZ || terms == T_HANKEL) {
    Amp Af, Ab;  // seeds :f -> (Aff, Abf); seeds :b -> (Afb, Abb)
    amplitude_at(c, obs_layer, zsrc, 1.0, 0.0, Af);
    amplitude_at(c, obs_layer, zsrc, 0.0, 1.0, Ab);
    if (terms == T_TOEPLITZ) { R.f = Af.f; R.b = Ab.b; return true; }
    R.f = Ab.f; R.b = Af.b; return false;
  }
  throw std::runtime_error("closed_form_G: bad terms");
}

// closed_form_G, 1D cache (:435-487). G layout: (Nx, Ny, Nz, 3, 3) column-major, complex.
static void green_1d(const Cache& c, int obs_layer, double zsrc, int nz, const double* zo, int nx, const double* xs,
                     int ny, const double* ys, int terms, cd* G) {
  int oi = c.oidx(obs_layer);
  if (oi < 0) throw std::runtime_error("closed_form_G: obs_layer not in cache");
  int Nk = c.n();
  Amp R;
  bool same = term_amplitudes(c, obs_layer, zsrc, terms, R);
  const std::vector<Basis>& Bs = c.basis[oi];
  double d = c.d_obs[oi];
  // distinct radii, first-occurrence order over (i fastest, j)
  std::vector<double> rpix(nx * ny);
  std::vector<double> ur;
  std::map<double, int> ridx;
  std::vector<int> rmap(nx * ny);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      double r = std::hypot(xs[i], ys[j]);
      rpix[i + nx * j] = r;
      auto it = ridx.find(r);
      if (it == ridx.end()) { ridx[r] = (int)ur.size(); rmap[i + nx * j] = (int)ur.size(); ur.push_back(r); }
      else rmap[i + nx * j] = it->second;
    }
  int Nr = (int)ur.size();
  std::vector<double> J0(Nk * (size_t)Nr), J1(Nk * (size_t)Nr), J2(Nk * (size_t)Nr);
#pragma omp parallel for
  for (int r = 0; r < Nr; ++r)
    for (int k = 0; k < Nk; ++k) {
      double x = c.kr[k] * ur[r];
      J0[k + (size_t)Nk * r] = ::j0(x);
      J1[k + (size_t)Nk * r] = ::j1(x);
      J2[k + (size_t)Nk * r] = ::jn(2, x);
    }
  std::vector<cd> W(Nk);
  for (int k = 0; k < Nk; ++k) W[k] = (I1 * c.wr[k]) / (2 * PI);
  // weighted amplitudes: wA[k][m][q] for f and b
  std::vector<cd> wf(Nk * 6), wb(Nk * 6), Pf(Nk * 2), Pb(Nk * 2);
  std::vector<cd> R3(9 * (size_t)Nr);
  for (int zi = 0; zi < nz; ++zi) {
    double z = zo[zi];
    if (same) {
      Amp D;
      direct_amplitude(c, zsrc, z, D);
      for (int k = 0; k < Nk; ++k)
        for (int m = 0; m < 2; ++m) {
          cd pf = phase(Bs[k].kzf[m], z), pb = phase(Bs[k].kzb[m], z - d);
          for (int q = 0; q < 3; ++q) {
            cd af = D.F(k, m, q) + R.F(k, m, q) * pf;
            cd ab = D.B(k, m, q) + R.B(k, m, q) * pb;
            wf[(k * 2 + m) * 3 + q] = finite_or_zero(W[k] * af);
            wb[(k * 2 + m) * 3 + q] = finite_or_zero(W[k] * ab);
          }
          Pf[k * 2 + m] = 1.0; Pb[k * 2 + m] = 1.0;
        }
    } else {
      for (int k = 0; k < Nk; ++k)
        for (int m = 0; m < 2; ++m) {
          for (int q = 0; q < 3; ++q) {
            wf[(k * 2 + m) * 3 + q] = finite_or_zero(W[k] * R.F(k, m, q));
            wb[(k * 2 + m) * 3 + q] = finite_or_zero(W[k] * R.B(k, m, q));
          }
          Pf[k * 2 + m] = phase(Bs[k].kzf[m], z);
          Pb[k * 2 + m] = phase(Bs[k].kzb[m], z - d);
        }
    }
    // _integrate_pixel_1d (:344-390) at (ρ, x = ρ) per distinct radius and unit moment
#pragma omp parallel for schedule(dynamic, 4)
    for (int r = 0; r < Nr; ++r) {
      double rho = ur[r];
      double cpsi = rho == 0.0 ? 0.0 : rho / rho;
      for (int q = 0; q < 3; ++q) {
        cd px = q == 0 ? 1.0 : 0.0, py = q == 1 ? 1.0 : 0.0, pz = q == 2 ? 1.0 : 0.0;
        cd vx = 0.0, vy = 0.0, vz = 0.0;
        for (int k = 0; k < Nk; ++k) {
          double j0v = J0[k + (size_t)Nk * r], j1v = J1[k + (size_t)Nk * r], j2v = J2[k + (size_t)Nk * r];
          if (!(std::isfinite(j0v) && std::isfinite(j1v) && std::isfinite(j2v))) continue;
          double kx = c.kr[k];
          for (int m = 0; m < 2; ++m) {
            const Basis& b = Bs[k];
            cd exf = b.exf[m], exb = b.exb[m], eyf = b.eyf[m], eyb = b.eyb[m], ezf = b.ezf[m], ezb = b.ezb[m];
            cd phf = Pf[k * 2 + m], phb = Pb[k * 2 + m];
            cd axf = wf[(k * 2 + m) * 3 + 0], ayf = wf[(k * 2 + m) * 3 + 1], azf = wf[(k * 2 + m) * 3 + 2];
            cd Af = px * axf + py * ayf, Bf = px * ayf - py * axf, Cf = pz * azf;
            cd half(0.0, 0.5);
            cd Ixf = half * ((j2v - j0v) * Af * exf - (j0v + j2v) * Bf * eyf) + j1v * cpsi * Cf * exf;
            cd Iyf = half * ((j2v - j0v) * Af * eyf + (j0v + j2v) * Bf * exf) + j1v * cpsi * Cf * eyf;
            cd Izf = j1v * cpsi * Af * ezf - I1 * j0v * Cf * ezf;
            cd axb = wb[(k * 2 + m) * 3 + 0], ayb = wb[(k * 2 + m) * 3 + 1], azb = wb[(k * 2 + m) * 3 + 2];
            cd Ab = px * axb + py * ayb, Bb = px * ayb - py * axb, Cb = pz * azb;
            cd Ixb = half * ((j2v - j0v) * Ab * exb - (j0v + j2v) * Bb * eyb) + j1v * cpsi * Cb * exb;
            cd Iyb = half * ((j2v - j0v) * Ab * eyb + (j0v + j2v) * Bb * exb) + j1v * cpsi * Cb * eyb;
            cd Izb = j1v * cpsi * Ab * ezb - I1 * j0v * Cb * ezb;
            vx += (Ixf * phf + Ixb * phb) * kx;
            vy += (Iyf * phf + Iyb * phb) * kx;
            vz += (Izf * phf + Izb * phb) * kx;
          }
        }
        R3[0 + 3 * q + 9 * (size_t)r] = vx;
        R3[1 + 3 * q + 9 * (size_t)r] = vy;
        R3[2 + 3 * q + 9 * (size_t)r] = vz;
      }
    }
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        double rho = rpix[i + nx * j];
        double cp = rho == 0.0 ? 1.0 : xs[i] / rho, sp = rho == 0.0 ? 0.0 : ys[j] / rho;
        double Rot[3][3] = {{cp, -sp, 0}, {sp, cp, 0}, {0, 0, 1}};
        const cd* Rm = &R3[9 * (size_t)rmap[i + nx * j]];
        for (int q = 0; q < 3; ++q)
          for (int cc = 0; cc < 3; ++cc) {
            cd s = 0.0;
            for (int a = 0; a < 3; ++a) {
              cd t = Rot[cc][0] * Rm[0 + 3 * a];
              t += Rot[cc][1] * Rm[1 + 3 * a];
              t += Rot[cc][2] * Rm[2 + 3 * a];
              s += t * Rot[q][a];
            }
            G[i + (size_t)nx * (j + (size_t)ny * (zi + (size_t)nz * (cc + 3 * (size_t)q)))] = s;
          }
      }
  }
}

// closed_form_G, 2D cache, lateral=:direct (:711-753 with _strengths_row! :616-659)
static void green_2d(const Cache& c, int obs_layer, double zsrc, int nz, const double* zo, int nx, const double* xs,
                     int ny, const double* ys, int terms, cd* G) {
  int oi = c.oidx(obs_layer);
  if (oi < 0) throw std::runtime_error("closed_form_G: obs_layer not in cache");
  int Nk = c.Nk, Np = c.Np, Nn = Nk * Np;
  std::vector<cd> W(Nn);
  for (int p = 0; p < Np; ++p)
    for (int k = 0; k < Nk; ++k) W[k + Nk * p] = cd(c.kr[k] * c.wr[k] * c.wphi[p] / (4 * PI * PI), 0.0);
  Amp R;
  bool same = term_amplitudes(c, obs_layer, zsrc, terms, R);
  const std::vector<Basis>& Bs = c.basis[oi];
  double d = c.d_obs[oi];
  std::vector<cd> Px((size_t)Nn * nx), Py((size_t)Nn * ny);
  for (int n = 0; n < Nn; ++n) {
    for (int i = 0; i < nx; ++i) { double a = c.kxn[n] * xs[i]; Px[n + (size_t)Nn * i] = cd(std::cos(a), std::sin(a)); }
    for (int j = 0; j < ny; ++j) { double a = c.kyn[n] * ys[j]; Py[n + (size_t)Nn * j] = cd(std::cos(a), std::sin(a)); }
  }
  std::vector<cd> S((size_t)Nn * 9);
  for (int zi = 0; zi < nz; ++zi) {
    double z = zo[zi];
    Amp D;
    if (same) direct_amplitude(c, zsrc, z, D);
    for (int n = 0; n < Nn; ++n) {
      cd w = W[n];
      cd s[3][3];
      for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) s[a][b] = 0.0;
      for (int m = 0; m < 2; ++m) {
        cd pf = phase(Bs[n].kzf[m], z), pb = phase(Bs[n].kzb[m], z - d);
        const Basis& b = Bs[n];
        for (int q = 0; q < 3; ++q) {
          cd af_ = R.F(n, m, q) * pf, ab_ = R.B(n, m, q) * pb;
          if (same) { af_ += D.F(n, m, q); ab_ += D.B(n, m, q); }
          cd af = finite_or_zero(w * af_), ab = finite_or_zero(w * ab_);
          s[0][q] += b.exf[m] * af + b.exb[m] * ab;
          s[1][q] += b.eyf[m] * af + b.eyb[m] * ab;
          s[2][q] += b.ezf[m] * af + b.ezb[m] * ab;
        }
      }
      for (int q = 0; q < 3; ++q)
        for (int cc = 0; cc < 3; ++cc) S[n + (size_t)Nn * (cc + 3 * q)] = s[cc][q];
    }
#pragma omp parallel for collapse(2)
    for (int cq = 0; cq < 9; ++cq)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          cd acc = 0.0;
          const cd* sp = &S[(size_t)Nn * cq];
          const cd* px = &Px[(size_t)Nn * i];
          const cd* py = &Py[(size_t)Nn * j];
          for (int n = 0; n < Nn; ++n) acc += px[n] * (sp[n] * py[n]);
          int cc = cq % 3, q = cq / 3;
          G[i + (size_t)nx * (j + (size_t)ny * (zi + (size_t)nz * (cc + 3 * (size_t)q)))] = acc;
        }
  }
}

// ---------------------------------------------------------------------------------
// k-grids (mod_KxGrid.jl, mod_KSpaceFeatures.jl)
// ---------------------------------------------------------------------------------
// Gauss-Legendre nodes/weights on [-1,1], ascending (FastGaussQuadrature.gausslegendre):
// Newton on the three-term recurrence in long double, rounded once to double.
static void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.resize(n); w.resize(n);
  for (int i = 0; i < n; ++i) {
    long double z = cosl(3.14159265358979323846264338327950288L * (i + 0.75L) / (n + 0.5L));
    long double dp = 0;
    for (int it = 0; it < 100; ++it) {
      long double p0 = 1, p1 = z;
      for (int k = 2; k <= n; ++k) { long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
      if (n == 1) { p1 = z; p0 = 1; }
      dp = n * (z * p1 - p0) / (z * z - 1);
      long double dz = p1 / dp;
      z -= dz;
      if (fabsl(dz) < 1e-30L) break;
    }
    long double p0 = 1, p1 = z;
    for (int k = 2; k <= n; ++k) { long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
    dp = n * (z * p1 - p0) / (z * z - 1);
    x[n - 1 - i] = (double)z;  // ascending order
    w[n - 1 - i] = (double)(2.0L / ((1 - z * z) * dp * dp));
  }
  if (n % 2 == 1) x[n / 2] = 0.0;
}

// gl_rule (mod_KxGrid.jl:361-384)
static void gl_rule(const std::vector<std::pair<double, double>>& panels, int order, const std::vector<double>& singular,
                    std::vector<double>& nodes, std::vector<double>& wts) {
  std::vector<double> xi, wx;
  gauss_legendre(order, xi, wx);
  std::set<double> S(singular.begin(), singular.end());
  nodes.resize(panels.size() * order); wts.resize(panels.size() * order);
  size_t idx = 0;
  for (auto& pb : panels) {
    double a = pb.first, b = pb.second;
    double L = NAN, sg = 0;
    if (S.count(a)) { L = a; sg = 1.0; }
    else if (S.count(b)) { L = b; sg = -1.0; }
    if (sg == 0) {
      double h = 0.5 * (b - a), c = 0.5 * (a + b);
      for (int j = 0; j < order; ++j) { nodes[idx] = c + h * xi[j]; wts[idx] = h * wx[j]; ++idx; }
    } else {
      double U = std::sqrt(b - a);
      for (int j = 0; j < order; ++j) {
        double u = (0.5 * U) * (1 + xi[j]);
        nodes[idx] = L + sg * (u * u);
        wts[idx] = ((0.5 * U) * wx[j]) * (2 * u);
        ++idx;
      }
    }
  }
}

// halve_panels (mod_KxGrid.jl:387-388)
static std::vector<std::pair<double, double>> halve_panels(const std::vector<std::pair<double, double>>& p) {
  std::vector<std::pair<double, double>> o;
  for (auto& ab : p) {
    double m = (ab.first + ab.second) / 2;
    o.push_back({ab.first, m});
    o.push_back({m, ab.second});
  }
  return o;
}

// _dedup (mod_KxGrid.jl:83-89)
static std::vector<double> dedup(const std::vector<double>& ks, double rtol = 1e-9) {
  std::vector<double> out;
  for (double k : ks)
    if (out.empty() || k - out.back() > rtol * std::max(std::fabs(k), 1e-300)) out.push_back(k);
  return out;
}

static cd det3(const cd A[3][3]) {
  return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
         A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}
static void inv3(const cd A[3][3], cd B[3][3]) {
  cd d = det3(A);
  B[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) / d;
  B[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) / d;
  B[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) / d;
  B[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) / d;
  B[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) / d;
  B[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) / d;
  B[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) / d;
  B[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) / d;
  B[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) / d;
}

// layer_light_lines (mod_KxGrid.jl:41-59)
static std::vector<double> layer_light_lines(const Layer& L, double w, double phi) {
  cd e[3][3], m[3][3], mi[3][3], K[3][3], M[3][3], T[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) { e[i][j] = L.E(i + 1, j + 1); m[i][j] = L.U(i + 1, j + 1); }
  double c = std::cos(phi), s = std::sin(phi);
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) K[i][j] = 0.0;
  K[0][2] = s; K[1][2] = -c; K[2][0] = -s; K[2][1] = c;
  inv3(m, mi);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) { cd a = 0; for (int k = 0; k < 3; ++k) a += K[i][k] * mi[k][j]; T[i][j] = a; }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) { cd a = 0; for (int k = 0; k < 3; ++k) a += T[i][k] * K[k][j]; M[i][j] = a; }
  double me = 0, mm = 0;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) { me = std::max(me, std::abs(e[i][j])); mm = std::max(mm, std::abs(m[i][j])); }
  double w2 = w * w;
  double sc = w2 * std::max(me * mm, std::numeric_limits<double>::epsilon());
  cd A0[3][3], A1[3][3], A2[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      A0[i][j] = w2 * e[i][j];
      A1[i][j] = A0[i][j] + sc * M[i][j];
      A2[i][j] = A0[i][j] + (2 * sc) * M[i][j];
    }
  cd p0 = det3(A0), p1 = det3(A1), p2 = det3(A2);
  cd c2 = (p2 - 2.0 * p1 + p0) / (2 * sc * sc);
  cd c1 = (p1 - p0) / sc - c2 * sc;
  cd c0 = p0;
  std::vector<cd> roots;
  if (std::abs(c2) * sc * sc <= 1e-12 * (std::abs(c1) * sc + std::abs(c0))) {
    if (std::abs(c1) > 0) roots.push_back(-c0 / c1);
  } else {
    cd D = c1 * c1 - 4.0 * c2 * c0;
    cd Dl = std::abs(D) <= 1e-10 * std::norm(c1) ? cd(0.0, 0.0) : std::sqrt(D);
    roots.push_back((-c1 + Dl) / (2.0 * c2));
    roots.push_back((-c1 - Dl) / (2.0 * c2));
  }
  std::vector<double> out;
  for (auto& q : roots) if (q.real() > 0) out.push_back(std::sqrt(q).real());
  std::sort(out.begin(), out.end());
  return dedup(out, 1e-7);
}

// material_class (mod_KSpaceFeatures.jl:59-66): 0 dielectric, 1 metallic, 2 hyperbolic, 3 gyrotropic
static void sym3_eigs(const double A[3][3], double ev[3]) {
  double a[3][3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) a[i][j] = A[i][j];
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = std::fabs(a[0][1]) + std::fabs(a[0][2]) + std::fabs(a[1][2]);
    if (off < 1e-300) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (a[p][q] == 0) continue;
        double th = (a[q][q] - a[p][p]) / (2 * a[p][q]);
        double t = (th >= 0 ? 1 : -1) / (std::fabs(th) + std::sqrt(th * th + 1));
        double cs = 1 / std::sqrt(t * t + 1), sn = t * cs;
        for (int k = 0; k < 3; ++k) {
          double akp = a[k][p], akq = a[k][q];
          a[k][p] = cs * akp - sn * akq; a[k][q] = sn * akp + cs * akq;
        }
        for (int k = 0; k < 3; ++k) {
          double apk = a[p][k], aqk = a[q][k];
          a[p][k] = cs * apk - sn * aqk; a[q][k] = sn * apk + cs * aqk;
        }
      }
  }
  for (int i = 0; i < 3; ++i) ev[i] = a[i][i];
}
static int material_class(const Layer& L) {
  for (int i = 1; i <= 3; ++i)
    for (int j = 1; j <= 3; ++j)
      if (L.E(i, j) != L.E(j, i) || L.U(i, j) != L.U(j, i)) return 3;
  double re[3][3], rm[3][3], ee[3], em[3];
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) { re[i][j] = L.E(i + 1, j + 1).real(); rm[i][j] = L.U(i + 1, j + 1).real(); }
  sym3_eigs(re, ee); sym3_eigs(rm, em);
  bool ep = ee[0] > 0 && ee[1] > 0 && ee[2] > 0, en = ee[0] < 0 && ee[1] < 0 && ee[2] < 0;
  bool mp = em[0] > 0 && em[1] > 0 && em[2] > 0;
  if (ep && mp) return 0;
  if (en && mp) return 1;
  return 2;
}

static double sigma_max(const M2& A) {
  M2 G = mul(adj(A), A);
  double t = (G(0, 0) + G(1, 1)).real(), dt = (G(0, 0) * G(1, 1) - G(0, 1) * G(1, 0)).real();
  return std::sqrt(std::max((t + std::sqrt(std::max(t * t - 4 * dt, 0.0))) / 2, 0.0));
}

// _cavity_response (mod_KSpaceFeatures.jl:109-127); s is 1-based
static double cavity_response(const Stack& st, double w, int s, double kr, double phi) {
  try {
    std::vector<Modes> modes;
    if (!modes_stack(st, w, kr * std::cos(phi), kr * std::sin(phi), modes)) return 0.0;
    SAll S;
    s_all(st, modes, S);
    M2 RR = blk(redheffer(S.Sint[s - 1], S.SRight[s]), 1, 0);
    M2 RL = blk(S.SLeft[s - 1], 0, 1);
    double r = std::max(sigma_max(RL), sigma_max(RR));
    if (s > 1) {
      double d = st[s - 1].d;
      V2 PF = sprop2(d, modes[s - 1].Qf), PB = sprop2(-d, modes[s - 1].Qb);
      M2 M = i_minus(mul(muld(dmul(PF, RL), PB), RR));
      r = std::max(r, sigma_max(inv2(M)));
    }
    return std::isfinite(r) ? r : 0.0;
  } catch (...) {
    return 0.0;
  }
}

struct Pole { double q, G, phi, prom; };

// real_axis_poles (mod_KSpaceFeatures.jl:151-204)
static std::vector<Pole> real_axis_poles(const Stack& st, double w, int src, const std::vector<double>& phis, double k_lo,
                                         double k_hi, double scan_step, double prominence, const std::vector<double>& exclude,
                                         double floor_rel = 1e-6, double floor_abs = 1e-10) {
  double span = std::log(k_hi / k_lo);
  int n = (int)std::floor(span / scan_step + 1e-10) + 1;
  std::vector<double> ks(n);
  for (int i = 0; i < n; ++i) ks[i] = k_lo * std::exp(i * scan_step);
  int Wn = (int)std::ceil(std::log(4.0) / scan_step);
  std::vector<std::vector<Pole>> out(phis.size());
  for (size_t mi = 0; mi < phis.size(); ++mi) {
    double phi = phis[mi];
    auto f = [&](double k) { return cavity_response(st, w, src, k, phi); };
    std::vector<double> y(n);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) y[i] = std::log(f(ks[i]) + 1e-300);
    double ymax = *std::max_element(y.begin(), y.end());
    double ymin = std::max(ymax + std::log(floor_rel), std::log(floor_abs));
    for (int i = 1; i < n - 1; ++i) {
      if (!(y[i] > y[i - 1] && y[i] >= y[i + 1] && y[i] >= ymin)) continue;
      int jl = i; double lmin = y[i];
      while (jl > std::max(0, i - Wn) && y[jl - 1] <= y[i]) { --jl; lmin = std::min(lmin, y[jl]); }
      int jr = i; double rmin = y[i];
      while (jr < std::min(n - 1, i + Wn) && y[jr + 1] <= y[i]) { ++jr; rmin = std::min(rmin, y[jr]); }
      double base = std::max(lmin, rmin);
      double prom = y[i] - base;
      if (!(prom >= std::log(prominence))) continue;
      double a = ks[i - 1], b = ks[i + 1];
      double g = (std::sqrt(5.0) - 1) / 2;
      double c = b - g * (b - a), d = a + g * (b - a);
      double fc = f(c), fd = f(d);
      for (int it = 0; it < 60; ++it) {
        if ((b - a) <= 1e-12 * b) break;
        if (fc >= fd) { b = d; d = c; fd = fc; c = b - g * (b - a); fc = f(c); }
        else { a = c; c = d; fc = fd; d = a + g * (b - a); fd = f(d); }
      }
      double q = (a + b) / 2;
      double P = std::max(f(q), std::exp(y[i]));
      bool excl = false;
      for (double L : exclude) if (std::fabs(q - L) <= 1e-6 * q) excl = true;
      if (excl) continue;
      double lvl = std::exp(base) + (P - std::exp(base)) / std::sqrt(2.0);
      auto cross = [&](double lo, double hi) {
        for (int it = 0; it < 50; ++it) {
          if (std::fabs(hi - lo) <= 1e-12 * q) break;
          double mid = (lo + hi) / 2;
          if (f(mid) > lvl) lo = mid; else hi = mid;
        }
        return (lo + hi) / 2;
      };
      int jlast = jl;
      for (int j = jl; j <= i; ++j) if (y[j] == lmin) jlast = j;
      int jfirst = i;
      for (int j = i; j <= jr; ++j) if (y[j] == rmin) { jfirst = j; break; }
      double kl = ks[jlast], kr = ks[jfirst];
      double G = std::min(q - cross(q, kl), cross(q, kr) - q);
      out[mi].push_back({q, std::max(G, 1e-12 * q), phi, prom});
    }
  }
  std::vector<Pole> all;
  for (auto& v : out) all.insert(all.end(), v.begin(), v.end());
  return all;
}

struct Cluster { double a, b, G; };
// _clusters (mod_KSpaceFeatures.jl:217-229)
static std::vector<Cluster> clusters(std::vector<Pole> ps, double merge_rel) {
  std::stable_sort(ps.begin(), ps.end(), [](const Pole& x, const Pole& y) { return x.q < y.q; });
  std::vector<Cluster> cl;
  auto push_u = [&](Cluster c) {
    for (auto& e : cl) if (e.a == c.a && e.b == c.b && e.G == c.G) return;
    cl.push_back(c);
  };
  for (size_t i = 0; i < ps.size(); ++i) {
    push_u({ps[i].q, ps[i].q, ps[i].G});
    if (i > 0) {
      const Pole& r = ps[i - 1];
      const Pole& p = ps[i];
      if (p.q - r.q <= std::max(merge_rel * p.q, 4 * std::min(p.G, r.G)) && p.q > r.q) push_u({r.q, p.q, std::min(p.G, r.G)});
    }
  }
  return cl;
}

struct Features {
  std::vector<double> light_lines, singular_lines;
  double kmax, Kcut, h_min, rho_max, K_geom, K_cap;
  bool capped;
  std::vector<Pole> poles;
  std::vector<Cluster> cl;
  int N_phi;
};

// kspace_features, dims = 1 (mod_KSpaceFeatures.jl:295-360), azimuthally symmetric or 1D scan at φ = 0
static Features kspace_features_1d(const Stack& st, double w, int src, double h_min, double rho_max, double target_decay,
                                   double kr_cap, double kr_cap_rel, bool scan, double scan_step, double prominence) {
  Features F;
  int N = (int)st.size();
  std::vector<double> ll, sing;
  for (int j = 0; j < N; ++j) {
    auto L = layer_light_lines(st[j], w, 0.0);
    ll.insert(ll.end(), L.begin(), L.end());
    if (j == 0 || j == N - 1) sing.insert(sing.end(), L.begin(), L.end());
  }
  std::sort(ll.begin(), ll.end()); std::sort(sing.begin(), sing.end());
  F.light_lines = dedup(ll); F.singular_lines = dedup(sing);
  F.kmax = F.light_lines.empty() ? w : F.light_lines.back();
  F.K_geom = target_decay / h_min;
  F.K_cap = kr_cap > 0 ? kr_cap : kr_cap_rel * F.kmax;
  F.Kcut = std::min(std::max(F.K_geom, 2.0 * F.kmax), F.K_cap);
  F.capped = F.Kcut < F.K_geom;
  F.h_min = h_min; F.rho_max = rho_max;
  if (scan) {
    double k_lo = 0.5 * (F.light_lines.empty() ? w : F.light_lines[0]);
    F.poles = real_axis_poles(st, w, src, {0.0}, k_lo, F.Kcut, scan_step, prominence, F.light_lines);
  }
  F.cl = clusters(F.poles, 0.0);
  F.N_phi = 0;
  return F;
}

// _pole_track_η (mod_KSpaceFeatures.jl:243-259): the smallest φ-width Γ dφ / |dq| of a pole
// track between neighbouring scanned directions (a wrap pair closes a full circle); ∞ with
// fewer than two directions or no track
static double pole_track_eta(const std::vector<Pole>& poles, std::vector<double> phis) {
  std::sort(phis.begin(), phis.end());
  phis.erase(std::unique(phis.begin(), phis.end()), phis.end());
  if (phis.size() < 2) return INFINITY;
  struct Pair { double p1, p2, dp; };
  std::vector<Pair> pairs;
  for (size_t i = 0; i + 1 < phis.size(); ++i) pairs.push_back({phis[i], phis[i + 1], phis[i + 1] - phis[i]});
  const double step = phis[1] - phis[0];
  if (std::fabs(phis.back() - phis.front() + step - 2 * M_PI) < 1e-9) pairs.push_back({phis.back(), phis.front(), step});
  double eta = INFINITY;
  for (auto& pr : pairs)
    for (auto& p : poles)
      for (auto& r : poles) {
        if (!(p.phi == pr.p1 && r.phi == pr.p2)) continue;
        const double dq = std::fabs(p.q - r.q);
        if (!(0 < dq && dq <= pr.dp * std::max(p.q, r.q))) continue;
        eta = std::min(eta, std::min(p.G, r.G) * pr.dp / dq);
      }
  return eta;
}

// kspace_features, dims = 2 (mod_KSpaceFeatures.jl:295-360): the scanned directions (φ = 0
// for an azimuthally symmetric stack; N_φ_scan/4 + 1 over [0, π/2] when every tensor is
// diagonal; N_φ_scan over [0, 2π) otherwise), light lines at every scanned φ mod π, the
// union of the poles of every direction, clusters merged at the φ step, and N_φ, the largest
// of N_φ_min, c_φ Kcut ρ_max and c_η log(10/rtol)/η_min, rounded up to even. The scan
// directions are p (π/2)/(n - 1) and 2πp/N_φ_scan.
static Features kspace_features_2d(const Stack& st, double w, int src, double h_min, double rho_max, double target_decay,
                                   double kr_cap, double kr_cap_rel, bool scan, double scan_step, double prominence,
                                   int n_phi_scan, double c_phi, int n_phi_min, double rtol, double c_eta) {
  Features F;
  const int N = (int)st.size();
  const bool sym = azimuthally_symmetric(st);
  bool diag = true;
  for (auto& L : st)
    for (int i = 1; i <= 3; ++i)
      for (int j = 1; j <= 3; ++j)
        if (i != j && (L.E(i, j) != cd(0.0, 0.0) || L.U(i, j) != cd(0.0, 0.0))) diag = false;
  std::vector<double> phis;
  double merge_rel = 0.0;
  if (sym) {
    phis = {0.0};
  } else if (diag) {
    const int m = std::max(2, n_phi_scan / 4 + 1);
    for (int p = 0; p < m; ++p) phis.push_back((M_PI / 2) * p / (m - 1));
    merge_rel = (M_PI / 2) / std::max(1, n_phi_scan / 4);
  } else {
    for (int p = 0; p < n_phi_scan; ++p) phis.push_back(2 * M_PI * p / n_phi_scan);
    merge_rel = 2 * M_PI / n_phi_scan;
  }
  std::vector<double> phi_ll;  // light lines are even in the direction: φ mod π, first occurrences
  if (sym) phi_ll = {0.0};
  else
    for (double ph : phis) {
      const double m = std::fmod(ph, M_PI);
      if (std::find(phi_ll.begin(), phi_ll.end(), m) == phi_ll.end()) phi_ll.push_back(m);
    }
  std::vector<double> ll, sing;
  for (int j = 0; j < N; ++j)
    for (double ph : phi_ll) {
      auto L = layer_light_lines(st[j], w, ph);
      ll.insert(ll.end(), L.begin(), L.end());
      if (j == 0 || j == N - 1) sing.insert(sing.end(), L.begin(), L.end());
    }
  std::sort(ll.begin(), ll.end()); std::sort(sing.begin(), sing.end());
  F.light_lines = dedup(ll); F.singular_lines = dedup(sing);
  F.kmax = F.light_lines.empty() ? w : F.light_lines.back();
  F.K_geom = target_decay / h_min;
  F.K_cap = kr_cap > 0 ? kr_cap : kr_cap_rel * F.kmax;
  F.Kcut = std::min(std::max(F.K_geom, 2.0 * F.kmax), F.K_cap);
  F.capped = F.Kcut < F.K_geom;
  F.h_min = h_min; F.rho_max = rho_max;
  if (scan) {
    double k_lo = 0.5 * (F.light_lines.empty() ? w : F.light_lines[0]);
    F.poles = real_axis_poles(st, w, src, phis, k_lo, F.Kcut, scan_step, prominence, F.light_lines);
  }
  F.cl = clusters(F.poles, merge_rel);
  const long n_lat = (long)std::ceil(c_phi * F.Kcut * rho_max);
  const double eta = pole_track_eta(F.poles, phis);
  const long n_pole = std::isfinite(eta) ? (long)std::ceil(c_eta * std::log(10 / rtol) / eta) : 0;
  const long m = std::max(std::max((long)n_phi_min, n_lat), n_pole);
  F.N_phi = (int)(2 * ((m + 1) / 2));
  return F;
}

// graded_panels (mod_KxGrid.jl:331-347)
template <class Wf>
static std::vector<std::pair<double, double>> graded_panels(std::vector<double> bs, Wf width, double alpha, long max_panels = 10000000) {
  std::sort(bs.begin(), bs.end());
  bs.erase(std::unique(bs.begin(), bs.end()), bs.end());
  std::vector<std::pair<double, double>> panels;
  for (size_t i = 0; i + 1 < bs.size(); ++i) {
    double a = bs[i], b = bs[i + 1];
    double x = a;
    while (x < b) {
      double s = width(x) / (1 + alpha);
      if (!(s > 0)) throw std::runtime_error("graded_panels: non-positive width");
      double y = x + s >= b - 1e-14 * std::fabs(b) ? b : x + s;
      panels.push_back({x, y});
      if ((long)panels.size() > max_panels) throw std::runtime_error("graded_panels: too many panels");
      x = y;
    }
  }
  return panels;
}

// fixed_kρ_rule (mod_KSpaceFeatures.jl:396-419)
static void fixed_kr_rule(const Features& F, int order, double rtol, double alpha, int grade, double r_rel, double c_h,
                          double c_rho, double pole_safety, std::vector<double>& nodes, std::vector<double>& wts,
                          std::vector<std::pair<double, double>>& panels) {
  if (!(r_rel <= alpha)) throw std::runtime_error("fixed_kρ_rule: r_rel must be ≤ α");
  double rB = std::pow(1 / rtol, 1.0 / (2 * order));
  double eB = (rB - 1 / rB) / 2;
  auto wG = [&](double G) { return pole_safety * (2 * G) / eB; };
  double w_flat = std::min(c_h / F.h_min, F.rho_max > 0 ? c_rho / F.rho_max : INFINITY);
  double w_floor = F.kmax / 40;
  double g2 = std::ldexp(1.0, -grade);
  auto width = [&](double k) {
    double w = std::min(w_flat, std::max(r_rel * k, w_floor));
    for (double L : F.singular_lines) w = std::min(w, std::max(L * g2, alpha * std::fabs(k - L)));
    for (auto& c : F.cl) {
      double dist = k < c.a ? c.a - k : (k > c.b ? k - c.b : 0.0);
      w = std::min(w, std::max(wG(c.G), alpha * dist));
    }
    return w;
  };
  std::vector<double> breaks;
  breaks.push_back(0.0);
  for (double L : F.light_lines) if (L < F.Kcut) breaks.push_back(L);
  breaks.push_back(F.Kcut);
  panels = graded_panels(breaks, width, alpha);
  gl_rule(panels, order, F.singular_lines, nodes, wts);
}

// own_reflectance of the plane-wave comparison (comparisons/gila_airy/airy_comparison.jl:71-82)
static double own_reflectance(const Stack& st, double k0, double theta_deg, int pol_s) {
  double th = theta_deg * PI / 180.0;
  double kx = k0 * std::sin(th);
  std::vector<Modes> modes;
  if (!modes_stack(st, k0, kx, 0.0, modes)) return NAN;
  SAll S;
  s_all(st, modes, S);
  const M4& SR = S.SRight[0];
  double ct = std::cos(th);
  cd psi[4];
  if (pol_s) { psi[0] = 0.0; psi[1] = 1.0; psi[2] = -ct; psi[3] = 0.0; }
  else { psi[0] = ct; psi[1] = 0.0; psi[2] = 0.0; psi[3] = 1.0; }
  // a = Vf \ ψ_inc (4x2 least squares; the incident wave lies in span(Vf))
  const M42& Vf = modes[0].Vf;
  M2 N = mul(adj(Vf), Vf);
  V2 rhs;
  for (int i = 0; i < 2; ++i) { cd s = 0; for (int r = 0; r < 4; ++r) s += std::conj(Vf(r, i)) * psi[r]; rhs.v[i] = s; }
  V2 a = solve2<1>(N, rhs);
  V2 ra = mul(blk(SR, 1, 0), a);
  Mt<4, 1> pr = mul(modes[0].Vb, ra);
  return std::norm(pr.v[1]) + std::norm(pr.v[0]) / (ct * ct);
}

}  // namespace ytfo

// =====================================================================================
// C ABI (consumed by oracle/ytf_oracle.py through ctypes)
// =====================================================================================
using namespace ytfo;

static thread_local std::string g_err;

static Stack make_stack(int nL, const int* ekind, const int* mkind, const double* eps, const double* mu, const double* d) {
  Stack st(nL);
  for (int l = 0; l < nL; ++l) {
    st[l].ekind = ekind[l];
    st[l].mkind = mkind ? mkind[l] : ISO;
    for (int i = 0; i < 9; ++i) {
      st[l].eps[i] = cd(eps[2 * (9 * l + i)], eps[2 * (9 * l + i) + 1]);
      st[l].mu[i] = mu ? cd(mu[2 * (9 * l + i)], mu[2 * (9 * l + i) + 1]) : (i % 4 == 0 ? cd(1, 0) : cd(0, 0));
    }
    st[l].d = d[l];
  }
  return st;
}

extern "C" {

const char* ytfo_last_error() { return g_err.c_str(); }

void ytfo_set_zgeevx(void* fp) { g_zgeevx = (zgeevx_t)fp; }

int ytfo_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void ytfo_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// Berreman matrix of one layer (4x4 complex, column-major, interleaved re/im)
int ytfo_berreman(int ekind, int mkind, const double* eps, const double* mu, double w, double kx, double ky, double* out) {
  double dd = 1.0;
  Stack st = make_stack(1, &ekind, &mkind, eps, mu, &dd);
  M4 B = berreman_core(st[0], w, kx, ky);
  for (int i = 0; i < 16; ++i) { out[2 * i] = B.v[i].real(); out[2 * i + 1] = B.v[i].imag(); }
  return 0;
}

// Modes_Stack: per layer, Vf Vb Wf Wb (4x2 each), Qf Qb (2 each) = 36 complex per layer
int ytfo_modes_stack(int nL, const int* ekind, const int* mkind, const double* eps, const double* mu, const double* d,
                     double w, double kx, double ky, double* out) {
  try {
    Stack st = make_stack(nL, ekind, mkind, eps, mu, d);
    std::vector<Modes> modes;
    if (!modes_stack(st, w, kx, ky, modes)) { g_err = "mode sort overflow"; return 2; }
    for (int l = 0; l < nL; ++l) {
      double* o = out + 72 * l;
      int k = 0;
      auto put = [&](const cd& z) { o[2 * k] = z.real(); o[2 * k + 1] = z.imag(); ++k; };
      for (int i = 0; i < 8; ++i) put(modes[l].Vf.v[i]);
      for (int i = 0; i < 8; ++i) put(modes[l].Vb.v[i]);
      for (int i = 0; i < 8; ++i) put(modes[l].Wf.v[i]);
      for (int i = 0; i < 8; ++i) put(modes[l].Wb.v[i]);
      put(modes[l].Qf.v[0]); put(modes[l].Qf.v[1]); put(modes[l].Qb.v[0]); put(modes[l].Qb.v[1]);
    }
    return 0;
  } catch (std::exception& e) { g_err = e.what(); return 1; }
}

// S_all_Matrix: SLeft, SRight per layer (16 complex each) and Sint (N-1)
int ytfo_s_all(int nL, const int* ekind, const int* mkind, const double* eps, const double* mu, const double* d, double w,
               double kx, double ky, double* sleft, double* sright, double* sint) {
  try {
    Stack st = make_stack(nL, ekind, mkind, eps, mu, d);
    std::vector<Modes> modes;
    if (!modes_stack(st, w, kx, ky, modes)) { g_err = "mode sort overflow"; return 2; }
    SAll S;
    s_all(st, modes, S);
    for (int l = 0; l < nL; ++l)
      for (int i = 0; i < 16; ++i) {
        sleft[2 * (16 * l + i)] = S.SLeft[l].v[i].real(); sleft[2 * (16 * l + i) + 1] = S.SLeft[l].v[i].imag();
        sright[2 * (16 * l + i)] = S.SRight[l].v[i].real(); sright[2 * (16 * l + i) + 1] = S.SRight[l].v[i].imag();
      }
    for (int l = 0; l + 1 < nL; ++l)
      for (int i = 0; i < 16; ++i) { sint[2 * (16 * l + i)] = S.Sint[l].v[i].real(); sint[2 * (16 * l + i) + 1] = S.Sint[l].v[i].imag(); }
    return 0;
  } catch (std::exception& e) { g_err = e.what(); return 1; }
}

// Foundation identity data for one node, source layer, moment q and depth z:
// out: per obs layer o (1..N): T^o u (4 complex) and the direct reference (4 complex):
//   o != layer: [Ef; Eb] of Modal_amp; o == layer: Modal_amp_profile reflected part.
// Also returns the norm used by the reference test for the same-layer case.
int ytfo_foundation(int nL, const int* ekind, const int* mkind, const double* eps, const double* mu, const double* d,
                    double w, double kx, double ky, int layer, int q, double z, double* tu, double* ref, double* same_norm) {
  try {
    Stack st = make_stack(nL, ekind, mkind, eps, mu, d);
    int N = nL;
    std::vector<Modes> modes;
    if (!modes_stack(st, w, kx, ky, modes)) { g_err = "mode sort overflow"; return 2; }
    SAll S;
    s_all(st, modes, S);
    M23 sif, sib;
    source_projection(kx, ky, w, st[layer - 1], modes[layer - 1], sif, sib);
    std::vector<int> obs;
    for (int o = 1; o <= N; ++o) obs.push_back(o);
    std::vector<M4> T;
    cavity_transfer_columns(st, layer, modes, S, obs, T);
    Cav cv = r_cavity(st, layer, modes, S);
    double dd = cv.d;
    V2 s_f, s_b;
    s_f.v[0] = sif(0, q); s_f.v[1] = sif(1, q);
    s_b.v[0] = -sib(0, q); s_b.v[1] = -sib(1, q);
    double zpos = layer == 1 ? dd - z : z;
    V4 u;
    if (layer < N) { V2 pf = sprop2(dd - zpos, cv.Qf); u.v[0] = s_f.v[0] * pf.v[0]; u.v[1] = s_f.v[1] * pf.v[1]; }
    V2 pb = sprop2(-zpos, cv.Qb);
    u.v[2] = s_b.v[0] * pb.v[0]; u.v[3] = s_b.v[1] * pb.v[1];
    std::vector<V2> Ef, Eb;
    modal_amp(st, layer, z, s_f, s_b, modes, S, Ef, Eb);
    double zz[2] = {0.0, dd};
    V2 pEf[2], pEb[2];
    modal_amp_profile(st, layer, z, s_f, s_b, modes, S, 2, zz, pEf, pEb);
    for (int o = 1; o <= N; ++o) {
      V4 v = mul(T[o - 1], u);
      V4 r;
      if (o == layer) {
        V2 a = sprop2(-zpos, cv.Qf), b = sprop2(dd - zpos, cv.Qb);
        r.v[0] = pEf[1].v[0] - s_f.v[0] * a.v[0]; r.v[1] = pEf[1].v[1] - s_f.v[1] * a.v[1];
        r.v[2] = pEb[0].v[0] - s_b.v[0] * b.v[0]; r.v[3] = pEb[0].v[1] - s_b.v[1] * b.v[1];
        double nn = std::norm(pEf[1].v[0]) + std::norm(pEf[1].v[1]) + std::norm(pEb[0].v[0]) + std::norm(pEb[0].v[1]);
        same_norm[0] = std::sqrt(nn);
      } else {
        r.v[0] = Ef[o - 1].v[0]; r.v[1] = Ef[o - 1].v[1]; r.v[2] = Eb[o - 1].v[0]; r.v[3] = Eb[o - 1].v[1];
      }
      for (int i = 0; i < 4; ++i) {
        tu[2 * (4 * (o - 1) + i)] = v.v[i].real(); tu[2 * (4 * (o - 1) + i) + 1] = v.v[i].imag();
        ref[2 * (4 * (o - 1) + i)] = r.v[i].real(); ref[2 * (4 * (o - 1) + i) + 1] = r.v[i].imag();
      }
    }
    return 0;
  } catch (std::exception& e) { g_err = e.what(); return 1; }
}

// Build a transfer cache. kind2d = 0: 1D (kr = kx nodes, ky = 0). kind2d = 1: 2D with
// rotation fill per `rotation` (-1 auto, 0 full solve, 1 rotation).
void* ytfo_cache_build(int nL, const int* ekind, const int* mkind, const double* eps, const double* mu, const double* d,
                       double w, int src, int nobs, const int* obs, int kind2d, int nk, const double* kr, const double* wr,
                       int np, const double* phi, const double* wphi, int rotation) {
  try {
    Cache* c = new Cache();
    c->st = make_stack(nL, ekind, mkind, eps, mu, d);
    c->w = w; c->src = src;
    std::set<int> os(obs, obs + nobs);
    c->obs.assign(os.begin(), os.end());
    c->is2d = kind2d != 0;
    c->Nk = nk;
    c->kr.assign(kr, kr + nk); c->wr.assign(wr, wr + nk);
    if (c->is2d) {
      c->Np = np;
      c->phi.assign(phi, phi + np); c->wphi.assign(wphi, wphi + np);
      bool sym = azimuthally_symmetric(c->st);
      c->rotation = rotation < 0 ? sym : rotation != 0;
      build_2d(*c);
    } else {
      c->Np = 1;
      build_1d(*c);
    }
    return c;
  } catch (std::exception& e) { g_err = e.what(); return nullptr; }
}

void ytfo_cache_free(void* h) { delete (Cache*)h; }

// Export the cache arrays. Any pointer may be NULL. Complex arrays are interleaved.
//   valid[n], tvalid[nobs*n], T[nobs][n][16], Qf[n][2], Qb[n][2], sf[n][6], sb[n][6] (column-major 2x3),
//   basis[nobs][n][16]: exf0 exf1 eyf0 eyf1 ezf0 ezf1 exb0 exb1 eyb0 eyb1 ezb0 ezb1 kzf0 kzf1 kzb0 kzb1
int ytfo_cache_export(void* h, unsigned char* valid, unsigned char* tvalid, double* T, double* Qf, double* Qb, double* sf,
                      double* sb, double* basis) {
  Cache* c = (Cache*)h;
  int n = c->n(), no = (int)c->obs.size();
  auto put = [](double* o, size_t i, const cd& z) { o[2 * i] = z.real(); o[2 * i + 1] = z.imag(); };
  for (int k = 0; k < n; ++k) {
    if (valid) valid[k] = c->valid[k];
    if (Qf) { put(Qf, 2 * k, c->Qf[k].v[0]); put(Qf, 2 * k + 1, c->Qf[k].v[1]); }
    if (Qb) { put(Qb, 2 * k, c->Qb[k].v[0]); put(Qb, 2 * k + 1, c->Qb[k].v[1]); }
    for (int i = 0; i < 6; ++i) {
      if (sf) put(sf, 6 * k + i, c->sf[k].v[i]);
      if (sb) put(sb, 6 * k + i, c->sb[k].v[i]);
    }
    for (int o = 0; o < no; ++o) {
      if (tvalid) tvalid[(size_t)o * n + k] = c->Tvalid[o][k];
      if (T) for (int i = 0; i < 16; ++i) put(T, ((size_t)o * n + k) * 16 + i, c->T[o][k].v[i]);
      if (basis) {
        const Basis& b = c->basis[o][k];
        size_t base = ((size_t)o * n + k) * 16;
        for (int m = 0; m < 2; ++m) {
          put(basis, base + 0 + m, b.exf[m]); put(basis, base + 2 + m, b.eyf[m]); put(basis, base + 4 + m, b.ezf[m]);
          put(basis, base + 6 + m, b.exb[m]); put(basis, base + 8 + m, b.eyb[m]); put(basis, base + 10 + m, b.ezb[m]);
          put(basis, base + 12 + m, b.kzf[m]); put(basis, base + 14 + m, b.kzb[m]);
        }
      }
    }
  }
  return 0;
}

int ytfo_green(void* h, int obs_layer, double zsrc, int nz, const double* zo, int nx, const double* xs, int ny,
               const double* ys, int terms, double* G) {
  try {
    Cache* c = (Cache*)h;
    if (c->is2d) green_2d(*c, obs_layer, zsrc, nz, zo, nx, xs, ny, ys, terms, (cd*)G);
    else green_1d(*c, obs_layer, zsrc, nz, zo, nx, xs, ny, ys, terms, (cd*)G);
    return 0;
  } catch (std::exception& e) { g_err = e.what(); return 1; }
}

// amplitude_at: Af, Ab as [n][2][3] complex
int ytfo_amplitude_at(void* h, int obs_layer, double zsrc, int seeds, double* Af, double* Ab) {
  try {
    Cache* c = (Cache*)h;
    Amp A;
    amplitude_at(*c, obs_layer, zsrc, seeds == 2 ? 0.0 : 1.0, seeds == 1 ? 0.0 : 1.0, A);
    std::memcpy(Af, A.f.data(), A.f.size() * sizeof(cd));
    std::memcpy(Ab, A.b.data(), A.b.size() * sizeof(cd));
    return 0;
  } catch (std::exception& e) { g_err = e.what(); return 1; }
}

// Strengths of one z-row of a 2D cache (_strengths_row!, mod_ClosedFormField.jl:616-659):
// S[n][c + 3q] complex, and the node wavevectors kx[n], ky[n].
int ytfo_strengths_2d(void* h, int obs_layer, double zsrc, double z, int terms, double* S, double* kx, double* ky) {
  try {
    Cache* c = (Cache*)h;
    if (!c->is2d) throw std::runtime_error("needs a 2D cache");
    int oi = c->oidx(obs_layer);
    if (oi < 0) throw std::runtime_error("obs layer not in cache");
    int Nk = c->Nk, Np = c->Np, Nn = Nk * Np;
    Amp R;
    bool same = term_amplitudes(*c, obs_layer, zsrc, terms, R);
    Amp D;
    if (same) direct_amplitude(*c, zsrc, z, D);
    double d = c->d_obs[oi];
    for (int p = 0; p < Np; ++p)
      for (int k = 0; k < Nk; ++k) {
        int n = k + Nk * p;
        cd w(c->kr[k] * c->wr[k] * c->wphi[p] / (4 * PI * PI), 0.0);
        cd sacc[3][3];
        for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) sacc[a][b] = 0.0;
        const Basis& b = c->basis[oi][n];
        for (int m = 0; m < 2; ++m) {
          cd pf = phase(b.kzf[m], z), pb = phase(b.kzb[m], z - d);
          for (int q = 0; q < 3; ++q) {
            cd af_ = R.F(n, m, q) * pf, ab_ = R.B(n, m, q) * pb;
            if (same) { af_ += D.F(n, m, q); ab_ += D.B(n, m, q); }
            cd af = finite_or_zero(w * af_), ab = finite_or_zero(w * ab_);
            sacc[0][q] += b.exf[m] * af + b.exb[m] * ab;
            sacc[1][q] += b.eyf[m] * af + b.eyb[m] * ab;
            sacc[2][q] += b.ezf[m] * af + b.ezb[m] * ab;
          }
        }
        for (int q = 0; q < 3; ++q)
          for (int cc = 0; cc < 3; ++cc) {
            S[2 * (9 * (size_t)n + cc + 3 * q)] = sacc[cc][q].real();
            S[2 * (9 * (size_t)n + cc + 3 * q) + 1] = sacc[cc][q].imag();
          }
        kx[n] = c->kxn[n];
        ky[n] = c->kyn[n];
      }
    return 0;
  } catch (std::exception& e) { g_err = e.what(); return 1; }
}

int ytfo_gauss_legendre(int n, double* x, double* w) {
  std::vector<double> xv, wv;
  gauss_legendre(n, xv, wv);
  std::memcpy(x, xv.data(), n * sizeof(double));
  std::memcpy(w, wv.data(), n * sizeof(double));
  return 0;
}

// gl_rule on explicit panels (pa, pb), singular values; out arrays sized np*order
int ytfo_gl_rule(int np, const double* pa, const double* pb, int order, int ns, const double* sing, double* nodes, double* wts) {
  std::vector<std::pair<double, double>> p(np);
  for (int i = 0; i < np; ++i) p[i] = {pa[i], pb[i]};
  std::vector<double> s(sing, sing + ns), nd, wt;
  gl_rule(p, order, s, nd, wt);
  std::memcpy(nodes, nd.data(), nd.size() * sizeof(double));
  std::memcpy(wts, wt.data(), wt.size() * sizeof(double));
  return 0;
}

int ytfo_light_lines(int ekind, int mkind, const double* eps, const double* mu, double w, double phi, double* out, int* n) {
  double dd = 1.0;
  Stack st = make_stack(1, &ekind, &mkind, eps, mu, &dd);
  auto L = layer_light_lines(st[0], w, phi);
  *n = (int)L.size();
  for (size_t i = 0; i < L.size(); ++i) out[i] = L[i];
  return 0;
}

int ytfo_material_class(int ekind, int mkind, const double* eps, const double* mu) {
  double dd = 1.0;
  Stack st = make_stack(1, &ekind, &mkind, eps, mu, &dd);
  return material_class(st[0]);
}

double ytfo_cavity_response(int nL, const int* ekind, const int* mkind, const double* eps, const double* mu,
                            const double* d, double w, int s, double kr, double phi) {
  Stack st = make_stack(nL, ekind, mkind, eps, mu, d);
  return cavity_response(st, w, s, kr, phi);
}

// point grid of the :fixed engine for a 1D stack: kspace_features(dims=1) + fixed_kρ_rule.
// Two-call protocol: first with nodes == NULL returns the count in *n.
int ytfo_fixed_grid_1d(int nL, const int* ekind, const int* mkind, const double* eps, const double* mu, const double* d,
                       double w, int src, double h_min, double rho_max, double target_decay, double kr_cap, int scan,
                       int order, double rtol, double* nodes, double* wts, int* n, double* info) {
  try {
    Stack st = make_stack(nL, ekind, mkind, eps, mu, d);
    Features F = kspace_features_1d(st, w, src, h_min, rho_max, target_decay, kr_cap, 1e5, scan != 0, 1e-3, 1.05);
    std::vector<double> nd, wt;
    std::vector<std::pair<double, double>> panels;
    fixed_kr_rule(F, order, rtol, 0.5, 12, 0.05, 4.0, 4.0, 0.5, nd, wt, panels);
    *n = (int)nd.size();
    if (info) { info[0] = F.Kcut; info[1] = F.kmax; info[2] = (double)F.poles.size(); info[3] = (double)panels.size(); }
    if (nodes) { std::memcpy(nodes, nd.data(), nd.size() * sizeof(double)); std::memcpy(wts, wt.data(), wt.size() * sizeof(double)); }
    return 0;
  } catch (std::exception& e) { g_err = e.what(); return 1; }
}

// adaptive_seeds (mod_KSpaceFeatures.jl:421-445) of kspace_features(dims = 1): light lines,
// L (1 ± 2^-j) for j = 1..grade at the singular lines (grade = _grade_for(rtol) =
// min(50, ceil(2 log2(10/rtol)))), [a - 4Γ, a, b, b + 4Γ] per cluster, 2 kmax, 4 kmax, ...
// below Kcut; kept in (0, Kcut), unique, sorted.
int ytfo_adaptive_seeds(int nL, const int* ekind, const int* mkind, const double* eps, const double* mu, const double* d,
                        double w, int src, double h_min, double rho_max, double target_decay, double kr_cap, int scan,
                        double rtol, double* seeds, int* n) {
  try {
    Stack st = make_stack(nL, ekind, mkind, eps, mu, d);
    Features F = kspace_features_1d(st, w, src, h_min, rho_max, target_decay, kr_cap, 1e5, scan != 0, 1e-3, 1.05);
    const int grade = std::min(50, (int)std::ceil(2 * std::log2(10 / rtol)));
    std::vector<double> s = F.light_lines;
    for (double L : F.singular_lines)
      for (int j = 1; j <= grade; ++j) { s.push_back(L * (1 - std::ldexp(1.0, -j))); s.push_back(L * (1 + std::ldexp(1.0, -j))); }
    for (auto& c : F.cl) { s.push_back(c.a - 4.0 * c.G); s.push_back(c.a); s.push_back(c.b); s.push_back(c.b + 4.0 * c.G); }
    for (double k = 2 * F.kmax; k < F.Kcut; k *= 2) s.push_back(k);
    std::vector<double> o;
    for (double x : s) if (0 < x && x < F.Kcut && std::find(o.begin(), o.end(), x) == o.end()) o.push_back(x);
    std::sort(o.begin(), o.end());
    *n = (int)o.size();
    if (seeds) std::memcpy(seeds, o.data(), o.size() * sizeof(double));
    return 0;
  } catch (std::exception& e) { g_err = e.what(); return 1; }
}

// point_kρ_grid_2d (mod_ClosedFormGrid.jl:536-585) with an explicit h_min: kspace_features
// (dims = 2) + fixed_kρ_rule; the kρ rule, and N_φ of the uniform φ trapezoid.
// info: Kcut, kmax, poles, panels, N_φ.
int ytfo_fixed_grid_2d(int nL, const int* ekind, const int* mkind, const double* eps, const double* mu, const double* d,
                       double w, int src, double h_min, double rho_max, double target_decay, double kr_cap, int scan,
                       int order, double rtol, int n_phi_scan, double* nodes, double* wts, int* n, double* info) {
  try {
    Stack st = make_stack(nL, ekind, mkind, eps, mu, d);
    Features F = kspace_features_2d(st, w, src, h_min, rho_max, target_decay, kr_cap, 1e5, scan != 0, 1e-3, 1.05,
                                    n_phi_scan, 2.5, 64, rtol, 1.5);
    std::vector<double> nd, wt;
    std::vector<std::pair<double, double>> panels;
    fixed_kr_rule(F, order, rtol, 0.5, 12, 0.05, 4.0, 4.0, 0.5, nd, wt, panels);
    *n = (int)nd.size();
    if (info) {
      info[0] = F.Kcut; info[1] = F.kmax; info[2] = (double)F.poles.size(); info[3] = (double)panels.size();
      info[4] = (double)F.N_phi;
    }
    if (nodes) { std::memcpy(nodes, nd.data(), nd.size() * sizeof(double)); std::memcpy(wts, wt.data(), wt.size() * sizeof(double)); }
    return 0;
  } catch (std::exception& e) { g_err = e.what(); return 1; }
}

double ytfo_own_reflectance(int nL, const int* ekind, const int* mkind, const double* eps, const double* mu, const double* d,
                            double k0, double theta_deg, int pol_s) {
  try {
    Stack st = make_stack(nL, ekind, mkind, eps, mu, d);
    return own_reflectance(st, k0, theta_deg, pol_s);
  } catch (std::exception& e) { g_err = e.what(); return NAN; }
}

}  // extern "C"

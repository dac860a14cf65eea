// ytf_transfer.cu -- per-k-node spectral solve on sm_100a: Berreman modes, S-matrix
// cascade, cavity transfer map T^o, source projection and observation-layer mode basis.
//
// Replaces build_cavity_transfer_1d / build_cavity_transfer_2d
// (mod_CavityTransfer.jl:196-258, 307-398) and everything they call per node
// (mod_ModeSolver.jl, mod_ScatteringMatrix.jl, mod_FieldSolver.jl:72-341,
// mod_SourceProj.jl:34-60).
//
// Work decomposition (B200-first, not a translation of the reference's loops):
//   k_layer_modes : one thread per (node, layer). Closed-form TE/TM modes for
//                   isotropic/uniaxial layers, otherwise a balanced complex Hessenberg QR
//                   of the 4x4 Berreman matrix. Eigenvectors are normalised as LAPACK's
//                   ZGEEVX does (unit 2-norm), eigenpairs sorted by (real, imag) as Julia's
//                   eigen, then split forward/backward by Poynting flux. Layer-major
//                   indexing keeps one layer (one material kind) per warp: no divergence
//                   between the closed-form and the general path.
//   k_chain       : one thread per node. Mode matching through the stack, interface
//                   matrices, forward/backward Redheffer scans, cavity resummation, the
//                   stack walk reduced to the observation layers, T^o, seeds and basis.
//   k_rotate_fill : one thread per (kρ, φ) node of an azimuthally symmetric 2D grid: the
//                   φ = 0 solve rotated exactly (mod_ModeSolver.jl:471-482).
// Per-(node, layer) intermediates live in a global scratch arena, structure-of-arrays
// with the node index fastest, so every warp access is one contiguous 512-byte line.
// All arithmetic is FP64 (B200 runs FP64 at half the FP32 rate; the branchy mode
// classification and the near-singular 2x2 solves keep the reference's FP64 semantics).
#include "ytf_complex.cuh"
#include "ytf_kernels.h"

namespace ytf {

// ------------------------------------------------------------------------------------
// scratch / output accessors (SoA: element-major, node fastest)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ cd ld(const double2* base, long elem, long n, long node) {
  double2 v = base[elem * n + node];
  return cd{v.x, v.y};
}
__device__ __forceinline__ void st(double2* base, long elem, long n, long node, cd v) {
  base[elem * n + node] = make_double2(v.x, v.y);
}

__device__ __forceinline__ const cd& E(const LayerDev& L, int i, int j) { return *reinterpret_cast<const cd*>(&L.eps[2 * ((i - 1) + 3 * (j - 1))]); }
__device__ __forceinline__ const cd& U(const LayerDev& L, int i, int j) { return *reinterpret_cast<const cd*>(&L.mu[2 * ((i - 1) + 3 * (j - 1))]); }

// in-plane wave vector of a node: real except for 1D nodes on a deformed contour (kr_im)
__device__ __forceinline__ void node_k(const TransferParams& p, long node, cd& kx, cd& ky) {
  if (p.mode == 0) {  // 1D radial nodes kt = (kx, 0)
    kx = cd{p.kr[node], p.kr_im ? p.kr_im[node] : 0.0};
    ky = cd{0.0, 0.0};
  } else if (p.mode == 1) {  // full 2D solve, node = k + Nk * q
    long k = node % p.Nk, q = node / p.Nk;
    double s, c;
    sincos(p.phi[q], &s, &c);
    kx = cd{p.kr[k] * c, 0.0};
    ky = cd{p.kr[k] * s, 0.0};
  } else {  // rotation base: φ = 0
    kx = cd{p.kr[node] * 1.0, 0.0};
    ky = cd{p.kr[node] * 0.0, 0.0};
  }
}

// ------------------------------------------------------------------------------------
// Berreman matrix (mod_ModeSolver.jl:122-193), real in-plane wavevector
// ------------------------------------------------------------------------------------
// kt enters as a complex pair: real on the real axis; on a deformed contour the matrix is the
// analytic continuation (no conjugation of kt anywhere, which changes nothing for real kt)
__device__ void berreman(const LayerDev& L, double w, cd kx, cd ky, cd B[4][4]) {
  cd e11 = E(L, 1, 1), e12 = E(L, 1, 2), e21 = E(L, 2, 1), e22 = E(L, 2, 2);
  cd e13 = E(L, 1, 3), e23 = E(L, 2, 3), e31 = E(L, 3, 1), e32 = E(L, 3, 2), e33 = E(L, 3, 3);
  cd m11 = U(L, 1, 1), m12 = U(L, 1, 2), m21 = U(L, 2, 1), m22 = U(L, 2, 2);
  cd m13 = U(L, 1, 3), m23 = U(L, 2, 3), m31 = U(L, 3, 1), m32 = U(L, 3, 2), m33 = U(L, 3, 3);
  const cd k1 = kx, k2 = ky;
  cd de = recip(e33), dm = recip(m33);
  cd iw{1.0 / w, 0.0};
  cd Se11 = e11 - e13 * de * e31, Se12 = e12 - e13 * de * e32;
  cd Se21 = e21 - e23 * de * e31, Se22 = e22 - e23 * de * e32;
  cd Sm11 = m11 - m13 * dm * m31, Sm12 = m12 - m13 * dm * m32;
  cd Sm21 = m21 - m23 * dm * m31, Sm22 = m22 - m23 * dm * m32;
  cd re1 = de * e31, re2 = de * e32, se1 = e13 * de, se2 = e23 * de;
  cd rm1 = dm * m31, rm2 = dm * m32, sm1 = m13 * dm, sm2 = m23 * dm;
  cd t21 = -k2, t22 = k1;
  cd t31 = iw * k1, t32 = iw * k2;
  cd Rsm1 = sm2, Rsm2 = -sm1, Rse1 = se2, Rse2 = -se1;
  B[0][0] = Rsm1 * t21 - k1 * re1; B[0][1] = Rsm1 * t22 - k1 * re2;
  B[1][0] = Rsm2 * t21 - k2 * re1; B[1][1] = Rsm2 * t22 - k2 * re2;
  B[0][2] = w * Sm21 - t31 * de * t21; B[0][3] = w * Sm22 - t31 * de * t22;
  B[1][2] = (-w) * Sm11 - t32 * de * t21; B[1][3] = (-w) * Sm12 - t32 * de * t22;
  B[2][0] = t31 * dm * t21 - w * Se21; B[2][1] = t31 * dm * t22 - w * Se22;
  B[3][0] = t32 * dm * t21 - (-w) * Se11; B[3][1] = t32 * dm * t22 - (-w) * Se12;
  B[2][2] = Rse1 * t21 - k1 * rm1; B[2][3] = Rse1 * t22 - k1 * rm2;
  B[3][2] = Rse2 * t21 - k2 * rm1; B[3][3] = Rse2 * t22 - k2 * rm2;
}

// ------------------------------------------------------------------------------------
// General 4x4 complex eigen solve: diagonal balancing, Householder reduction to
// Hessenberg form, single-shift complex QR with Wilkinson shifts and full Schur-vector
// accumulation, eigenvectors of the triangular factor by back substitution.
// Published algorithm (Golub & Van Loan, Matrix Computations, §7.4-7.6; the LAPACK
// ZGEBAL/ZGEHRD/ZLAHQR/ZTREVC sequence). Every array index is a compile-time constant
// (the active QR window is a template parameter, the sweep start a predicate), so the
// matrices stay in registers. Returns false if QR does not converge.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void givens(cd x, cd y, cd& c, cd& s) {
  double ax = cabs(x), ay = cabs(y);
  if (ay == 0.0) { c = cd{1.0, 0.0}; s = cd{0.0, 0.0}; return; }
  if (ax == 0.0) { c = cd{0.0, 0.0}; s = conj(y) * (1.0 / ay); return; }
  double nr = hypot(ax, ay);
  c = cd{ax / nr, 0.0};
  s = (x * (1.0 / ax)) * conj(y) * (1.0 / nr);
}

// QR iterations on the window [l, HI] until H[HI][HI-1] deflates
template <int HI>
__device__ __forceinline__ bool qr_window(cd H[4][4], cd Z[4][4]) {
  const double eps = 2.220446049250313e-16;
  for (int it = 0; it < 60; ++it) {
    int l = 0;
#pragma unroll
    for (int m = HI; m >= 1; --m) {
      if (l == 0) {
        double sm = cabs1(H[m - 1][m - 1]) + cabs1(H[m][m]);
        if (cabs1(H[m][m - 1]) <= eps * sm || cabs1(H[m][m - 1]) < 1e-300) {
          H[m][m - 1] = cd{0.0, 0.0};
          l = m;
        }
      }
    }
    if (l == HI) return true;
    cd mu;
    if (it == 10 || it == 20 || it == 40) {
      mu = H[HI][HI] + cd{0.75 * fabs(H[HI][HI - 1].x), 0.0};  // exceptional shift
    } else {
      cd a = H[HI - 1][HI - 1], b = H[HI - 1][HI], c = H[HI][HI - 1], d = H[HI][HI];
      cd hd = (a - d) * 0.5;
      cd disc = csqrt(hd * hd + b * c);
      cd m1 = iszero(hd + disc) ? d : d - (b * c) / (hd + disc);
      cd m2 = iszero(hd - disc) ? d : d - (b * c) / (hd - disc);
      mu = norm2(m1 - d) <= norm2(m2 - d) ? m1 : m2;
      if (!isfin(mu)) mu = d;
    }
    cd x{0.0, 0.0}, y{0.0, 0.0};
#pragma unroll
    for (int m = 0; m < HI; ++m)
      if (m == l) { x = H[m][m] - mu; y = H[m + 1][m]; }
#pragma unroll
    for (int k = 0; k < HI; ++k) {
      if (k < l) continue;
      if (k > l) { x = H[k][k - 1]; y = H[k + 1][k - 1]; }
      cd c, s;
      givens(x, y, c, s);
      // rows k, k+1 of H; columns k, k+1 of H and Z (entries outside the Hessenberg band
      // are exact zeros and stay zero)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        cd h1 = H[k][j], h2 = H[k + 1][j];
        H[k][j] = c * h1 + s * h2;
        H[k + 1][j] = c * h2 - conj(s) * h1;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        cd h1 = H[i][k], h2 = H[i][k + 1];
        H[i][k] = c * h1 + conj(s) * h2;
        H[i][k + 1] = c * h2 - s * h1;
        cd z1 = Z[i][k], z2 = Z[i][k + 1];
        Z[i][k] = c * z1 + conj(s) * z2;
        Z[i][k + 1] = c * z2 - s * z1;
      }
      if (k > l) H[k + 1][k - 1] = cd{0.0, 0.0};
    }
  }
  return false;
}

__device__ bool eig4(cd A[4][4], cd lam[4], cd V[4][4]) {
  // balancing by powers of 2 (scaling only, as ZGEBAL with job 'S')
  double D[4] = {1.0, 1.0, 1.0, 1.0};
  for (int sweep = 0; sweep < 8; ++sweep) {
    bool changed = false;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      double c = 0.0, r = 0.0;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j != i) { c += cabs1(A[j][i]); r += cabs1(A[i][j]); }
      if (c == 0.0 || r == 0.0) continue;
      double s = c + r, f = 1.0, g = r / 2.0;
      while (c < g && f < 1e150) { f *= 2.0; c *= 2.0; r /= 2.0; g /= 2.0; }
      g = c / 2.0;
      while (g >= r && f > 1e-150) { f /= 2.0; c /= 2.0; g /= 2.0; r *= 2.0; }
      if (c + r >= 0.95 * s) continue;
      changed = true;
      D[i] *= f;
      const double fi = 1.0 / f;
#pragma unroll
      for (int j = 0; j < 4; ++j) { A[i][j] = A[i][j] * fi; A[j][i] = A[j][i] * f; }
    }
    if (!changed) break;
  }
  cd Z[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) Z[i][j] = cd{i == j ? 1.0 : 0.0, 0.0};
  // Householder reduction to upper Hessenberg
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    double xn = 0.0;
#pragma unroll
    for (int i = k + 1; i < 4; ++i) xn += norm2(A[i][k]);
    if (xn == 0.0) continue;
    xn = sqrt(xn);
    cd a = A[k + 1][k];
    double aa = cabs(a);
    cd ph = aa > 0.0 ? a * (1.0 / aa) : cd{1.0, 0.0};
    cd v[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    v[k + 1] = a + ph * xn;
#pragma unroll
    for (int i = k + 2; i < 4; ++i) v[i] = A[i][k];
    double vn = 0.0;
#pragma unroll
    for (int i = k + 1; i < 4; ++i) vn += norm2(v[i]);
    if (vn == 0.0) continue;
    const double tau = 2.0 / vn;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      cd s{0, 0};
#pragma unroll
      for (int i = k + 1; i < 4; ++i) s += conj(v[i]) * A[i][j];
      s = s * tau;
#pragma unroll
      for (int i = k + 1; i < 4; ++i) A[i][j] -= v[i] * s;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      cd s{0, 0}, t{0, 0};
#pragma unroll
      for (int j = k + 1; j < 4; ++j) { s += A[i][j] * v[j]; t += Z[i][j] * v[j]; }
      s = s * tau;
      t = t * tau;
#pragma unroll
      for (int j = k + 1; j < 4; ++j) { A[i][j] -= s * conj(v[j]); Z[i][j] -= t * conj(v[j]); }
    }
#pragma unroll
    for (int i = k + 2; i < 4; ++i) A[i][k] = cd{0, 0};
  }
  if (!qr_window<3>(A, Z)) return false;
  if (!qr_window<2>(A, Z)) return false;
  if (!qr_window<1>(A, Z)) return false;
#pragma unroll
  for (int i = 0; i < 4; ++i) lam[i] = A[i][i];
  // eigenvectors of the upper-triangular Schur factor
  const double eps = 2.220446049250313e-16;
  double anorm = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = i; j < 4; ++j) anorm = fmax(anorm, cabs1(A[i][j]));
  const double smin = fmax(eps * anorm, 1e-290);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    cd xv[4] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}};
    xv[k] = cd{1.0, 0.0};
#pragma unroll
    for (int i = k - 1; i >= 0; --i) {
      cd s{0, 0};
#pragma unroll
      for (int j = i + 1; j <= k; ++j) s += A[i][j] * xv[j];
      cd den = A[i][i] - A[k][k];
      if (cabs1(den) < smin) den = cd{smin, 0.0};
      xv[i] = -(s / den);
    }
    cd v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      cd s{0, 0};
#pragma unroll
      for (int j = 0; j <= k; ++j) s += Z[i][j] * xv[j];
      v[i] = s * D[i];
    }
    // LAPACK normalisation: unit 2-norm, largest component real
    double nn = 0.0, best = -1.0;
    cd vb{1.0, 0.0};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      double a2 = norm2(v[i]);
      nn += a2;
      if (a2 > best) { best = a2; vb = v[i]; }
    }
    const double inv = rsqrt(nn);
    const cd ph = conj(vb) * rsqrt(best);
#pragma unroll
    for (int i = 0; i < 4; ++i) V[i][k] = (v[i] * ph) * inv;
  }
  // sort eigenpairs by (real, imag) (Julia's eigsortby): a 4-input sorting network
  auto cswap = [&](int a, int b) {
    bool sw = lam[b].x < lam[a].x || (lam[b].x == lam[a].x && lam[b].y < lam[a].y);
    if (sw) {
      cd t = lam[a]; lam[a] = lam[b]; lam[b] = t;
#pragma unroll
      for (int r = 0; r < 4; ++r) { cd u = V[r][a]; V[r][a] = V[r][b]; V[r][b] = u; }
    }
  };
  cswap(0, 1); cswap(2, 3); cswap(0, 2); cswap(1, 3); cswap(1, 2);
  return true;
}

// closed-form TE/TM modes (mod_ModeSolver.jl:243-265)
__device__ void closed_modes(const LayerDev& L, double w, cd kx, cd ky, cd Q[4], cd V[4][4]) {
  cd et = E(L, 1, 1), ez = E(L, 3, 3), mr = U(L, 1, 1);
  cd wc{w, 0.0};
  double s, c;
  cd kr2;
  if (kx.y == 0.0 && ky.y == 0.0) {
    const double kr = hypot(kx.x, ky.x);
    const double phi = kr == 0 ? 0.0 : atan2(ky.x, kx.x);
    sincos(phi, &s, &c);
    kr2 = cd{kr * kr, 0.0};
  } else {  // complex 1D node on a deformed contour: direction (1, 0), kt² = kx²
    s = 0.0;
    c = 1.0;
    kr2 = kx * kx + ky * ky;
  }
  cd kzo = csqrt(wc * wc * et * mr - kr2);
  cd kze = csqrt(et * (wc * wc * mr - kr2 / ez));
  cd A = recip(wc * mr), Bn = recip(wc * et);
  cd mA = -A, mB = -Bn;
  V[0][0] = cd{-s, 0}; V[1][0] = cd{c, 0}; V[2][0] = mA * kzo * c; V[3][0] = mA * kzo * s;
  V[0][1] = cd{-s, 0}; V[1][1] = cd{c, 0}; V[2][1] = A * kzo * c; V[3][1] = A * kzo * s;
  V[0][2] = Bn * kze * c; V[1][2] = Bn * kze * s; V[2][2] = cd{-s, 0}; V[3][2] = cd{c, 0};
  V[0][3] = mB * kze * c; V[1][3] = mB * kze * s; V[2][3] = cd{-s, 0}; V[3][3] = cd{c, 0};
  Q[0] = kzo; Q[1] = -kzo; Q[2] = kze; Q[3] = -kze;
}

// ------------------------------------------------------------------------------------
// Layers without xz/yz coupling (ε13 = ε23 = ε31 = ε32 = 0 and the same for μ: every
// biaxial and every ε_xy-gyrotropic layer) have ρ = σ = 0 in the Berreman construction, so
// B = [[0, B12], [B21, 0]] and B² = diag(B12 B21, B21 B12). The eigenvalues are
// q = ±√μ_i with μ_i the eigenvalues of the 2x2 matrix M = B12 B21, and the eigenvectors
// (a; ±B21 a / q) with M a = μ_i a. Returns false (general QR path) when the two μ_i are
// within 1e-6 of each other or q ≈ 0, where this construction loses accuracy.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ bool no_z_coupling(const LayerDev& L) {
  return iszero(E(L, 1, 3)) && iszero(E(L, 2, 3)) && iszero(E(L, 3, 1)) && iszero(E(L, 3, 2)) && iszero(U(L, 1, 3)) &&
         iszero(U(L, 2, 3)) && iszero(U(L, 3, 1)) && iszero(U(L, 3, 2));
}

__device__ bool block_modes(const LayerDev& L, double w, cd kx, cd ky, cd Q[4], cd V[4][4]) {
  cd B[4][4];
  berreman(L, w, kx, ky, B);
  // M = B12 B21 (B12 = rows 0-1, cols 2-3; B21 = rows 2-3, cols 0-1)
  cd m11 = B[0][2] * B[2][0] + B[0][3] * B[3][0], m12 = B[0][2] * B[2][1] + B[0][3] * B[3][1];
  cd m21 = B[1][2] * B[2][0] + B[1][3] * B[3][0], m22 = B[1][2] * B[2][1] + B[1][3] * B[3][1];
  cd hd = (m11 - m22) * 0.5;
  cd disc = csqrt(hd * hd + m12 * m21);
  cd mid = (m11 + m22) * 0.5;
  cd mu[2] = {mid + disc, mid - disc};
  double scale = fmax(fmax(cabs(m11), cabs(m22)), fmax(cabs(m12), cabs(m21)));
  if (!(scale > 0) || !isfinite(scale)) return false;
  if (cabs(mu[0] - mu[1]) <= 1e-6 * fmax(cabs(mu[0]), cabs(mu[1]))) return false;
  int col = 0;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    // eigenvector of M for mu_i: (m12, mu_i - m11) or (mu_i - m22, m21), the larger one;
    // mu_i - m11 = -hd ± disc and mu_i - m22 = hd ± disc, formed without cancellation
    const cd sg = i == 0 ? disc : -disc;
    cd a1x = m12, a1y = sg - hd;
    cd a2x = hd + sg, a2y = m21;
    double n1 = norm2(a1x) + norm2(a1y), n2 = norm2(a2x) + norm2(a2y);
    cd ax = n1 >= n2 ? a1x : a2x, ay = n1 >= n2 ? a1y : a2y;
    if (!(fmax(n1, n2) > 0)) return false;
    cd q = csqrt(mu[i]);
    if (!(cabs(q) > 1e-12 * sqrt(scale))) return false;
    // b = B21 a / q
    const cd rq = recip(q);
    cd bx = (B[2][0] * ax + B[2][1] * ay) * rq, by = (B[3][0] * ax + B[3][1] * ay) * rq;
#pragma unroll
    for (int sgn = 0; sgn < 2; ++sgn) {
      cd v[4] = {ax, ay, sgn ? -bx : bx, sgn ? -by : by};
      double nn = 0.0, best = -1.0;
      cd vb{1.0, 0.0};
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        double a2 = norm2(v[r]);
        nn += a2;
        if (a2 > best) { best = a2; vb = v[r]; }
      }
      const double inv = rsqrt(nn);  // unit 2-norm, largest component real (ZGEEVX)
      const cd ph = conj(vb) * rsqrt(best);
#pragma unroll
      for (int r = 0; r < 4; ++r) V[r][col] = (v[r] * ph) * inv;
      Q[col] = sgn ? -q : q;
      ++col;
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c)
    if (!isfin(Q[c]) || !isfin(V[0][c]) || !isfin(V[1][c]) || !isfin(V[2][c]) || !isfin(V[3][c])) return false;
  // sort eigenpairs by (real, imag) (Julia's eigsortby): a 4-input sorting network
  auto cswap = [&](int x, int y) {
    bool sw = Q[y].x < Q[x].x || (Q[y].x == Q[x].x && Q[y].y < Q[x].y);
    if (sw) {
      cd t = Q[x]; Q[x] = Q[y]; Q[y] = t;
#pragma unroll
      for (int r = 0; r < 4; ++r) { cd u = V[r][x]; V[r][x] = V[r][y]; V[r][y] = u; }
    }
  };
  cswap(0, 1); cswap(2, 3); cswap(0, 2); cswap(1, 3); cswap(1, 2);
  return true;
}

// Forward/backward split of one layer's four eigenpairs (mod_ModeSolver.jl:274-326) and
// the scratch record: Vf[4x2] (8), Vb[4x2] (8), Qf (2), Qb (2); column-major. Each
// eigenpair is written straight to its slot, so no register array is indexed at run time.
__device__ __forceinline__ uint8_t classify_store(const TransferParams& p, int layer, long node, const cd Q[4],
                                                  const cd V[4][4]) {
  const long n = p.n;
  const double tol = 1.4901161193847656e-08;
  // complex nodes (a deformed contour, or circles around complex poles): the two half-spaces
  // take the proper sheet, the wave that decays away from the stack (Im Q > 0) as forward,
  // so the integrand is the analytic continuation of its real-axis values on both sides of
  // the real axis (the principal square root alone gives the growing wave above it, past the
  // half-space's light line). On the real axis and below it the two rules agree.
  const bool proper = p.kr_im && (layer == 0 || layer == p.nL - 1);
  int cls[4];  // 0 forward, 1 backward, 2 degenerate
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    // Poynting flux Pz = ¼ Re(V_j · W_j), W = R4s V = (V3, -V2, -V1, V0)
    cd s = conj(V[0][j]) * V[3][j];
    s += conj(V[1][j]) * (-V[2][j]);
    s += conj(V[2][j]) * (-V[1][j]);
    s += conj(V[3][j]) * V[0][j];
    double Pz = 0.25 * s.x;
    if (proper && fabs(Q[j].y) > tol * cabs(Q[j])) cls[j] = Q[j].y > 0 ? 0 : 1;
    else if (fabs(Pz) > tol) cls[j] = Pz > 0 ? 0 : 1;
    else if (fabs(Q[j].y) > tol) cls[j] = Q[j].y > tol ? 0 : 1;
    else cls[j] = 2;
  }
  // slots in eigen order; the degenerate ones then fill forward first (the reference's order)
  int nf = 0, nb = 0, slot[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (cls[j] == 0) slot[j] = nf++;
    else if (cls[j] == 1) slot[j] = 2 + nb++;
  }
  if (nf > 2 || nb > 2) return ST_SORT;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    if (cls[j] == 2) {
      if (nf < 2) slot[j] = nf++;
      else slot[j] = 2 + nb++;
    }
  }
  double2* rec = p.modes + (long)layer * 20 * n;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int sl = slot[j];
    const int dirb = sl >> 1, m = sl & 1;  // dirb 0: forward, 1: backward
#pragma unroll
    for (int i = 0; i < 4; ++i) st(rec, 8 * dirb + i + 4 * m, n, node, V[i][j]);
    st(rec, 16 + 2 * dirb + m, n, node, Q[j]);
  }
  return 0;
}

constexpr uint8_t ST_NEED_QR = 128;  // internal: this (node, layer) awaits the general QR pass

// K1: closed-form TE/TM modes (isotropic/uniaxial) and the block path; everything else is
// flagged for k_layer_modes_qr. Layer-major indexing: one layer, one material kind per warp.
__device__ __forceinline__ void layer_modes_body(const TransferParams& p, int layer, long node) {
  const long n = p.n;
  cd kx, ky;
  node_k(p, p.off + node, kx, ky);
  const LayerDev& L = p.layers[layer];
  cd Q[4], V[4][4];
  bool done;
  if ((L.ekind == 0 || L.ekind == 1) && L.mkind == 0) {
    closed_modes(L, p.omega, kx, ky, Q, V);
    done = true;
  } else {
    done = no_z_coupling(L) && block_modes(L, p.omega, kx, ky, Q, V);
  }
  p.lstat[(long)layer * n + node] = done ? classify_store(p, layer, node, Q, V) : ST_NEED_QR;
}
__global__ void __launch_bounds__(128) k_layer_modes(TransferParams p) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.n * p.nL) return;
  const int layer = (int)(t / p.n);
  layer_modes_body(p, layer, t - (long)layer * p.n);
}

// K1b: the general 4x4 QR path for the (node, layer) pairs K1 left
__device__ __forceinline__ void layer_modes_qr_body(const TransferParams& p, int layer, long node) {
  const long n = p.n;
  if (p.lstat[(long)layer * n + node] != ST_NEED_QR) return;
  cd kx, ky;
  node_k(p, p.off + node, kx, ky);
  const LayerDev& L = p.layers[layer];
  cd Q[4], V[4][4], B[4][4];
  berreman(L, p.omega, kx, ky, B);
  uint8_t stat = 0;
  if (!eig4(B, Q, V)) stat = ST_EIGEN;
  else stat = classify_store(p, layer, node, Q, V);
  p.lstat[(long)layer * n + node] = stat;
}
__global__ void __launch_bounds__(128) k_layer_modes_qr(TransferParams p) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.n * p.nL) return;
  if (p.lstat[t] != ST_NEED_QR) return;  // units are layer-major: t = layer n + node
  const int layer = (int)(t / p.n);
  layer_modes_qr_body(p, layer, t - (long)layer * p.n);
}

// ------------------------------------------------------------------------------------
// K2 helpers
// ------------------------------------------------------------------------------------
struct Mode4 {  // one layer's modes: Vf, Vb (4x2, V[i][m]), Qf, Qb
  cd vf[4][2], vb[4][2], qf[2], qb[2];
};

__device__ __forceinline__ void load_modes(const TransferParams& p, int layer, long node, Mode4& M) {
  const double2* rec = p.modes + (long)layer * 20 * p.n;
  for (int m = 0; m < 2; ++m) {
    for (int i = 0; i < 4; ++i) {
      M.vf[i][m] = ld(rec, i + 4 * m, p.n, node);
      M.vb[i][m] = ld(rec, 8 + i + 4 * m, p.n, node);
    }
    M.qf[m] = ld(rec, 16 + m, p.n, node);
    M.qb[m] = ld(rec, 18 + m, p.n, node);
  }
}
__device__ __forceinline__ void store_modes(const TransferParams& p, int layer, long node, const Mode4& M) {
  double2* rec = p.modes + (long)layer * 20 * p.n;
  for (int m = 0; m < 2; ++m) {
    for (int i = 0; i < 4; ++i) {
      st(rec, i + 4 * m, p.n, node, M.vf[i][m]);
      st(rec, 8 + i + 4 * m, p.n, node, M.vb[i][m]);
    }
    st(rec, 16 + m, p.n, node, M.qf[m]);
    st(rec, 18 + m, p.n, node, M.qb[m]);
  }
}
// W = R4s V row map: W0 = V3, W1 = -V2, W2 = -V1, W3 = V0
__device__ __forceinline__ cd Wof(const cd v[4][2], int i, int m) {
  switch (i) {
    case 0: return v[3][m];
    case 1: return -v[2][m];
    case 2: return -v[1][m];
    default: return v[0][m];
  }
}
// _match_modes (mod_ModeSolver.jl:333-349) for one direction: swap b's columns if needed
__device__ __forceinline__ void match_dir(const cd wa_src[4][2], cd vb[4][2], cd qb[2]) {
  cd C[2][2];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      cd s = conj(Wof(wa_src, 0, a)) * vb[0][b];
      for (int i = 1; i < 4; ++i) s += conj(Wof(wa_src, i, a)) * vb[i][b];
      C[a][b] = s;
    }
  double sid = norm2(C[0][0]) + norm2(C[1][1]);
  double ssw = norm2(C[0][1]) + norm2(C[1][0]);
  if (ssw > sid) {
    for (int i = 0; i < 4; ++i) { cd t = vb[i][0]; vb[i][0] = vb[i][1]; vb[i][1] = t; }
    cd t = qb[0]; qb[0] = qb[1]; qb[1] = t;
  }
}

// 4x4 LU solve with partial pivoting, NR right-hand sides; false on an exact zero pivot.
// Every array index is a compile-time constant (the pivot row swap is a predicated exchange
// with each candidate row), so the matrices stay in registers.
template <int NR>
__device__ __forceinline__ bool lu_solve4(cd A[4][4], cd B[4][NR]) {
  bool ok = true;
  cd rp[4];  // reciprocal pivots, reused by the back substitution
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    int pv = k;
    double best = norm2(A[k][k]);
#pragma unroll
    for (int i = k + 1; i < 4; ++i) {
      double v = norm2(A[i][k]);
      if (v > best) { best = v; pv = i; }
    }
    if (best == 0.0) ok = false;
#pragma unroll
    for (int i = k + 1; i < 4; ++i) {
      const bool sw = pv == i;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const cd t = A[i][j];
        A[i][j] = sw ? A[k][j] : t;
        A[k][j] = sw ? t : A[k][j];
      }
#pragma unroll
      for (int j = 0; j < NR; ++j) {
        const cd t = B[i][j];
        B[i][j] = sw ? B[k][j] : t;
        B[k][j] = sw ? t : B[k][j];
      }
    }
    const cd piv = recip(A[k][k]);
    rp[k] = piv;
#pragma unroll
    for (int i = k + 1; i < 4; ++i) {
      const cd l = A[i][k] * piv;
#pragma unroll
      for (int j = k + 1; j < 4; ++j) A[i][j] -= l * A[k][j];
#pragma unroll
      for (int j = 0; j < NR; ++j) B[i][j] -= l * B[k][j];
    }
  }
  if (!ok) return false;
#pragma unroll
  for (int j = 0; j < NR; ++j)
#pragma unroll
    for (int i = 3; i >= 0; --i) {
      cd s = B[i][j];
#pragma unroll
      for (int k = i + 1; k < 4; ++k) s -= A[i][k] * B[k][j];
      B[i][j] = s * rp[i];
    }
  return true;
}

__device__ __forceinline__ void interface_lhs_rhs(const Mode4& A, const Mode4& B, cd L[4][4], cd R[4][4]) {
  for (int i = 0; i < 4; ++i) {
    L[i][0] = -B.vf[i][0]; L[i][1] = -B.vf[i][1]; L[i][2] = A.vb[i][0]; L[i][3] = A.vb[i][1];
    R[i][0] = -A.vf[i][0]; R[i][1] = -A.vf[i][1]; R[i][2] = B.vb[i][0]; R[i][3] = B.vb[i][1];
  }
}

// The singular-interface branch of _S_Interface_Matrix (mod_ScatteringMatrix.jl:35-44,
// qr(LHS, ColumnNorm()) \ RHS), taken when the LU meets an exactly zero pivot (e.g. two
// identical layers at tangential incidence, where both forward modes coincide). Householder
// QR with column pivoting: step k moves the remaining column of largest 2-norm to the front
// and reflects it onto e_k (reflector v = x + e^{i arg x_k} |x| e_k, applied to the
// right-hand sides as well); the numerical rank counts the diagonal entries of R above
// 4 eps |R_11|; the basic least-squares solution sets the unknowns past the rank to zero and
// undoes the column permutation. Exact degeneracies are rare, so this stays out of line and
// costs the LU path no registers.
__device__ __noinline__ void interface_qr(const Mode4& A, const Mode4& B, S4& S) {
  cd a[4][4], r[4][4], x[4][4];
  int perm[4] = {0, 1, 2, 3};
  interface_lhs_rhs(A, B, a, r);
  for (int k = 0; k < 4; ++k) {
    int pc = k;
    double best = -1.0;
    for (int j = k; j < 4; ++j) {
      double c = 0.0;
      for (int i = k; i < 4; ++i) c += norm2(a[i][j]);
      if (c > best) { best = c; pc = j; }
    }
    if (pc != k) {
      for (int i = 0; i < 4; ++i) { const cd t = a[i][pc]; a[i][pc] = a[i][k]; a[i][k] = t; }
      const int t = perm[pc]; perm[pc] = perm[k]; perm[k] = t;
    }
    double nx = 0.0;
    for (int i = k; i < 4; ++i) nx += norm2(a[i][k]);
    nx = sqrt(nx);
    if (nx == 0.0) continue;
    const cd xk = a[k][k];
    const double axk = cabs(xk);
    const cd ph = axk > 0.0 ? xk / axk : cd{1.0, 0.0};
    cd v[4] = {};
    v[k] = xk + ph * nx;
    for (int i = k + 1; i < 4; ++i) v[i] = a[i][k];
    double vv = 0.0;
    for (int i = k; i < 4; ++i) vv += norm2(v[i]);
    if (vv == 0.0) continue;
    for (int j = k; j < 4; ++j) {
      cd t{0.0, 0.0};
      for (int i = k; i < 4; ++i) t += conj(v[i]) * a[i][j];
      t = t * (2.0 / vv);
      for (int i = k; i < 4; ++i) a[i][j] -= t * v[i];
    }
    for (int j = 0; j < 4; ++j) {
      cd t{0.0, 0.0};
      for (int i = k; i < 4; ++i) t += conj(v[i]) * r[i][j];
      t = t * (2.0 / vv);
      for (int i = k; i < 4; ++i) r[i][j] -= t * v[i];
    }
  }
  const double tol = 2.220446049250313e-16 * 4.0 * cabs(a[0][0]);
  int rank = 0;
  for (int k = 0; k < 4; ++k)
    if (cabs(a[k][k]) > tol) rank = k + 1;
  for (int j = 0; j < 4; ++j) {
    cd y[4] = {};
    for (int i = rank - 1; i >= 0; --i) {
      cd t = r[i][j];
      for (int k = i + 1; k < rank; ++k) t -= a[i][k] * y[k];
      y[i] = t / a[i][i];
    }
    for (int i = 0; i < 4; ++i) x[perm[i]][j] = y[i];
  }
  S.b11 = M2{x[0][0], x[0][1], x[1][0], x[1][1]};
  S.b12 = M2{x[0][2], x[0][3], x[1][2], x[1][3]};
  S.b21 = M2{x[2][0], x[2][1], x[3][0], x[3][1]};
  S.b22 = M2{x[2][2], x[2][3], x[3][2], x[3][3]};
}

// _S_Interface_Matrix (mod_ScatteringMatrix.jl:27-47): [-Vf_B Vb_A] \ [-Vf_A Vb_B] by LU with
// partial pivoting, and by the pivoted-QR least-squares solve when a pivot is exactly zero;
// always succeeds (a non-finite result is caught downstream as in the reference)
__device__ __forceinline__ bool interface_matrix(const Mode4& A, const Mode4& B, S4& S) {
  cd L[4][4], R[4][4];
  interface_lhs_rhs(A, B, L, R);
  if (!lu_solve4<4>(L, R)) {
    interface_qr(A, B, S);
    return true;
  }
  S.b11 = M2{R[0][0], R[0][1], R[1][0], R[1][1]};
  S.b12 = M2{R[0][2], R[0][3], R[1][2], R[1][3]};
  S.b21 = M2{R[2][0], R[2][1], R[3][0], R[3][1]};
  S.b22 = M2{R[2][2], R[2][3], R[3][2], R[3][3]};
  return true;
}

__device__ __forceinline__ void st_s4(double2* base, long slot, long n, long node, const S4& S) {
  double2* b = base + slot * 16 * n;
  const cd* v = reinterpret_cast<const cd*>(&S);
  for (int e = 0; e < 16; ++e) st(b, e, n, node, v[e]);
}
__device__ __forceinline__ S4 ld_s4(const double2* base, long slot, long n, long node) {
  S4 S;
  cd* v = reinterpret_cast<cd*>(&S);
  const double2* b = base + slot * 16 * n;
  for (int e = 0; e < 16; ++e) v[e] = ld(b, e, n, node);
  return S;
}

// Source_projection_Berreman_xyz (mod_SourceProj.jl:34-60); returns (sif, sib) 2x3 each
__device__ bool source_projection(cd kx, cd ky, double w, const LayerDev& L, const Mode4& M, cd sif[2][3], cd sib[2][3]) {
  cd etz1 = E(L, 1, 3), etz2 = E(L, 2, 3), ezz = E(L, 3, 3);
  cd jw{0.0, -w};
  cd J[4][3];
  const cd rezw = recip(ezz * w), rezz = recip(ezz);
  cd jz = jw;  // (-iω)·ẑ column only
  for (int q = 0; q < 3; ++q) {
    cd z = q == 2 ? jz : cd{0.0, 0.0} * jw;
    J[0][q] = kx * z * rezw;
    J[1][q] = ky * z * rezw;
    cd jtx = q == 0 ? jw : cd{0.0, 0.0}, jty = q == 1 ? jw : cd{0.0, 0.0};
    J[2][q] = jty - etz2 * z * rezz;
    J[3][q] = -jtx - (-etz1) * z * rezz;
  }
  cd V[4][4], W[4][4];
  for (int i = 0; i < 4; ++i) {
    V[i][0] = M.vf[i][0]; V[i][1] = M.vf[i][1]; V[i][2] = M.vb[i][0]; V[i][3] = M.vb[i][1];
  }
  for (int j = 0; j < 4; ++j) {
    W[0][j] = V[3][j]; W[1][j] = -V[2][j]; W[2][j] = -V[1][j]; W[3][j] = V[0][j];
  }
  cd WV[4][4], WJ[4][3];
  for (int a = 0; a < 4; ++a) {
    for (int b = 0; b < 4; ++b) {
      cd s = conj(W[0][a]) * V[0][b];
      for (int i = 1; i < 4; ++i) s += conj(W[i][a]) * V[i][b];
      WV[a][b] = s;
    }
    for (int q = 0; q < 3; ++q) {
      cd s = conj(W[0][a]) * J[0][q];
      for (int i = 1; i < 4; ++i) s += conj(W[i][a]) * J[i][q];
      WJ[a][q] = s;
    }
  }
  if (!lu_solve4<3>(WV, WJ)) return false;
  for (int q = 0; q < 3; ++q) {
    sif[0][q] = WJ[0][q]; sif[1][q] = WJ[1][q];
    sib[0][q] = WJ[2][q]; sib[1][q] = WJ[3][q];
  }
  return true;
}

// mode field basis of one obs layer (mod_CavityTransfer.jl:87-130)
__device__ void write_basis(const TransferParams& p, int oi, long node, long nout, const LayerDev& L, const Mode4& M,
                            cd kx, cd ky) {
  cd ezt1 = E(L, 3, 1), ezt2 = E(L, 3, 2), ezz = E(L, 3, 3);
  double iw = 1.0 / p.omega;
  const cd rezz = recip(ezz);
  double2* b = p.basis + (long)oi * 16 * nout;
  for (int m = 0; m < 2; ++m) {
    cd exf = M.vf[0][m], eyf = M.vf[1][m];
    cd ezf = -(ezt1 * M.vf[0][m] + ezt2 * M.vf[1][m] + iw * (kx * M.vf[3][m] - ky * M.vf[2][m])) * rezz;
    cd exb = M.vb[0][m], eyb = M.vb[1][m];
    cd ezb = -(ezt1 * M.vb[0][m] + ezt2 * M.vb[1][m] + iw * (kx * M.vb[3][m] - ky * M.vb[2][m])) * rezz;
    cd kzf = M.qf[m], kzb = M.qb[m];
    bool ok = isfin(exf) && isfin(eyf) && isfin(ezf) && isfin(exb) && isfin(eyb) && isfin(ezb) && isfin(kzf) && isfin(kzb);
    cd z{0, 0};
    st(b, 0 + m, nout, node, ok ? exf : z);
    st(b, 2 + m, nout, node, ok ? eyf : z);
    st(b, 4 + m, nout, node, ok ? ezf : z);
    st(b, 6 + m, nout, node, ok ? exb : z);
    st(b, 8 + m, nout, node, ok ? eyb : z);
    st(b, 10 + m, nout, node, ok ? ezb : z);
    st(b, 12 + m, nout, node, ok ? kzf : z);
    st(b, 14 + m, nout, node, ok ? kzb : z);
  }
}

__device__ __forceinline__ void write_seeds(const TransferParams& p, long node, long nout, const Mode4& M, cd sif[2][3], cd sib[2][3]) {
  for (int m = 0; m < 2; ++m) {
    st(p.Qf, m, nout, node, M.qf[m]);
    st(p.Qb, m, nout, node, M.qb[m]);
    for (int q = 0; q < 3; ++q) {
      st(p.sf, m + 2 * q, nout, node, sif[m][q]);
      st(p.sb, m + 2 * q, nout, node, -sib[m][q]);
    }
  }
}

// 2x4 matrix (two column pairs)
struct M24 {
  M2 L, R;
};
__device__ __forceinline__ M24 mul24(const M2& A, const M24& B) { return M24{mul(A, B.L), mul(A, B.R)}; }
__device__ __forceinline__ M24 add24(const M24& A, const M24& B) { return M24{add(A.L, B.L), add(A.R, B.R)}; }
__device__ __forceinline__ M24 dl24(cd p0, cd p1, const M24& A) { return M24{dl(p0, p1, A.L), dl(p0, p1, A.R)}; }
__device__ __forceinline__ M2 flush2(const M2& A) { return M2{flush(A.a00), flush(A.a01), flush(A.a10), flush(A.a11)}; }
__device__ __forceinline__ M24 flush24(const M24& A) { return M24{flush2(A.L), flush2(A.R)}; }
__device__ __forceinline__ bool fin2(const M2& A) { return isfin(A.a00) && isfin(A.a01) && isfin(A.a10) && isfin(A.a11); }

__device__ __forceinline__ void write_T(const TransferParams& p, int oi, long idx, long nT, const M24& Ef, const M24& Eb) {
  // T^o = [Ef; Eb] (4x4), stored column-major: element r + 4 c
  double2* b = p.Tout + (long)oi * 16 * nT;
  const M24* rows[2] = {&Ef, &Eb};
  for (int h = 0; h < 2; ++h) {
    const M24& X = *rows[h];
    st(b, 2 * h + 0 + 4 * 0, nT, idx, X.L.a00); st(b, 2 * h + 0 + 4 * 1, nT, idx, X.L.a01);
    st(b, 2 * h + 1 + 4 * 0, nT, idx, X.L.a10); st(b, 2 * h + 1 + 4 * 1, nT, idx, X.L.a11);
    st(b, 2 * h + 0 + 4 * 2, nT, idx, X.R.a00); st(b, 2 * h + 0 + 4 * 3, nT, idx, X.R.a01);
    st(b, 2 * h + 1 + 4 * 2, nT, idx, X.R.a10); st(b, 2 * h + 1 + 4 * 3, nT, idx, X.R.a11);
  }
}

// ------------------------------------------------------------------------------------
// K2: per-node chain
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void chain_body(const TransferParams& p, long node) {
  const long n = p.n;
  const int N = p.nL, src = p.src;
  const bool base = p.mode == 2;  // rotation base: seeds/basis are filled per φ later
  const long nT = base ? n : p.nout;
  const long gnode = base ? node : p.off + node;  // index into the outputs
  uint8_t stat = 0;
  for (int l = 0; l < N; ++l) stat |= p.lstat[(long)l * n + node];
  cd kx, ky;
  node_k(p, p.off + node, kx, ky);
  const cd z{0.0, 0.0};
  // outputs default to "invalid"
  if (!base) p.valid[gnode] = 0;
  for (int oi = 0; oi < p.nobs; ++oi) p.tvalid[(long)oi * nT + gnode] = 0;
  if (stat & (ST_EIGEN | ST_SORT)) {
    p.status[gnode] = stat;
    return;
  }
  // forward pass: matching, interfaces, SLeft prefix scan
  Mode4 prev;
  load_modes(p, 0, node, prev);
  S4 S0 = s4_diag(expi(prev.qf[0], p.layers[0].d), expi(prev.qf[1], p.layers[0].d), expi(-prev.qb[0], p.layers[0].d),
                  expi(-prev.qb[1], p.layers[0].d));
  S4 SLsrc = s4_identity();
  if ((p.needL >> 0) & 1u) st_s4(p.sleft, 0, n, node, s4_identity());
  bool seeds_ok = true;
  cd sif[2][3], sib[2][3];
  if (src == 1 && !base) {
    seeds_ok = source_projection(kx, ky, p.omega, p.layers[0], prev, sif, sib);
  }
  for (int oi = 0; oi < p.nobs; ++oi)
    if (p.obs[oi] == 1 && !base) write_basis(p, oi, gnode, p.nout, p.layers[0], prev, kx, ky);
  if (src == 1 && !base) write_seeds(p, gnode, p.nout, prev, sif, sib);
  for (int j = 2; j <= N; ++j) {
    Mode4 cur;
    load_modes(p, j - 1, node, cur);
    {
      cd wf[4][2], wb[4][2];
      for (int i = 0; i < 4; ++i)
        for (int m = 0; m < 2; ++m) { wf[i][m] = prev.vf[i][m]; wb[i][m] = prev.vb[i][m]; }
      match_dir(wf, cur.vf, cur.qf);
      match_dir(wb, cur.vb, cur.qb);
    }
    store_modes(p, j - 1, node, cur);
    S4 Si;
    if (!interface_matrix(prev, cur, Si)) stat |= ST_SINGULAR;
    st_s4(p.sint, j - 2, n, node, Si);
    S4 SL = redheffer(S0, Si);
    if ((p.needL >> (j - 1)) & 1u) st_s4(p.sleft, j - 1, n, node, SL);
    if (j == src) SLsrc = SL;
    const double d = p.layers[j - 1].d;
    cd pf0 = expi(cur.qf[0], d), pf1 = expi(cur.qf[1], d), pb0 = expi(-cur.qb[0], d), pb1 = expi(-cur.qb[1], d);
    // Redheffer(SL, diag(pf0, pf1, pb0, pb1))
    S0.b11 = dl(pf0, pf1, SL.b11);
    S0.b12 = dl(pf0, pf1, dr(SL.b12, pb0, pb1));
    S0.b21 = SL.b21;
    S0.b22 = dr(SL.b22, pb0, pb1);
    if (!base) {
      if (j == src) {
        seeds_ok = source_projection(kx, ky, p.omega, p.layers[j - 1], cur, sif, sib);
        write_seeds(p, gnode, p.nout, cur, sif, sib);
      }
      for (int oi = 0; oi < p.nobs; ++oi)
        if (p.obs[oi] == j) write_basis(p, oi, gnode, p.nout, p.layers[j - 1], cur, kx, ky);
    }
    prev = cur;
  }
  if (stat & ST_SINGULAR) {
    p.status[gnode] = stat;
    return;
  }
  // backward pass: SRight suffix scan down to the source layer
  S4 SR = s4_identity();
  if (N >= 1 && ((p.needR >> (N - 1)) & 1u)) st_s4(p.sright, N - 1, n, node, SR);
  for (int k = N - 1; k >= src; --k) {
    // Q of layer k (1-based) from the matched records
    const double2* rec = p.modes + (long)(k - 1) * 20 * n;
    cd qf0 = ld(rec, 16, n, node), qf1 = ld(rec, 17, n, node), qb0 = ld(rec, 18, n, node), qb1 = ld(rec, 19, n, node);
    const double d = p.layers[k - 1].d;
    S4 Si = ld_s4(p.sint, k - 1, n, node);
    S4 eff = redheffer_diag_left(expi(qf0, d), expi(qf1, d), expi(-qb0, d), expi(-qb1, d), Si);
    SR = redheffer(eff, SR);
    if ((p.needR >> (k - 1)) & 1u) st_s4(p.sright, k - 1, n, node, SR);
  }
  // cavity at the source layer (_R_cavity, _cavity_resummation)
  const double2* srec = p.modes + (long)(src - 1) * 20 * n;
  cd Qf0 = ld(srec, 16, n, node), Qf1 = ld(srec, 17, n, node), Qb0 = ld(srec, 18, n, node), Qb1 = ld(srec, 19, n, node);
  const double ds = p.layers[src - 1].d;
  M2 RL = SLsrc.b12;
  M2 RR = M2{z, z, z, z};
  S4 RRr = s4_identity();
  M24 Fp, Fm;
  const M2 I2 = M2{cd{1, 0}, z, z, cd{1, 0}}, Z2 = M2{z, z, z, z};
  if (src < N) {
    // SΦ = diag(e^{iQf(-d)}, e^{iQb d}) ⋆ SRight[src]
    RRr = redheffer_diag_left(expi(Qf0, -ds), expi(Qf1, -ds), expi(Qb0, ds), expi(Qb1, ds), SR);
    RR = RRr.b21;
    cd PF0 = expi(Qf0, ds), PF1 = expi(Qf1, ds), PB0 = expi(Qb0, -ds), PB1 = expi(Qb1, -ds);
    M2 Mx = mul(dr(dl(PF0, PF1, RL), PB0, PB1), RR);
    M2 D = imin(Mx);
    // RHS = S₊ + ΦF (RL S₋) = [I, ΦF RL]
    Fp.L = solve(D, I2);
    Fp.R = solve(D, dl(PF0, PF1, RL));
    // F⁻ = S₋ + ΦB (RR F⁺)
    Fm.L = dl(PB0, PB1, mul(RR, Fp.L));
    Fm.R = add(I2, dl(PB0, PB1, mul(RR, Fp.R)));
  } else {
    Fp = M24{Z2, Z2};
    Fm = M24{Z2, I2};
  }
  // T^o per observation layer
  bool any_tbad = false;
  for (int oi = 0; oi < p.nobs; ++oi) {
    const int o = p.obs[oi];
    M24 Ef, Eb;
    if (o == src) {
      Ef = mul24(RL, Fm);
      Eb = mul24(RR, Fp);
    } else if (o > src) {
      M24 cp = mul24(RRr.b11, Fp);
      if (o == N) {
        Ef = flush24(cp);
        Eb = M24{Z2, Z2};
      } else {
        S4 SRo = ld_s4(p.sright, o - 1, n, node);
        M24 bp = cond2x2_eq(SRo.b11) > 1e8 ? M24{Z2, Z2} : M24{solve(SRo.b11, cp.L), solve(SRo.b11, cp.R)};
        Ef = flush24(bp);
        M24 Ebn;
        if (o + 1 == N) {
          Ebn = M24{Z2, Z2};
        } else {
          S4 SRn = ld_s4(p.sright, o, n, node);
          M24 bn = cond2x2_eq(SRn.b11) > 1e8 ? M24{Z2, Z2} : M24{solve(SRn.b11, cp.L), solve(SRn.b11, cp.R)};
          Ebn = flush24(mul24(SRn.b21, bn));
        }
        const double2* orec = p.modes + (long)(o - 1) * 20 * n;
        const double dO = p.layers[o - 1].d;
        cd f0 = expi(ld(orec, 16, n, node), dO), f1 = expi(ld(orec, 17, n, node), dO);
        S4 Si = ld_s4(p.sint, o - 1, n, node);
        Eb = flush24(add24(mul24(Si.b21, dl24(f0, f1, Ef)), mul24(Si.b22, Ebn)));
      }
    } else {  // o < src
      M2 S22 = SLsrc.b22;
      M24 am = mul24(S22, Fm);
      auto bminus = [&](int k) -> M24 {  // b₋ of walk-left layer k (2 ≤ k ≤ src-1)
        S4 SLk = ld_s4(p.sleft, k - 1, n, node);
        return cond2x2_eq(SLk.b22) > 1e8 ? M24{Z2, Z2} : M24{solve(SLk.b22, am.L), solve(SLk.b22, am.R)};
      };
      if (o == 1) {
        Ef = M24{Z2, Z2};
      } else {
        S4 SLo = ld_s4(p.sleft, o - 1, n, node);
        M24 bm = cond2x2_eq(SLo.b22) > 1e8 ? M24{Z2, Z2} : M24{solve(SLo.b22, am.L), solve(SLo.b22, am.R)};
        Ef = flush24(mul24(SLo.b12, bm));
      }
      M24 Ebn = (o == src - 1) ? Fm : flush24(bminus(o + 1));
      const double2* orec = p.modes + (long)(o - 1) * 20 * n;
      const double dO = p.layers[o - 1].d;
      cd f0 = expi(ld(orec, 16, n, node), dO), f1 = expi(ld(orec, 17, n, node), dO);
      S4 Si = ld_s4(p.sint, o - 1, n, node);
      Eb = flush24(add24(mul24(Si.b21, dl24(f0, f1, Ef)), mul24(Si.b22, Ebn)));
    }
    bool fin = fin2(Ef.L) && fin2(Ef.R) && fin2(Eb.L) && fin2(Eb.R);
    if (!fin) any_tbad = true;
    if (fin) write_T(p, oi, gnode, nT, Ef, Eb);
    else write_T(p, oi, gnode, nT, M24{Z2, Z2}, M24{Z2, Z2});
    p.tvalid[(long)oi * nT + gnode] = fin ? 1 : 0;
  }
  if (any_tbad) stat |= ST_TNONFINITE;
  if (!base) {
    bool sfin = seeds_ok;
    for (int m = 0; m < 2 && sfin; ++m)
      for (int q = 0; q < 3; ++q) sfin = sfin && isfin(sif[m][q]) && isfin(sib[m][q]);
    if (!seeds_ok) stat |= ST_SINGULAR;
    if (!sfin) {
      stat |= ST_SEEDS;
      for (int oi = 0; oi < p.nobs; ++oi) p.tvalid[(long)oi * p.nout + gnode] = 0;
      p.valid[gnode] = 0;
    } else {
      p.valid[gnode] = 1;
      stat |= ST_VALID;
    }
  } else {
    stat |= ST_VALID;  // the base solve succeeded; seeds are checked per φ
  }
  p.status[gnode] = stat;
}

// ------------------------------------------------------------------------------------
// K2': the same solve when every observation layer is the source layer (needL = needR = 0):
// no walk to other layers, so SRight is needed at the source layer only. The Redheffer
// product is associative, so SRight[src] = eff_src ⋆ eff_src+1 ⋆ … ⋆ eff_N-1 accumulates in
// a forward sweep (left to right) instead of a backward scan: N-1 star products instead of
// N-1 + (N-src), and no SLeft, SRight or matched-mode records. One S4 register set serves as
// the SLeft prefix up to the source layer and as the SRight product after it. The solve runs
// as three kernels with short code, so that more warps stay resident than in one fused
// kernel (255 registers with spills):
//   k_iface  (per node, interface)  the interface matrix (4x4 LU) of the two layers' RAW mode
//                                   columns and the two matching decisions (match_decision);
//                                   past the source layer the propagation of the layer on its
//                                   left folded in: X_j = diag(e^{iQf d}, e^{-iQb d}) ⋆ Sint_j
//   k_seeds  (per node)             the swap mask up to the source layer from the decisions,
//                                   source projection and mode basis of the source layer
//   k_scan   (per node)             the swap mask of the stack, then acc = acc ⋆ X_j over the
//                                   interfaces (each X_j relabelled to the matched columns),
//                                   cavity, T^o
// Relabelling is exact; only the LU's pivot order differs from a solve on matched columns.
// The interface matrices live in the `sint` scratch, the decisions in `dec`; the LU failures
// and the projection's status travel in the layer status bytes, which k_scan reads and
// translates.
// ------------------------------------------------------------------------------------
// largest singular value of a 2x2 complex matrix: √ of the larger eigenvalue of A^H A
__device__ __forceinline__ double sigma_max2(const M2& A) {
  const double g00 = norm2(A.a00) + norm2(A.a10), g11 = norm2(A.a01) + norm2(A.a11);
  const cd g01 = conj(A.a00) * A.a01 + conj(A.a10) * A.a11;
  const double t = g00 + g11, dt = g00 * g11 - norm2(g01);
  return sqrt(fmax((t + sqrt(fmax(t * t - 4.0 * dt, 0.0))) / 2.0, 0.0));
}

struct ModeV {  // one layer's mode vectors: Vf, Vb (4x2)
  cd vf[4][2], vb[4][2];
};

__device__ __forceinline__ void load_v(const TransferParams& p, int layer, long node, uint64_t swaps, ModeV& M) {
  const double2* rec = p.modes + (long)layer * 20 * p.n;
  const int sf = (swaps >> (2 * layer)) & 1, sb = (swaps >> (2 * layer + 1)) & 1;
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      M.vf[i][m] = ld(rec, i + 4 * (m ^ sf), p.n, node);
      M.vb[i][m] = ld(rec, 8 + i + 4 * (m ^ sb), p.n, node);
    }
}
__device__ __forceinline__ void load_q(const TransferParams& p, int layer, long node, uint64_t swaps, cd qf[2], cd qb[2]) {
  const double2* rec = p.modes + (long)layer * 20 * p.n;
  const int sf = (swaps >> (2 * layer)) & 1, sb = (swaps >> (2 * layer + 1)) & 1;
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    qf[m] = ld(rec, 16 + (m ^ sf), p.n, node);
    qb[m] = ld(rec, 18 + (m ^ sb), p.n, node);
  }
}
__device__ __forceinline__ void load_matched(const TransferParams& p, int layer, long node, uint64_t swaps, Mode4& M) {
  ModeV v;
  load_v(p, layer, node, swaps, v);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int m = 0; m < 2; ++m) { M.vf[i][m] = v.vf[i][m]; M.vb[i][m] = v.vb[i][m]; }
  load_q(p, layer, node, swaps, M.qf, M.qb);
}
// _match_modes (mod_ModeSolver.jl:333-349) for one direction, on the RAW columns of both
// layers: the overlaps C[a][b] = <W(va)_a, vb_b>, X = |C01|² + |C10|², Y = |C00|² + |C11|².
// b's columns swap when X > Y if a's columns stand as computed, and when Y > X if a's columns
// were themselves swapped by the matching above them (swapping a's columns swaps C's rows, so
// X and Y trade places, sums of the same two terms; on a tie neither swaps). Returns
// (X > Y) | (Y > X) << 1.
__device__ __forceinline__ uint32_t match_decision(const cd va[4][2], const cd vb[4][2]) {
  cd C[2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      cd s = conj(Wof(va, 0, a)) * vb[0][b];
#pragma unroll
      for (int i = 1; i < 4; ++i) s += conj(Wof(va, i, a)) * vb[i][b];
      C[a][b] = s;
    }
  const double X = norm2(C[0][1]) + norm2(C[1][0]), Y = norm2(C[0][0]) + norm2(C[1][1]);
  return (X > Y ? 1u : 0u) | (Y > X ? 2u : 0u);
}

// the matching swap mask of layers 0 .. nlayers-1 (bit 2l: forward columns of layer l swapped,
// bit 2l+1: backward) from the per-interface decisions k_iface stored
__device__ __forceinline__ uint64_t swaps_upto(const TransferParams& p, long node, int nlayers) {
  uint64_t s = 0;
  for (int j = 2; j <= nlayers; ++j) {
    const int a = j - 2, b = j - 1;
    const uint32_t d = p.dec[(long)a * p.n + node];
    const uint32_t saf = (uint32_t)(s >> (2 * a)) & 1u, sab = (uint32_t)(s >> (2 * a + 1)) & 1u;
    const uint64_t sf = (d >> (saf ? 1 : 0)) & 1u, sb = (d >> (sab ? 3 : 2)) & 1u;
    s |= sf << (2 * b) | sb << (2 * b + 1);
  }
  return s;
}

// relabel an interface S-matrix formed on raw mode columns to the matched columns: rows of
// b11, b12 follow layer b's forward swap, rows of b21, b22 layer a's backward swap; columns of
// b11, b21 layer a's forward swap, of b12, b22 layer b's backward swap
__device__ __forceinline__ M2 m2_swap_rows(const M2& A, bool s) { return s ? M2{A.a10, A.a11, A.a00, A.a01} : A; }
__device__ __forceinline__ M2 m2_swap_cols(const M2& A, bool s) { return s ? M2{A.a01, A.a00, A.a11, A.a10} : A; }
__device__ __forceinline__ S4 relabel(const S4& X, bool saf, bool sab, bool sbf, bool sbb) {
  S4 o;
  o.b11 = m2_swap_cols(m2_swap_rows(X.b11, sbf), saf);
  o.b12 = m2_swap_cols(m2_swap_rows(X.b12, sbf), sbb);
  o.b21 = m2_swap_cols(m2_swap_rows(X.b21, sab), saf);
  o.b22 = m2_swap_cols(m2_swap_rows(X.b22, sab), sbb);
  return o;
}

constexpr uint8_t ST_PROJ_SINGULAR = 64;  // internal: the source projection's 4x4 solve failed

__device__ __forceinline__ uint8_t node_status(const TransferParams& p, long node) {
  uint8_t stat = 0;
  for (int l = 0; l < p.nL; ++l) stat |= p.lstat[(long)l * p.n + node];
  return stat;
}

__device__ __forceinline__ void seeds_body(const TransferParams& p, long node) {
  if (p.mode == 2 || p.resp) return;
  if (node_status(p, node) & (ST_EIGEN | ST_SORT)) return;
  const long gnode = p.off + node;
  const int layer = p.src - 1;
  cd kx, ky;
  node_k(p, p.off + node, kx, ky);
  Mode4 M;
  load_matched(p, layer, node, swaps_upto(p, node, p.src), M);
  cd sif[2][3], sib[2][3];
  const bool ok = source_projection(kx, ky, p.omega, p.layers[layer], M, sif, sib);
  bool fin = true;
  for (int m = 0; m < 2; ++m)
    for (int q = 0; q < 3; ++q) fin = fin && isfin(sif[m][q]) && isfin(sib[m][q]);
  write_seeds(p, gnode, p.nout, M, sif, sib);
  for (int oi = 0; oi < p.nobs; ++oi) write_basis(p, oi, gnode, p.nout, p.layers[layer], M, kx, ky);
  uint8_t f = 0;
  if (!ok) f |= ST_PROJ_SINGULAR;
  if (!(ok && fin)) f |= ST_SEEDS;
  if (f) p.lstat[(long)layer * p.n + node] |= f;
}

__device__ __forceinline__ void iface_body(const TransferParams& p, int j, long node) {
  const int a = j - 2, b = j - 1;
  S4 X;
  {
    ModeV va, vb;
    load_v(p, a, node, 0, va);
    load_v(p, b, node, 0, vb);
    p.dec[(long)a * p.n + node] = (uint8_t)(match_decision(va.vf, vb.vf) | match_decision(va.vb, vb.vb) << 2);
    Mode4 A, B;
    for (int i = 0; i < 4; ++i)
      for (int m = 0; m < 2; ++m) {
        A.vf[i][m] = va.vf[i][m]; A.vb[i][m] = va.vb[i][m];
        B.vf[i][m] = vb.vf[i][m]; B.vb[i][m] = vb.vb[i][m];
      }
    if (!interface_matrix(A, B, X)) p.lstat[(long)b * p.n + node] |= ST_SINGULAR;
  }
  if (j > p.src) {  // layer a's propagation, in its raw column order as X
    cd qf[2], qb[2];
    load_q(p, a, node, 0, qf, qb);
    const double d = p.layers[a].d;
    X = redheffer_diag_left(expi(qf[0], d), expi(qf[1], d), expi(-qb[0], d), expi(-qb[1], d), X);
  }
  st_s4(p.sint, j - 2, p.n, node, X);
}

__device__ __forceinline__ void scan_body(const TransferParams& p, long node) {
  const long n = p.n;
  const int N = p.nL, src = p.src;
  const bool base = p.mode == 2;
  const long nT = base ? n : p.nout;
  const long gnode = base ? node : p.off + node;
  uint8_t stat = node_status(p, node);
  const bool seeds_ok = !(stat & ST_PROJ_SINGULAR), seeds_fin = !(stat & ST_SEEDS);
  stat &= (uint8_t)~(ST_PROJ_SINGULAR | ST_SEEDS);
  const cd z{0.0, 0.0};
  if (!p.resp) {
    if (!base) p.valid[gnode] = 0;
    for (int oi = 0; oi < p.nobs; ++oi) p.tvalid[(long)oi * nT + gnode] = 0;
  }
  if (stat & (ST_EIGEN | ST_SORT)) {
    p.status[gnode] = stat;
    if (p.resp) p.resp[gnode] = 0.0;
    return;
  }
  const uint64_t swaps = swaps_upto(p, node, N);
  cd Qs[4];
  M2 RL = M2{z, z, z, z};
  S4 acc;
  {
    cd qf[2], qb[2];
    load_q(p, 0, node, 0, qf, qb);
    const double d0 = p.layers[0].d;
    if (src == 1) {
      Qs[0] = qf[0]; Qs[1] = qf[1]; Qs[2] = qb[0]; Qs[3] = qb[1];
      acc = s4_identity();
    } else {
      acc = s4_diag(expi(qf[0], d0), expi(qf[1], d0), expi(-qb[0], d0), expi(-qb[1], d0));
    }
  }
  for (int j = 2; j <= N; ++j) {
    const int la = j - 2, lb = j - 1;
    const S4 X = relabel(ld_s4(p.sint, j - 2, n, node), (swaps >> (2 * la)) & 1, (swaps >> (2 * la + 1)) & 1,
                         (swaps >> (2 * lb)) & 1, (swaps >> (2 * lb + 1)) & 1);
    const S4 R = redheffer(acc, X);
    if (j > src) {
      acc = R;
    } else {
      cd qf[2], qb[2];
      load_q(p, j - 1, node, swaps, qf, qb);
      if (j == src) {
        RL = R.b12;
        Qs[0] = qf[0]; Qs[1] = qf[1]; Qs[2] = qb[0]; Qs[3] = qb[1];
        acc = s4_identity();
      } else {
        const double d = p.layers[j - 1].d;
        const cd pf0 = expi(qf[0], d), pf1 = expi(qf[1], d), pb0 = expi(-qb[0], d), pb1 = expi(-qb[1], d);
        acc.b11 = dl(pf0, pf1, R.b11);
        acc.b12 = dl(pf0, pf1, dr(R.b12, pb0, pb1));
        acc.b21 = R.b21;
        acc.b22 = dr(R.b22, pb0, pb1);
      }
    }
  }
  if (stat & ST_SINGULAR) {
    p.status[gnode] = stat;
    if (p.resp) p.resp[gnode] = 0.0;
    return;
  }
  // cavity at the source layer (_R_cavity, _cavity_resummation), as k_chain
  const double ds = p.layers[src - 1].d;
  M2 RR = M2{z, z, z, z};
  M24 Fp, Fm;
  const M2 I2 = M2{cd{1, 0}, z, z, cd{1, 0}}, Z2 = M2{z, z, z, z};
  if (src < N) {
    const S4 RRr = redheffer_diag_left(expi(Qs[0], -ds), expi(Qs[1], -ds), expi(Qs[2], ds), expi(Qs[3], ds), acc);
    RR = RRr.b21;
    const cd PF0 = expi(Qs[0], ds), PF1 = expi(Qs[1], ds), PB0 = expi(Qs[2], -ds), PB1 = expi(Qs[3], -ds);
    const M2 Mx = mul(dr(dl(PF0, PF1, RL), PB0, PB1), RR);
    const M2 D = imin(Mx);
    Fp.L = solve(D, I2);
    Fp.R = solve(D, dl(PF0, PF1, RL));
    Fm.L = dl(PB0, PB1, mul(RR, Fp.L));
    Fm.R = add(I2, dl(PB0, PB1, mul(RR, Fp.R)));
  } else {
    Fp = M24{Z2, Z2};
    Fm = M24{Z2, I2};
  }
  if (p.resp) {
    // _cavity_response (mod_KSpaceFeatures.jl:109-127): max σ of RL, RR and, below the top
    // layer, of (I - ΦF RL ΦB RR)^-1 = F⁺'s left block
    double r = fmax(sigma_max2(RL), sigma_max2(RR));
    if (src > 1 && src < N) r = fmax(r, sigma_max2(Fp.L));
    p.resp[gnode] = isfinite(r) ? r : 0.0;
    p.status[gnode] = stat | ST_VALID;
    return;
  }
  // T^o of the source layer: Ef = RL F⁻, Eb = RR F⁺ (the same for every listed obs index)
  const M24 Ef = mul24(RL, Fm), Eb = mul24(RR, Fp);
  const bool fin = fin2(Ef.L) && fin2(Ef.R) && fin2(Eb.L) && fin2(Eb.R);
  for (int oi = 0; oi < p.nobs; ++oi) {
    if (fin) write_T(p, oi, gnode, nT, Ef, Eb);
    else write_T(p, oi, gnode, nT, M24{Z2, Z2}, M24{Z2, Z2});
    p.tvalid[(long)oi * nT + gnode] = fin ? 1 : 0;
  }
  if (!fin && p.nobs > 0) stat |= ST_TNONFINITE;
  if (!base) {
    if (!seeds_ok) stat |= ST_SINGULAR;
    if (!(seeds_ok && seeds_fin)) {
      stat |= ST_SEEDS;
      for (int oi = 0; oi < p.nobs; ++oi) p.tvalid[(long)oi * p.nout + gnode] = 0;
      p.valid[gnode] = 0;
    } else {
      p.valid[gnode] = 1;
      stat |= ST_VALID;
    }
  } else {
    stat |= ST_VALID;
  }
  p.status[gnode] = stat;
}

__global__ void __launch_bounds__(128) k_seeds(TransferParams p) {
  const long node = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (node < p.n) seeds_body(p, node);
}
// at most 170 registers: three 128-thread CTAs per SM (16 B of spills)
__global__ void __launch_bounds__(128, 3) k_iface(TransferParams p) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long n = p.n;
  if (t >= n * (p.nL - 1)) return;
  const int j = (int)(t / n) + 2;
  iface_body(p, j, t - (long)(j - 2) * n);
}
__global__ void __launch_bounds__(128) k_scan(TransferParams p) {
  const long node = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (node < p.n) scan_body(p, node);
}

__global__ void __launch_bounds__(128) k_chain(TransferParams p) {
  const long node = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (node < p.n) chain_body(p, node);
}

// ------------------------------------------------------------------------------------
// Batched forms: many independent problems (stacks, frequencies, grids) in one launch.
// probs[i] is problem i's parameter block; off[i] the first flat index of problem i
// (off[nb] = total): (node, layer) pairs for the mode kernels, nodes for the chains. A
// thread finds its problem by binary search over off.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ int find_problem(const long* __restrict__ off, int nb, long t) {
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
__global__ void __launch_bounds__(128) k_layer_modes_batch(const TransferParams* __restrict__ probs,
                                                           const long* __restrict__ off, int nb) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= off[nb]) return;
  const int i = find_problem(off, nb, t);
  const TransferParams& p = probs[i];
  const long lt = t - off[i];
  const int layer = (int)(lt / p.n);
  layer_modes_body(p, layer, lt - (long)layer * p.n);
}
__global__ void __launch_bounds__(128) k_layer_modes_qr_batch(const TransferParams* __restrict__ probs,
                                                              const long* __restrict__ off, int nb) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= off[nb]) return;
  const int i = find_problem(off, nb, t);
  const TransferParams& p = probs[i];
  const long lt = t - off[i];
  if (p.lstat[lt] != ST_NEED_QR) return;  // the status byte of unit lt, before any division
  const int layer = (int)(lt / p.n);
  layer_modes_qr_body(p, layer, lt - (long)layer * p.n);
}
__global__ void __launch_bounds__(128) k_chain_batch(const TransferParams* __restrict__ probs,
                                                     const long* __restrict__ off, int nb) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= off[nb]) return;
  const int i = find_problem(off, nb, t);
  chain_body(probs[i], t - off[i]);
}

// ------------------------------------------------------------------------------------
// Persistent forms of the batched transfer kernels (uneven batches replayed as one CUDA
// graph): a fixed grid of CTAs pulls tiles (problem, unit range) from a device counter until
// the queue is empty, so CTAs that drew short problems take more tiles instead of idling
// behind the longest one; a tile's units go to the CTA's threads in a block-stride loop.
// Units per stage: 0 modes and 1 QR = (layer, node) pairs, layer-major; 3 chain, 4 match,
// 5 seeds, 7 scan = nodes; 6 iface = (interface, node) pairs. The counter is zeroed before
// each launch (a memset node of the same graph). No CTA waits on another.
// ------------------------------------------------------------------------------------
template <int STAGE>
__device__ __forceinline__ void stage_unit(const TransferParams& p, long u) {
  if constexpr (STAGE == 0 || STAGE == 1) {
    if constexpr (STAGE == 1)
      if (p.lstat[u] != ST_NEED_QR) return;  // most units: one status byte, no division
    const int layer = (int)(u / p.n);
    if constexpr (STAGE == 0) layer_modes_body(p, layer, u - (long)layer * p.n);
    else layer_modes_qr_body(p, layer, u - (long)layer * p.n);
  } else if constexpr (STAGE == 3) {
    chain_body(p, u);
  } else if constexpr (STAGE == 5) {
    seeds_body(p, u);
  } else if constexpr (STAGE == 6) {
    const int j = (int)(u / p.n) + 2;
    iface_body(p, j, u - (long)(j - 2) * p.n);
  } else {
    scan_body(p, u);
  }
}

// the interface stage at three 128-thread CTAs per SM (as k_iface), the mode stage at four
// (128 registers, no spills)
template <int STAGE, int BLOCK>
__global__ void __launch_bounds__(BLOCK, (STAGE == 6 && BLOCK == 128) ? 3 : ((STAGE == 0 && BLOCK == 128) ? 4 : 1))
    k_persist(const TransferParams* __restrict__ probs, TileQueue q) {
  __shared__ int tile;
  for (;;) {
    if (threadIdx.x == 0) tile = (int)atomicAdd(q.counter, 1u);
    __syncthreads();
    const int t = tile;
    __syncthreads();
    if (t >= q.ntiles) return;
    const TransferParams& p = probs[q.prob[t]];
    const long e = q.end[t];
    for (long u = q.start[t] + threadIdx.x; u < e; u += BLOCK) stage_unit<STAGE>(p, u);
  }
}

template <int BLOCK>
cudaError_t launch_persist_b(int stage, int grid, const TransferParams* probs, const TileQueue& q, cudaStream_t s) {
  switch (stage) {
    case 0: k_persist<0, BLOCK><<<grid, BLOCK, 0, s>>>(probs, q); break;
    case 1: k_persist<1, BLOCK><<<grid, BLOCK, 0, s>>>(probs, q); break;
    case 3: k_persist<3, BLOCK><<<grid, BLOCK, 0, s>>>(probs, q); break;
    case 5: k_persist<5, BLOCK><<<grid, BLOCK, 0, s>>>(probs, q); break;
    case 6: k_persist<6, BLOCK><<<grid, BLOCK, 0, s>>>(probs, q); break;
    case 7: k_persist<7, BLOCK><<<grid, BLOCK, 0, s>>>(probs, q); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_persist(int stage, int block, int grid, const TransferParams* probs, const TileQueue& q,
                           cudaStream_t s) {
  if (q.ntiles <= 0) return cudaSuccess;
  if (grid <= 0) return cudaErrorInvalidValue;
  if (block == 128) return launch_persist_b<128>(stage, grid, probs, q, s);
  if (block == 256) return launch_persist_b<256>(stage, grid, probs, q, s);
  return cudaErrorInvalidValue;
}

// ------------------------------------------------------------------------------------
// K3: rotation fill of an azimuthally symmetric 2D grid (mod_CavityTransfer.jl:361-378)
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_rotate_fill(TransferParams p, const uint8_t* base_status, const uint8_t* base_tvalid,
                                                     const double2* Tbase) {
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long nout = p.nout, nb = p.n;  // p.n = Nk (base nodes)
  if (idx >= nout) return;
  long k = idx % p.Nk, q = idx / p.Nk;
  double s, c;
  sincos(p.phi[q], &s, &c);
  const cd kx{p.kr[k] * c, 0.0}, ky{p.kr[k] * s, 0.0};
  p.valid[idx] = 0;
  for (int oi = 0; oi < p.nobs; ++oi) p.tvalid[(long)oi * nout + idx] = 0;
  uint8_t bst = base_status[k];
  if (!(bst & ST_VALID)) { p.status[idx] = bst; return; }
  auto rot = [&](Mode4& M) {
    for (int m = 0; m < 2; ++m) {
      cd a0 = M.vf[0][m], a1 = M.vf[1][m], a2 = M.vf[2][m], a3 = M.vf[3][m];
      M.vf[0][m] = c * a0 - s * a1; M.vf[1][m] = s * a0 + c * a1;
      M.vf[2][m] = c * a2 - s * a3; M.vf[3][m] = s * a2 + c * a3;
      cd b0 = M.vb[0][m], b1 = M.vb[1][m], b2 = M.vb[2][m], b3 = M.vb[3][m];
      M.vb[0][m] = c * b0 - s * b1; M.vb[1][m] = s * b0 + c * b1;
      M.vb[2][m] = c * b2 - s * b3; M.vb[3][m] = s * b2 + c * b3;
    }
  };
  TransferParams pb = p;
  pb.n = nb;
  Mode4 Ms;
  load_modes(pb, p.src - 1, k, Ms);
  rot(Ms);
  cd sif[2][3], sib[2][3];
  bool ok = source_projection(kx, ky, p.omega, p.layers[p.src - 1], Ms, sif, sib);
  for (int m = 0; m < 2 && ok; ++m)
    for (int qq = 0; qq < 3; ++qq) ok = ok && isfin(sif[m][qq]) && isfin(sib[m][qq]);
  uint8_t stat = bst & ~ST_VALID;
  if (!ok) { p.status[idx] = stat | ST_SEEDS; return; }
  for (int oi = 0; oi < p.nobs; ++oi) {
    uint8_t tv = base_tvalid[(long)oi * nb + k];
    const double2* tb = Tbase + (long)oi * 16 * nb;
    double2* to = p.Tout + (long)oi * 16 * nout;
    for (int e = 0; e < 16; ++e) to[e * nout + idx] = tv ? tb[e * nb + k] : make_double2(0.0, 0.0);
    p.tvalid[(long)oi * nout + idx] = tv;
    Mode4 Mo;
    load_modes(pb, p.obs[oi] - 1, k, Mo);
    rot(Mo);
    write_basis(p, oi, idx, nout, p.layers[p.obs[oi] - 1], Mo, kx, ky);
  }
  write_seeds(p, idx, nout, Ms, sif, sib);
  p.valid[idx] = 1;
  p.status[idx] = stat | ST_VALID;
}

// ------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------
cudaError_t launch_layer_modes(const TransferParams& p, cudaStream_t stream) {
  long tot = (long)p.n * p.nL;
  if (tot <= 0) return cudaSuccess;
  k_layer_modes<<<(unsigned)((tot + 127) / 128), 128, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_layer_modes_qr(const TransferParams& p, cudaStream_t stream) {
  long tot = (long)p.n * p.nL;
  if (tot <= 0) return cudaSuccess;
  k_layer_modes_qr<<<(unsigned)((tot + 127) / 128), 128, 0, stream>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_chain(const TransferParams& p, cudaStream_t stream) {
  if (p.n <= 0) return cudaSuccess;
  k_chain<<<(unsigned)((p.n + 127) / 128), 128, 0, stream>>>(p);
  return cudaGetLastError();
}

__global__ void __launch_bounds__(128) k_seeds_batch(const TransferParams* __restrict__ probs, const long* __restrict__ off,
                                                     int nb) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= off[nb]) return;
  const int i = find_problem(off, nb, t);
  seeds_body(probs[i], t - off[i]);
}
// off: per-item (nL - 1) x n interface-node pairs
__global__ void __launch_bounds__(128, 3) k_iface_batch(const TransferParams* __restrict__ probs, const long* __restrict__ off,
                                                     int nb) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= off[nb]) return;
  const int i = find_problem(off, nb, t);
  const TransferParams& p = probs[i];
  const long lt = t - off[i];
  const int j = (int)(lt / p.n) + 2;
  iface_body(p, j, lt - (long)(j - 2) * p.n);
}
__global__ void __launch_bounds__(128) k_scan_batch(const TransferParams* __restrict__ probs, const long* __restrict__ off,
                                                    int nb) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= off[nb]) return;
  const int i = find_problem(off, nb, t);
  scan_body(probs[i], t - off[i]);
}

cudaError_t launch_chain_part(int part, const TransferParams& p, cudaStream_t stream) {
  if (p.n <= 0) return cudaSuccess;
  const unsigned g = (unsigned)((p.n + 127) / 128);
  switch (part) {
    case 0:
      if (p.nL > 1) k_iface<<<(unsigned)((p.n * (p.nL - 1) + 127) / 128), 128, 0, stream>>>(p);
      break;
    case 1: k_seeds<<<g, 128, 0, stream>>>(p); break;
    default: k_scan<<<g, 128, 0, stream>>>(p); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_transfer_batch(int kernel, const TransferParams* probs, const long* off, int nb, long total,
                                  cudaStream_t stream) {
  if (nb <= 0 || total <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)((total + 127) / 128);
  switch (kernel) {
    case 0: k_layer_modes_batch<<<grid, 128, 0, stream>>>(probs, off, nb); break;
    case 1: k_layer_modes_qr_batch<<<grid, 128, 0, stream>>>(probs, off, nb); break;
    case 5: k_seeds_batch<<<grid, 128, 0, stream>>>(probs, off, nb); break;
    case 6: k_iface_batch<<<grid, 128, 0, stream>>>(probs, off, nb); break;
    case 7: k_scan_batch<<<grid, 128, 0, stream>>>(probs, off, nb); break;
    default: k_chain_batch<<<grid, 128, 0, stream>>>(probs, off, nb); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_rotate_fill(const TransferParams& p, const uint8_t* base_status, const uint8_t* base_tvalid,
                               const double2* Tbase, cudaStream_t stream) {
  if (p.nout <= 0) return cudaSuccess;
  k_rotate_fill<<<(unsigned)((p.nout + 127) / 128), 128, 0, stream>>>(p, base_status, base_tvalid, Tbase);
  return cudaGetLastError();
}

}  // namespace ytf

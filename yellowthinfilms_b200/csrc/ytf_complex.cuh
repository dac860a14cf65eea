// ytf_complex.cuh -- FP64 complex arithmetic and small dense helpers for the per-k-node
// kernels (one thread owns one node's 4x4 / 2x2 systems, held in registers).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace ytf {

struct cd {
  double x, y;
};

__host__ __device__ __forceinline__ cd mk(double a, double b = 0.0) { return cd{a, b}; }
__host__ __device__ __forceinline__ cd operator+(cd a, cd b) { return cd{a.x + b.x, a.y + b.y}; }
__host__ __device__ __forceinline__ cd operator-(cd a, cd b) { return cd{a.x - b.x, a.y - b.y}; }
__host__ __device__ __forceinline__ cd operator-(cd a) { return cd{-a.x, -a.y}; }
__host__ __device__ __forceinline__ cd operator*(cd a, cd b) { return cd{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__host__ __device__ __forceinline__ cd operator*(double s, cd a) { return cd{s * a.x, s * a.y}; }
__host__ __device__ __forceinline__ cd operator*(cd a, double s) { return cd{s * a.x, s * a.y}; }
__host__ __device__ __forceinline__ cd& operator+=(cd& a, cd b) { a.x += b.x; a.y += b.y; return a; }
__host__ __device__ __forceinline__ cd& operator-=(cd& a, cd b) { a.x -= b.x; a.y -= b.y; return a; }
__host__ __device__ __forceinline__ cd conj(cd a) { return cd{a.x, -a.y}; }
__host__ __device__ __forceinline__ double norm2(cd a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ __forceinline__ double cabs(cd a) { return hypot(a.x, a.y); }
__host__ __device__ __forceinline__ double cabs1(cd a) { return fabs(a.x) + fabs(a.y); }
__host__ __device__ __forceinline__ bool isfin(cd a) { return isfinite(a.x) && isfinite(a.y); }
__host__ __device__ __forceinline__ bool iszero(cd a) { return a.x == 0.0 && a.y == 0.0; }
// i * a
__host__ __device__ __forceinline__ cd mul_i(cd a) { return cd{-a.y, a.x}; }

// a / b with scaling (Smith's algorithm)
__host__ __device__ __forceinline__ cd operator/(cd a, cd b) {
  if (fabs(b.x) >= fabs(b.y)) {
    if (b.x == 0.0 && b.y == 0.0) return cd{a.x / b.x, a.y / b.x};
    double r = b.y / b.x, den = b.x + b.y * r;
    return cd{(a.x + a.y * r) / den, (a.y - a.x * r) / den};
  }
  double r = b.x / b.y, den = b.x * r + b.y;
  return cd{(a.x * r + a.y) / den, (a.y * r - a.x) / den};
}
__host__ __device__ __forceinline__ cd operator/(cd a, double s) { return cd{a.x / s, a.y / s}; }
// 1 / b by Smith's scaling with two real divisions
__host__ __device__ __forceinline__ cd recip(cd b) {
  if (fabs(b.x) >= fabs(b.y)) {
    if (b.x == 0.0 && b.y == 0.0) return cd{1.0 / b.x, 0.0 / b.x};
    const double r = b.y / b.x, t = 1.0 / (b.x + b.y * r);
    return cd{t, -r * t};
  }
  const double r = b.x / b.y, t = 1.0 / (b.x * r + b.y);
  return cd{r * t, -t};
}

// principal square root, signed-zero aware (branch cut on the negative real axis)
__host__ __device__ __forceinline__ cd csqrt(cd z) {
  if (z.x == 0.0 && z.y == 0.0) return cd{0.0, z.y};
  double t = sqrt(0.5 * (fabs(z.x) + hypot(z.x, z.y)));
  if (z.x >= 0.0) return cd{t, z.y / (2.0 * t)};
  return cd{fabs(z.y) / (2.0 * t), copysign(t, z.y)};
}

__host__ __device__ __forceinline__ cd cexp(cd z) {
  double e = exp(z.x);
  double s, c;
  sincos(z.y, &s, &c);
  if (z.y == 0.0) return cd{e, z.y};
  return cd{e * c, e * s};
}
// exp(i q d)
__host__ __device__ __forceinline__ cd expi(cd q, double d) { return cexp(mul_i(q) * d); }

// 2x2 complex matrix, row-major a[r][c]
struct M2 {
  cd a00, a01, a10, a11;
};
__host__ __device__ __forceinline__ M2 m2(cd a00, cd a01, cd a10, cd a11) { return M2{a00, a01, a10, a11}; }
__host__ __device__ __forceinline__ M2 mul(const M2& A, const M2& B) {
  return M2{A.a00 * B.a00 + A.a01 * B.a10, A.a00 * B.a01 + A.a01 * B.a11, A.a10 * B.a00 + A.a11 * B.a10,
            A.a10 * B.a01 + A.a11 * B.a11};
}
__host__ __device__ __forceinline__ M2 add(const M2& A, const M2& B) {
  return M2{A.a00 + B.a00, A.a01 + B.a01, A.a10 + B.a10, A.a11 + B.a11};
}
__host__ __device__ __forceinline__ M2 imin(const M2& A) {  // I - A
  return M2{cd{1.0 - A.a00.x, -A.a00.y}, -A.a01, -A.a10, cd{1.0 - A.a11.x, -A.a11.y}};
}
__host__ __device__ __forceinline__ cd det(const M2& A) { return A.a00 * A.a11 - A.a01 * A.a10; }
// A \ B by Cramer's rule (one reciprocal of the determinant)
__host__ __device__ __forceinline__ M2 solve(const M2& A, const M2& B) {
  const cd r = recip(det(A));
  return M2{(A.a11 * B.a00 - A.a01 * B.a10) * r, (A.a11 * B.a01 - A.a01 * B.a11) * r,
            (A.a00 * B.a10 - A.a10 * B.a00) * r, (A.a00 * B.a11 - A.a10 * B.a01) * r};
}
__host__ __device__ __forceinline__ M2 inv(const M2& A) {
  const cd r = recip(det(A));
  return M2{A.a11 * r, -(A.a01 * r), -(A.a10 * r), A.a00 * r};
}
// diag(p) * A and A * diag(p)
__host__ __device__ __forceinline__ M2 dl(cd p0, cd p1, const M2& A) { return M2{p0 * A.a00, p0 * A.a01, p1 * A.a10, p1 * A.a11}; }
__host__ __device__ __forceinline__ M2 dr(const M2& A, cd p0, cd p1) { return M2{A.a00 * p0, A.a01 * p1, A.a10 * p0, A.a11 * p1}; }

// 4x4 complex matrix as 2x2 blocks (Redheffer form)
struct S4 {
  M2 b11, b12, b21, b22;
};
__host__ __device__ __forceinline__ S4 s4_identity() {
  cd o{1.0, 0.0}, z{0.0, 0.0};
  return S4{M2{o, z, z, o}, M2{z, z, z, z}, M2{z, z, z, z}, M2{o, z, z, o}};
}
__host__ __device__ __forceinline__ S4 s4_diag(cd p0, cd p1, cd p2, cd p3) {
  cd z{0.0, 0.0};
  return S4{M2{p0, z, z, p1}, M2{z, z, z, z}, M2{z, z, z, z}, M2{p2, z, z, p3}};
}

// Redheffer star product (mod_ScatteringMatrix.jl:65-85), regrouped around the two 2x2
// inverses: E = B11 (I - A12 B21)^-1, F = A22 (I - B21 A12)^-1, then
//   S11 = E A11, S12 = B12 + E A12 B22, S21 = A21 + F B21 A11, S22 = F B22
// (two complex reciprocals instead of sixteen complex divisions)
__host__ __device__ __forceinline__ S4 redheffer(const S4& A, const S4& B) {
  const M2 E = mul(B.b11, inv(imin(mul(A.b12, B.b21))));
  const M2 F = mul(A.b22, inv(imin(mul(B.b21, A.b12))));
  S4 o;
  o.b11 = mul(E, A.b11);
  o.b12 = add(B.b12, mul(mul(E, A.b12), B.b22));
  o.b21 = add(A.b21, mul(mul(F, B.b21), A.b11));
  o.b22 = mul(F, B.b22);
  return o;
}
// Redheffer with a diagonal left factor diag(p0,p1,p2,p3) (blocks 12 = 21 = 0)
__host__ __device__ __forceinline__ S4 redheffer_diag_left(cd p0, cd p1, cd p2, cd p3, const S4& B) {
  // A.b12 = 0 => D1 = D2 = I
  S4 o;
  o.b11 = dr(B.b11, p0, p1);
  o.b12 = B.b12;
  o.b21 = dr(dl(p2, p3, B.b21), p0, p1);
  o.b22 = dl(p2, p3, B.b22);
  return o;
}

// equilibrated 2x2 condition number (mod_FieldSolver.jl:33-53)
__host__ __device__ __forceinline__ double cond2x2(const M2& A) {
  cd g00 = conj(A.a00) * A.a00 + conj(A.a10) * A.a10;
  cd g01 = conj(A.a00) * A.a01 + conj(A.a10) * A.a11;
  cd g10 = conj(A.a01) * A.a00 + conj(A.a11) * A.a10;
  cd g11 = conj(A.a01) * A.a01 + conj(A.a11) * A.a11;
  double tr = (g00 + g11).x;
  double dt = (g00 * g11 - g01 * g10).x;
  double disc = sqrt(fmax(tr * tr - 4.0 * dt, 0.0));
  double l1 = (tr + disc) / 2, l2 = (tr - disc) / 2;
  if (l2 <= 0) return INFINITY;
  return sqrt(l1 / l2);
}
__host__ __device__ __forceinline__ double cond2x2_eq(const M2& A) {
  double n1 = sqrt(norm2(A.a00) + norm2(A.a10)), n2 = sqrt(norm2(A.a01) + norm2(A.a11));
  if (!(n1 > 0 && n2 > 0 && isfinite(n1) && isfinite(n2))) return INFINITY;
  return cond2x2(dr(A, cd{1.0 / n1, 0.0}, cd{1.0 / n2, 0.0}));
}

__host__ __device__ __forceinline__ cd flush(cd x) { return cabs(x) < 1e-250 ? cd{0.0, 0.0} : x; }

}  // namespace ytf

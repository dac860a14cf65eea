// ytf_bessel.cuh -- Bessel functions J_0, J_1, J_2 of a complex argument (device), for the
// synthesis on a deformed kρ contour (kρ ρ complex). Three regimes, each a published method:
//   |z| <= 8      : the power series J_n(z) = (z/2)^n Σ_m (-z²/4)^m / (m! (m+n)!)
//                   (A&S 9.1.10); the largest term is ~1e2, so ~1e-14 absolute accuracy;
//   8 < |z| < 25  : Miller's backward recurrence J_{k-1} = (2k/z) J_k - J_{k+1} from an order
//                   N = |z| + 32 with the normalisation J_0 + 2 Σ_{k≥1} J_{2k} = 1 (A&S 9.1.27,
//                   9.1.46), valid for complex z;
//   |z| >= 25     : the Hankel asymptotic expansion J_n(z) = √(2/(πz)) (P cos χ - Q sin χ),
//                   χ = z - nπ/2 - π/4 (A&S 9.2.5, 9.2.9-10), 24 terms (the terms fall below
//                   1e-16 of the first well before the expansion's smallest term at k ~ 2|z|).
// J_2 from the recurrence 2J_1/z - J_0 above |z| = 1, from its series below. Principal
// branches (Re z > 0 on the contour).
#pragma once
#include "ytf_complex.cuh"

namespace ytf {

__device__ __forceinline__ cd ccos(cd z) { return cd{cos(z.x) * cosh(z.y), -sin(z.x) * sinh(z.y)}; }
__device__ __forceinline__ cd csin(cd z) { return cd{sin(z.x) * cosh(z.y), cos(z.x) * sinh(z.y)}; }

// (z/2)^n Σ_m (-z²/4)^m / (m! (m+n)!), n = 0, 1, 2
__device__ inline cd bessel_series(int n, cd z) {
  const cd h = z * 0.5;
  const cd q = -(h * h);
  cd t{1.0, 0.0};
  double f = 1.0;
  for (int i = 1; i <= n; ++i) f *= i;
  t = t * (1.0 / f);
  cd s = t;
  for (int m = 1; m < 60; ++m) {
    t = t * q * (1.0 / ((double)m * (double)(m + n)));
    s += t;
    if (norm2(t) < 1e-36 * norm2(s)) break;
  }
  cd p{1.0, 0.0};
  for (int i = 0; i < n; ++i) p = p * h;
  return s * p;
}

__device__ inline void bessel_j01_c(cd z, cd& J0, cd& J1) {
  const double az = cabs(z);
  if (az <= 8.0) {
    J0 = bessel_series(0, z);
    J1 = bessel_series(1, z);
    return;
  }
  if (az < 25.0) {
    const int N = 2 * (((int)az + 32) / 2);  // even start order
    const cd iz = recip(z);
    cd jp1{0.0, 0.0}, jk{1e-200, 0.0};
    cd sum{0.0, 0.0}, j0v{0.0, 0.0}, j1v{0.0, 0.0};
    for (int k = N; k >= 1; --k) {
      const cd jm1 = iz * (2.0 * k) * jk - jp1;  // J_{k-1}
      jp1 = jk;
      jk = jm1;
      const int km1 = k - 1;
      if (km1 > 0 && (km1 % 2) == 0) sum += jk * 2.0;
      if (km1 == 1) j1v = jk;
      if (km1 == 0) j0v = jk;
      if (cabs(jk) > 1e200) {  // rescale on growth
        jk = jk * 1e-200; jp1 = jp1 * 1e-200; sum = sum * 1e-200; j1v = j1v * 1e-200;
      }
    }
    sum += j0v;
    const cd r = recip(sum);
    J0 = j0v * r;
    J1 = j1v * r;
    return;
  }
  // Hankel asymptotic expansion
  const cd iz = recip(z);
  const cd sq = csqrt(iz * (2.0 / 3.14159265358979323846));
  for (int n = 0; n <= 1; ++n) {
    const double mu = 4.0 * n * n;
    cd P{1.0, 0.0}, Q{0.0, 0.0};
    cd term{1.0, 0.0};
    for (int k = 1; k <= 24; ++k) {
      const double a = (mu - (2.0 * k - 1) * (2.0 * k - 1)) / (8.0 * k);
      term = term * iz * a;
      if (k % 2 == 1) Q += ((k / 2) % 2 == 0 ? term : -term);
      else P += ((k / 2) % 2 == 0 ? term : -term);
    }
    const cd chi = z - cd{n * 3.14159265358979323846 / 2 + 3.14159265358979323846 / 4, 0.0};
    const cd J = sq * (P * ccos(chi) - Q * csin(chi));
    if (n == 0) J0 = J;
    else J1 = J;
  }
}

__device__ inline void bessel_j012_c(cd z, cd& J0, cd& J1, cd& J2) {
  bessel_j01_c(z, J0, J1);
  if (cabs(z) < 1.0) J2 = bessel_series(2, z);
  else J2 = recip(z) * J1 * 2.0 - J0;
}

}  // namespace ytf

// ytf_synth.cu -- synthesis of G(ρ, z, z') from a device transfer cache.
//
// 1D (point source, azimuthally symmetric stack; closed_form_G for CavityTransferCache1D,
// mod_ClosedFormField.jl:435-487): the Jacobi–Anger pixel integral
// (_integrate_pixel_1d, :344-390) is linear in (J0, J1, J2)(kρ), so for every distinct
// radius and z-row it is the contraction
//     R[ρ, col] = Σ_k J_n(k ρ) · C_n[k, col],   n = 0, 1, 2,
// of a Bessel table with per-node coefficients (weighted amplitude × mode field × phase ×
// k). k_coef1d builds C_n (13 complex columns per z-row), k_bessel the tables, a GEMM
// does the contraction and k_assemble1d combines orders, rotates by the pixel azimuth
// and writes Julia's (Nx, Ny, Nz, 3, 3) column-major layout.
//
// 2D (any stack; closed_form_G for CavityTransferCache2D, lateral=:direct, :711-753):
// k_strengths2d forms the 9 strengths per (node, z-row) (_strengths_row!, :616-659) and
// k_lateral evaluates G[pix, col] = Σ_n e^{i(kx_n x + ky_n y)} S[col, n] as a complex GEMM
// whose A operand is generated in shared memory from the node's (kx, ky).
#include "ytf_complex.cuh"
#include "ytf_kernels.h"
#include "ytf_bessel.cuh"

#include <algorithm>

namespace ytf {

__device__ __forceinline__ cd ldc(const double2* b, long e, long n, long i) {
  double2 v = b[e * n + i];
  return cd{v.x, v.y};
}

// _phase (mod_ClosedFormField.jl:59-69): clamped exp(i kz z)
__device__ __forceinline__ cd phase_cl(cd kz, double z) {
  double a = -kz.y * z, b = kz.x * z;
  if (!isfinite(a) || !isfinite(b) || a > 700.0 || a < -700.0) return cd{0.0, 0.0};
  return cexp(cd{a, b});
}
__device__ __forceinline__ cd fin0(cd z) { return isfin(z) ? z : cd{0.0, 0.0}; }

// reflected amplitudes of node k (amplitude_at, :175-203) with the term masks
__device__ __forceinline__ void reflected_amp(const SynthParams& p, long k, cd Af[2][3], cd Ab[2][3]) {
  const CacheView& c = p.c;
  for (int m = 0; m < 2; ++m)
    for (int q = 0; q < 3; ++q) { Af[m][q] = cd{0, 0}; Ab[m][q] = cd{0, 0}; }
  if (!(c.valid[k] && c.tvalid[k])) return;
  const double d = c.d_src, zp = p.zpos;
  cd Pf[2], Pb[2];
  for (int m = 0; m < 2; ++m) {
    Pf[m] = cexp(mul_i(ldc(c.Qf, m, c.n, k)) * (d - zp));
    Pb[m] = cexp(mul_i(-ldc(c.Qb, m, c.n, k)) * zp);
  }
  cd T[4][4];
  for (int r = 0; r < 4; ++r)
    for (int cc = 0; cc < 4; ++cc) T[r][cc] = ldc(c.T, r + 4 * cc, c.n, k);
  for (int q = 0; q < 3; ++q) {
    cd sf0 = ldc(c.sf, 0 + 2 * q, c.n, k) * Pf[0], sf1 = ldc(c.sf, 1 + 2 * q, c.n, k) * Pf[1];
    cd sb0 = ldc(c.sb, 0 + 2 * q, c.n, k) * Pb[0], sb1 = ldc(c.sb, 1 + 2 * q, c.n, k) * Pb[1];
    // rows 0,1 (Af) use the F masks, rows 2,3 (Ab) the B masks
    cd uF[4] = {p.uf_F * sf0, p.uf_F * sf1, p.ub_F * sb0, p.ub_F * sb1};
    cd uB[4] = {p.uf_B * sf0, p.uf_B * sf1, p.ub_B * sb0, p.ub_B * sb1};
    for (int m = 0; m < 2; ++m) {
      cd a = T[m][0] * uF[0];
      a += T[m][1] * uF[1];
      a += T[m][2] * uF[2];
      a += T[m][3] * uF[3];
      Af[m][q] = a;
      cd b = T[2 + m][0] * uB[0];
      b += T[2 + m][1] * uB[1];
      b += T[2 + m][2] * uB[2];
      b += T[2 + m][3] * uB[3];
      Ab[m][q] = b;
    }
  }
}

// same-layer direct amplitudes at z_obs (direct_amplitude, :232-259), point source
__device__ __forceinline__ void direct_amp(const SynthParams& p, long k, double z, cd Afd[2][3], cd Abd[2][3]) {
  const CacheView& c = p.c;
  for (int m = 0; m < 2; ++m)
    for (int q = 0; q < 3; ++q) { Afd[m][q] = cd{0, 0}; Abd[m][q] = cd{0, 0}; }
  if (!c.valid[k]) return;
  const double zeta = z - p.zpos;
  if (zeta > 0) {
    for (int m = 0; m < 2; ++m) {
      cd e = phase_cl(ldc(c.Qf, m, c.n, k), zeta);
      for (int q = 0; q < 3; ++q) Afd[m][q] = ldc(c.sf, m + 2 * q, c.n, k) * e;
    }
  } else if (zeta < 0) {
    for (int m = 0; m < 2; ++m) {
      cd e = phase_cl(ldc(c.Qb, m, c.n, k), zeta);
      for (int q = 0; q < 3; ++q) Abd[m][q] = ldc(c.sb, m + 2 * q, c.n, k) * e;
    }
  }
}

// ------------------------------------------------------------------------------------
// 1D coefficients. Columns per z-row: order 0: xx yx xy yy zz; order 1: zx zy xz yz;
// order 2: xx yx xy yy (c q); stored: the 9 independent ones (store_coef_row, C1D_R* real rows
// per height). Output rows are real: row 2*(zi*ncol + col) + part, node fastest.
// ------------------------------------------------------------------------------------
// the 13 coefficient columns of one (node, z row) (_integrate_pixel_1d's integrand,
// mod_ClosedFormField.jl:435-487): order 0: xx yx xy yy zz; order 1: zx zy xz yz; order 2:
// xx yx xy yy
__device__ __forceinline__ void coef1d_row(const SynthParams& p, long k, double z, const cd Af[2][3], const cd Ab[2][3],
                                           cd c0[5], cd c1[4], cd c2[4]) {
  const CacheView& c = p.c;
  const long n = c.n;
  // i w / (2π) with a complex weight and node on a deformed contour (kri, wri), real otherwise
  const cd W = cd{0.0, 1.0 / (2.0 * 3.14159265358979323846)} * cd{c.wr[k], c.wri ? c.wri[k] : 0.0};
  const cd kx{c.kr[k], c.kri ? c.kri[k] : 0.0};
  for (int i = 0; i < 5; ++i) c0[i] = cd{0, 0};
  for (int i = 0; i < 4; ++i) { c1[i] = cd{0, 0}; c2[i] = cd{0, 0}; }
  cd Afd[2][3], Abd[2][3];
  if (p.with_direct) direct_amp(p, k, z, Afd, Abd);
  const cd half_i{0.0, 0.5};
  for (int m = 0; m < 2; ++m) {
    cd kzf = ldc(c.basis, 12 + m, n, k), kzb = ldc(c.basis, 14 + m, n, k);
    cd af[3], ab[3], gf, gb;
    if (p.with_direct) {
      cd pf = phase_cl(kzf, z), pb = phase_cl(kzb, z - p.d_obs);
      for (int q = 0; q < 3; ++q) {
        af[q] = fin0(W * (Afd[m][q] + Af[m][q] * pf));
        ab[q] = fin0(W * (Abd[m][q] + Ab[m][q] * pb));
      }
      gf = kx;
      gb = kx;
    } else {
      for (int q = 0; q < 3; ++q) { af[q] = fin0(W * Af[m][q]); ab[q] = fin0(W * Ab[m][q]); }
      gf = phase_cl(kzf, z) * kx;
      gb = phase_cl(kzb, z - p.d_obs) * kx;
    }
    for (int br = 0; br < 2; ++br) {
      const cd* a = br == 0 ? af : ab;
      cd g = br == 0 ? gf : gb;
      cd ex = ldc(c.basis, (br == 0 ? 0 : 6) + m, n, k);
      cd ey = ldc(c.basis, (br == 0 ? 2 : 8) + m, n, k);
      cd ez = ldc(c.basis, (br == 0 ? 4 : 10) + m, n, k);
      cd ax = a[0] * g, ay = a[1] * g, az = a[2] * g;
      // q = x: A = ax, B = ay
      c0[0] += half_i * (-(ax * ex) - ay * ey);  // xx
      c2[0] += half_i * (ax * ex - ay * ey);
      c0[1] += half_i * (-(ax * ey) + ay * ex);  // yx
      c2[1] += half_i * (ax * ey + ay * ex);
      c1[0] += ax * ez;                          // zx
      // q = y: A = ay, B = -ax
      c0[2] += half_i * (-(ay * ex) + ax * ey);  // xy
      c2[2] += half_i * (ay * ex + ax * ey);
      c0[3] += half_i * (-(ay * ey) - ax * ex);  // yy
      c2[3] += half_i * (ay * ey - ax * ex);
      c1[1] += ay * ez;                          // zy
      // q = z: C = az
      c1[2] += az * ex;                          // xz
      c1[3] += az * ey;                          // yz
      c0[4] += cd{0.0, -1.0} * (az * ez);        // zz
    }
  }
}

// the 9 stored complex columns of one (node, height) as real rows (C1D_R* per height) of
// C0, C1, C2 (row stride `stride`)
template <class T>
__device__ __forceinline__ void store_coef_row(T* C0, T* C1, T* C2, long stride, long k, int zi, const cd c0[5],
                                               const cd c1[4], const cd c2[4]) {
  const cd s0[3] = {c0[0], c0[1], c0[4]};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const long r = 2L * (zi * 3 + j);
    C0[r * stride + k] = (T)s0[j].x;
    C0[(r + 1) * stride + k] = (T)s0[j].y;
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const long r = 2L * (zi * 4 + j);
    C1[r * stride + k] = (T)c1[j].x;
    C1[(r + 1) * stride + k] = (T)c1[j].y;
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const long r = 2L * (zi * 2 + j);
    C2[r * stride + k] = (T)c2[j].x;
    C2[(r + 1) * stride + k] = (T)c2[j].y;
  }
}

// the 13 order sums of one (radius, height) from the stored ones (Pn(col) = the complex value
// of stored column col of order n): yy = xx, xy = -yx of order 0; xy = yx, yy = -xx of order 2
template <class F0, class F1, class F2>
__device__ __forceinline__ void unpack_order_sums(F0 P0, F1 P1, F2 P2, cd g0[5], cd g1[4], cd g2[4]) {
  g0[0] = P0(0);
  g0[1] = P0(1);
  g0[2] = -g0[1];
  g0[3] = g0[0];
  g0[4] = P0(2);
#pragma unroll
  for (int j = 0; j < 4; ++j) g1[j] = P1(j);
  g2[0] = P2(0);
  g2[1] = P2(1);
  g2[2] = g2[1];
  g2[3] = -g2[0];
}

__global__ void __launch_bounds__(128) k_coef1d(SynthParams p, double* C0, double* C1, double* C2) {
  long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int zi = blockIdx.y;
  const CacheView& c = p.c;
  if (k >= c.n) return;
  const long n = c.n;
  cd Af[2][3], Ab[2][3];
  reflected_amp(p, k, Af, Ab);
  cd c0[5], c1[4], c2[4];
  coef1d_row(p, k, p.zo[zi], Af, Ab, c0, c1, c2);
  store_coef_row(C0, C1, C2, n, k, zi, c0, c1, c2);
}

cudaError_t launch_coef1d(const SynthParams& p, double* C0, double* C1, double* C2, cudaStream_t s) {
  dim3 grid((unsigned)((p.c.n + 127) / 128), (unsigned)p.nz);
  k_coef1d<<<grid, 128, 0, s>>>(p, C0, C1, C2);
  return cudaGetLastError();
}

// J_0, J_1, J_2 of a real argument: CUDA's j0/j1, J2 by its power series below |x| = 1 and the
// three-term recurrence above
__device__ __forceinline__ void bessel_j012(double x, double& a0, double& a1, double& a2) {
  a0 = j0(x);
  a1 = j1(x);
  if (fabs(x) < 1.0) {
    // J2(x) = Σ_m (-1)^m (x/2)^{2m+2} / (m! (m+2)!)  (A&S 9.1.10); exact 0 at x = 0
    double h2 = 0.25 * x * x, t = 0.5 * h2, s = t;
    for (int m = 0; m < 12; ++m) {
      t *= -h2 / ((m + 1.0) * (m + 3.0));
      s += t;
    }
    a2 = s;
  } else {
    a2 = (2.0 / x) * a1 - a0;  // three-term recurrence (A&S 9.1.27)
  }
}

// Bessel tables J_n(k ρ), n = 0, 1, 2; row r = radius, k contiguous
__global__ void k_bessel(const double* kr, long nk, const double* rho, int nr, double* J0, double* J1, double* J2) {
  long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (k >= nk) return;
  double x = kr[k] * rho[r];
  long o = (long)r * nk + k;
  double a0, a1, a2;
  bessel_j012(x, a0, a1, a2);
  J0[o] = a0;
  J1[o] = a1;
  J2[o] = a2;
}

// J_n(kρ ρ) of complex nodes (deformed contour): real and imaginary tables of each order
__global__ void k_bessel_c(const double* kr, const double* kri, long nk, const double* rho, int nr, double* J) {
  long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (k >= nk) return;
  const cd z = cd{kr[k], kri[k]} * rho[r];
  cd a0, a1, a2;
  if (z.x == 0.0 && z.y == 0.0) {
    a0 = cd{1.0, 0.0}; a1 = cd{0.0, 0.0}; a2 = cd{0.0, 0.0};
  } else {
    bessel_j012_c(z, a0, a1, a2);
  }
  const long o = (long)r * nk + k, plane = (long)nr * nk;
  J[o] = a0.x; J[plane + o] = a0.y;
  J[2 * plane + o] = a1.x; J[3 * plane + o] = a1.y;
  J[4 * plane + o] = a2.x; J[5 * plane + o] = a2.y;
}

cudaError_t launch_bessel_c(const double* kr, const double* kri, long nk, const double* rho, int nr, double* J,
                            cudaStream_t s) {
  if (nk <= 0 || nr <= 0) return cudaSuccess;
  dim3 grid((unsigned)((nk + 127) / 128), (unsigned)nr);
  k_bessel_c<<<grid, 128, 0, s>>>(kr, kri, nk, rho, nr, J);
  return cudaGetLastError();
}

// complex J times the real/imag column pairs: P[r][2c] = A[2c] - B[2c+1], P[r][2c+1] = A[2c+1] + B[2c]
// with A = Re J · C^T and B = Im J · C^T
__global__ void k_combine_complex(long M, int N2, const double* A, const double* B, double* P) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M * (N2 / 2)) return;
  const long r = t / (N2 / 2), c = t % (N2 / 2);
  const long o = r * N2 + 2 * c;
  P[o] = A[o] - B[o + 1];
  P[o + 1] = A[o + 1] + B[o];
}

cudaError_t launch_combine_complex(long M, int N2, const double* A, const double* B, double* P, cudaStream_t s) {
  const long tot = M * (N2 / 2);
  if (tot <= 0) return cudaSuccess;
  k_combine_complex<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(M, N2, A, B, P);
  return cudaGetLastError();
}

// one complex J_n evaluation per thread (the device Bessel functions, exposed for testing)
__global__ void k_bessel_eval(long n, int order, const double* zr, const double* zi, double* outr, double* outi) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  cd a0, a1, a2;
  const cd z{zr[t], zi[t]};
  if (z.x == 0.0 && z.y == 0.0) {
    a0 = cd{1.0, 0.0}; a1 = cd{0.0, 0.0}; a2 = cd{0.0, 0.0};
  } else {
    bessel_j012_c(z, a0, a1, a2);
  }
  const cd v = order == 0 ? a0 : (order == 1 ? a1 : a2);
  outr[t] = v.x;
  outi[t] = v.y;
}

cudaError_t launch_bessel_eval(long n, int order, const double* zr, const double* zi, double* outr, double* outi,
                               cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_bessel_eval<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(n, order, zr, zi, outr, outi);
  return cudaGetLastError();
}

cudaError_t launch_bessel(const double* kr, long nk, const double* rho, int nr, double* J0, double* J1, double* J2,
                          cudaStream_t s) {
  dim3 grid((unsigned)((nk + 127) / 128), (unsigned)nr);
  k_bessel<<<grid, 128, 0, s>>>(kr, nk, rho, nr, J0, J1, J2);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// FP64 GEMM C[M][N] = A[M][K] · B[N][K]^T (both operands K-contiguous), split-K with a
// deterministic reduction. 128x128 tile, 8 k per stage, 8x8 outputs per thread.
// ------------------------------------------------------------------------------------
constexpr int GT = 128, GK = 8;
__global__ void __launch_bounds__(256) k_dgemm_nt(int M, int N, int K, const double* __restrict__ A,
                                                  const double* __restrict__ B, double* __restrict__ Cp, int kchunk) {
  __shared__ double As[GK][GT];
  __shared__ double Bs[GK][GT];
  const int bm = blockIdx.y * GT, bn = blockIdx.x * GT, sp = blockIdx.z;
  const long k0 = (long)sp * kchunk;
  const long k1 = min((long)K, k0 + kchunk);
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  for (long kk = k0; kk < k1; kk += GK) {
    // 128x8 tile of A and of B: 1024 elements each, 4 per thread; k fastest in memory
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      int idx = tid + 256 * e;
      int row = idx / GK, col = idx % GK;
      long kg = kk + col;
      int ra = bm + row, rb = bn + row;
      As[col][row] = (ra < M && kg < k1) ? A[(long)ra * K + kg] : 0.0;
      Bs[col][row] = (rb < N && kg < k1) ? B[(long)rb * K + kg] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < GK; ++t) {
      double a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = As[t][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = Bs[t][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  double* C = Cp + (long)sp * M * N;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    int r = bm + ty + 16 * i;
    if (r >= M) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      int cc = bn + tx + 16 * j;
      if (cc < N) C[(long)r * N + cc] = acc[i][j];
    }
  }
}

__global__ void k_reduce_splits(long len, int splits, const double* __restrict__ P, double* __restrict__ C) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len) return;
  double s = 0.0;
  for (int k = 0; k < splits; ++k) s += P[(long)k * len + i];
  C[i] = s;
}

int dgemm_splits(int K, int splits) {
  int kchunk = (K + splits - 1) / splits;
  kchunk = ((kchunk + GK - 1) / GK) * GK;
  if (kchunk <= 0) return 1;
  return std::max(1, (K + kchunk - 1) / kchunk);
}

cudaError_t launch_dgemm_nt(int M, int N, int K, const double* A, const double* B, double* partial, int splits,
                            cudaStream_t s) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  splits = dgemm_splits(K, splits);
  int kchunk = (K + splits - 1) / splits;
  kchunk = ((kchunk + GK - 1) / GK) * GK;
  dim3 grid((unsigned)((N + GT - 1) / GT), (unsigned)((M + GT - 1) / GT), (unsigned)splits);
  k_dgemm_nt<<<grid, 256, 0, s>>>(M, N, K, A, B, partial, kchunk);
  return cudaGetLastError();
}

__global__ void k_add(long len, const double* __restrict__ x, double* __restrict__ acc) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long)gridDim.x * blockDim.x) acc[i] += x[i];
}

cudaError_t launch_add(long len, const double* x, double* acc, cudaStream_t s) {
  if (len <= 0) return cudaSuccess;
  k_add<<<(unsigned)std::min<long>((len + 255) / 256, 148L * 8), 256, 0, s>>>(len, x, acc);
  return cudaGetLastError();
}

cudaError_t launch_reduce_splits(long len, int splits, const double* partial, double* C, cudaStream_t s) {
  if (len <= 0) return cudaSuccess;
  k_reduce_splits<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(len, splits, partial, C);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// 1D assembly: combine orders, rotate per pixel, Julia layout (Nx, Ny, Nz, 3, 3)
// obs-layer basis of one node: kz and the field components (E_f, E_b) of the two modes
__device__ __forceinline__ void load_obs_basis(const CacheView& c, long node, cd kzf[2], cd kzb[2], cd ef[2][3],
                                               cd eb[2][3]) {
  const long n = c.n;
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    kzf[m] = ldc(c.basis, 12 + m, n, node);
    kzb[m] = ldc(c.basis, 14 + m, n, node);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      ef[m][a] = ldc(c.basis, 2 * a + m, n, node);
      eb[m][a] = ldc(c.basis, 6 + 2 * a + m, n, node);
    }
  }
}

// the nine strengths of one (node, z row) (_strengths_row!, mod_ClosedFormField.jl:616-659):
// s[a][q] = Σ_m E_f[m][a] w (A_f[m][q] e^{i kzf z} + direct) + E_b[m][a] w (A_b ... )
__device__ __forceinline__ void strengths_row(const SynthParams& p, long node, double z, cd W, const cd Af[2][3],
                                              const cd Ab[2][3], const cd kzf[2], const cd kzb[2], const cd ef[2][3],
                                              const cd eb[2][3], cd s[3][3]) {
  // the direct term (direct_amp) is formed per mode inline: sf[m][q] e^{i Qf zeta} above the
  // source, sb[m][q] e^{i Qb zeta} below it, exact zeros elsewhere (as direct_amp's arrays)
  const CacheView& c = p.c;
  const double zeta = z - p.zpos;
  const bool dir = p.with_direct && c.valid[node];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) s[a][b] = cd{0, 0};
#pragma unroll
  for (int m = 0; m < 2; ++m) {
    const cd pf = phase_cl(kzf[m], z);
    const cd pb = phase_cl(kzb[m], z - p.d_obs);
    cd edf{0.0, 0.0}, edb{0.0, 0.0};
    const bool up = dir && zeta > 0, dn = dir && zeta < 0;
    if (up) edf = phase_cl(ldc(c.Qf, m, c.n, node), zeta);
    if (dn) edb = phase_cl(ldc(c.Qb, m, c.n, node), zeta);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      cd tf = Af[m][q] * pf, tb = Ab[m][q] * pb;
      if (p.with_direct) {
        tf += up ? ldc(c.sf, m + 2 * q, c.n, node) * edf : cd{0.0, 0.0};
        tb += dn ? ldc(c.sb, m + 2 * q, c.n, node) * edb : cd{0.0, 0.0};
      }
      const cd af = fin0(W * tf), ab = fin0(W * tb);
#pragma unroll
      for (int a = 0; a < 3; ++a) s[a][q] += ef[m][a] * af + eb[m][a] * ab;
    }
  }
}

// ------------------------------------------------------------------------------------
// one pixel of the 1D assembly: the order sums g0[5], g1[4], g2[4] of its radius combined
// into the 3x3 dyadic of the frame along the pixel's azimuth, then rotated to (x, y):
// G = Rot R Rotᵀ, written at pix + npix (zi + nz (cc + 3 q))
__device__ __forceinline__ void assemble1d_pixel(double x, double y, const cd g0[5], const cd g1[4], const cd g2[4],
                                                 long pix, long npix, int zi, int nz, double2* G) {
  cd R[3][3];
  R[0][0] = g0[0] + g2[0];
  R[1][0] = g0[1] + g2[1];
  R[2][0] = g1[0];
  R[0][1] = g0[2] + g2[2];
  R[1][1] = g0[3] + g2[3];
  R[2][1] = g1[1];
  R[0][2] = g1[2];
  R[1][2] = g1[3];
  R[2][2] = g0[4];
  double rho = hypot(x, y);
  double cp = rho == 0.0 ? 1.0 : x / rho, sp = rho == 0.0 ? 0.0 : y / rho;
  double Rot[3][3] = {{cp, -sp, 0.0}, {sp, cp, 0.0}, {0.0, 0.0, 1.0}};
  for (int q = 0; q < 3; ++q)
    for (int cc = 0; cc < 3; ++cc) {
      cd s{0, 0};
      for (int a = 0; a < 3; ++a) {
        cd tt = Rot[cc][0] * R[0][a] + Rot[cc][1] * R[1][a] + Rot[cc][2] * R[2][a];
        s += tt * Rot[q][a];
      }
      G[pix + npix * (zi + (long)nz * (cc + 3 * q))] = make_double2(s.x, s.y);
    }
}

__global__ void k_assemble1d(int nx, int ny, int nz, const double* xs, const double* ys, const int* rmap, int nr,
                             const double* P0, const double* P1, const double* P2, double2* G) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long npix = (long)nx * ny;
  if (t >= npix * nz) return;
  long pix = t % npix;
  int zi = (int)(t / npix);
  int i = (int)(pix % nx), j = (int)(pix / nx);
  int r = rmap[pix];
  const long n0 = (long)C1D_R0 * nz, n1 = (long)C1D_R1 * nz, n2 = (long)C1D_R2 * nz;
  cd g0[5], g1[4], g2[4];
  unpack_order_sums([&](int c) { const long o = (long)r * n0 + 2L * (zi * 3 + c); return cd{P0[o], P0[o + 1]}; },
                    [&](int c) { const long o = (long)r * n1 + 2L * (zi * 4 + c); return cd{P1[o], P1[o + 1]}; },
                    [&](int c) { const long o = (long)r * n2 + 2L * (zi * 2 + c); return cd{P2[o], P2[o + 1]}; },
                    g0, g1, g2);
  assemble1d_pixel(xs[i], ys[j], g0, g1, g2, pix, npix, zi, nz, G);
}

cudaError_t launch_assemble1d(int nx, int ny, int nz, const double* xs, const double* ys, const int* rmap, int nr,
                              const double* P0, const double* P1, const double* P2, double2* G, cudaStream_t s) {
  long tot = (long)nx * ny * nz;
  k_assemble1d<<<(unsigned)((tot + 127) / 128), 128, 0, s>>>(nx, ny, nz, xs, ys, rmap, nr, P0, P1, P2, G);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// 2D strengths per (node, z-row): S[col'][n], col' = zi + nz (c + 3q)
// One thread per (node, group of SG_Z z-rows): the reflected amplitudes (z-independent) and
// the mode basis are formed once per group. With `colmax` set, the kernel also reduces
// max(|Re S|, |Im S|) over each (node slice of `kchunk` nodes, column): a warp max (a warp's
// 32 nodes lie in one slice, kchunk being a multiple of 32) and one atomicMax per warp on
// the IEEE bits, which order like the values for non-negative doubles (Inf/NaN sort above
// every finite value, so a non-finite strength shows in the slice's maximum).
// ------------------------------------------------------------------------------------
constexpr int SG_Z = 8;  // z-rows per thread

__global__ void __launch_bounds__(128) k_strengths2d(SynthParams p, double2* S, unsigned long long* colmax, long kchunk) {
  const long nidx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const CacheView& c = p.c;
  const long n = c.n;
  const bool live = nidx < n;
  const long node = live ? nidx : n - 1;
  const long k = node % c.Nk, pp = node / c.Nk;
  const double w = c.kr[k] * c.wr[k] * c.wphi[pp] / (4.0 * 3.14159265358979323846 * 3.14159265358979323846);
  const cd W{w, 0.0};
  cd Af[2][3], Ab[2][3];
  reflected_amp(p, node, Af, Ab);
  cd kzf[2], kzb[2], ef[2][3], eb[2][3];
  load_obs_basis(c, node, kzf, kzb, ef, eb);
  const int z0 = blockIdx.y * SG_Z, z1 = min(p.nz, z0 + SG_Z);
  for (int zi = z0; zi < z1; ++zi) {
    cd s[3][3];
    strengths_row(p, node, p.zo[zi], W, Af, Ab, kzf, kzb, ef, eb, s);
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        const long col = zi + (long)p.nz * (cc + 3 * q);
        if (live) S[col * n + nidx] = make_double2(s[cc][q].x, s[cc][q].y);
        if (colmax) {
          double m = live ? fmax(fabs(s[cc][q].x), fabs(s[cc][q].y)) : 0.0;
          if (live && !(isfinite(s[cc][q].x) && isfinite(s[cc][q].y))) m = __longlong_as_double(0x7ff0000000000000LL);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
          // fmax drops a NaN operand; Inf (set above for any non-finite entry) survives
          if ((threadIdx.x & 31) == 0 && live)
            atomicMax(colmax + (nidx / kchunk) * (long)(9 * p.nz) + col, (unsigned long long)__double_as_longlong(m));
        }
      }
  }
}

// ------------------------------------------------------------------------------------
// The same strengths in two kernels, for callers that give a scratch array `amp`:
// k_reflect2d writes each node's reflected amplitudes (A_f, A_b: 12 complex, node fastest)
// once; k_strengths_rows stages 32 nodes' amplitudes, basis, seeds and q's in shared memory
// (coalesced, once per block), then each of its 4 warps takes every fourth z row of the 32
// nodes, one node per lane. The arithmetic per row is strengths_row's, in the same order.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 4) k_reflect2d(SynthParams p, double2* __restrict__ amp) {
  const long node = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long n = p.c.n;
  if (node >= n) return;
  cd Af[2][3], Ab[2][3];
  reflected_amp(p, node, Af, Ab);
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      amp[(long)(3 * m + q) * n + node] = make_double2(Af[m][q].x, Af[m][q].y);
      amp[(long)(6 + 3 * m + q) * n + node] = make_double2(Ab[m][q].x, Ab[m][q].y);
    }
}

// 1D coefficient columns from the reflected amplitudes k_reflect2d wrote once per node (the
// amplitudes do not depend on the z row); the arithmetic per (node, row) is k_coef1d's
// heights per thread of k_coef1d_amp: a node's amplitudes are loaded once for COEF1D_ZB
// z rows (the per-row arithmetic and outputs are those of one row per thread)
constexpr int COEF1D_ZB = 4;

// T = double for the FP64 contraction; float for the int8x3 one, whose digit images need 24
// significant bits (an FP32 rounding of a column's value adds at most half a step of its
// fixed-point scale) and whose coefficient columns are then half the memory traffic
template <class T>
__global__ void __launch_bounds__(128) k_coef1d_amp(SynthParams p, const double2* __restrict__ amp, T* C0, T* C1,
                                                     T* C2) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long n = p.c.n;
  if (k >= n) return;
  cd Af[2][3], Ab[2][3];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      Af[m][q] = ldc(amp, 3 * m + q, n, k);
      Ab[m][q] = ldc(amp, 6 + 3 * m + q, n, k);
    }
  const int z0 = blockIdx.y * COEF1D_ZB;
  const int z1 = min(p.nz, z0 + COEF1D_ZB);
  for (int zi = z0; zi < z1; ++zi) {
    cd c0[5], c1[4], c2[4];
    coef1d_row(p, k, p.zo[zi], Af, Ab, c0, c1, c2);
    store_coef_row(C0, C1, C2, n, k, zi, c0, c1, c2);
  }
}

template <class T>
static cudaError_t coef1d_amp_impl(const SynthParams& p, double2* amp, T* C0, T* C1, T* C2, cudaStream_t s) {
  if (p.c.n <= 0 || p.nz <= 0) return cudaSuccess;
  k_reflect2d<<<(unsigned)((p.c.n + 127) / 128), 128, 0, s>>>(p, amp);
  k_coef1d_amp<T><<<dim3((unsigned)((p.c.n + 127) / 128), (unsigned)((p.nz + COEF1D_ZB - 1) / COEF1D_ZB)), 128, 0, s>>>(
      p, amp, C0, C1, C2);
  return cudaGetLastError();
}

cudaError_t launch_coef1d_amp(const SynthParams& p, double2* amp, double* C0, double* C1, double* C2, cudaStream_t s) {
  return coef1d_amp_impl<double>(p, amp, C0, C1, C2, s);
}

cudaError_t launch_coef1d_amp(const SynthParams& p, double2* amp, float* C0, float* C1, float* C2, cudaStream_t s) {
  return coef1d_amp_impl<float>(p, amp, C0, C1, C2, s);
}

// per node of a k_strengths_rows block: 12 amplitudes, the obs-layer basis (16), sf, sb (6 each),
// Qf, Qb (2 each)
constexpr int SR_F = 44;
// at most 128 registers: four CTAs per SM (no spills)
__global__ void __launch_bounds__(128, 4) k_strengths_rows(SynthParams p, const double2* __restrict__ amp,
                                                         double2* __restrict__ S, unsigned long long* colmax,
                                                         long kchunk) {
  __shared__ double2 sh[SR_F][32];
  __shared__ double wsh[32];
  __shared__ int vsh[32];
  const CacheView& c = p.c;
  const long n = c.n;
  const long node0 = (long)blockIdx.x * 32;
  const int tid = threadIdx.x, lane = tid & 31;
  // stage the 32 nodes' inputs: field f of node node0 + j at sh[f][j] (coalesced over j)
  for (int e = tid; e < SR_F * 32; e += 128) {
    const int j = e & 31, f = e >> 5;
    const long node = min(node0 + j, n - 1);
    const double2* src;
    long fe;
    if (f < 12) { src = amp; fe = f; }
    else if (f < 28) { src = c.basis; fe = f - 12; }
    else if (f < 34) { src = c.sf; fe = f - 28; }
    else if (f < 40) { src = c.sb; fe = f - 34; }
    else if (f < 42) { src = c.Qf; fe = f - 40; }
    else { src = c.Qb; fe = f - 42; }
    sh[f][j] = src[fe * n + node];
  }
  if (tid < 32) {
    const long node = min(node0 + tid, n - 1);
    const long k = node % c.Nk, pp = node / c.Nk;
    wsh[tid] = c.kr[k] * c.wr[k] * c.wphi[pp] / (4.0 * 3.14159265358979323846 * 3.14159265358979323846);
    vsh[tid] = c.valid[node];
  }
  __syncthreads();
  const long nidx = node0 + lane;
  const bool live = nidx < n;
  auto g = [&](int f) { const double2 v = sh[f][lane]; return cd{v.x, v.y}; };
  const cd W{wsh[lane], 0.0};
  const bool dir = p.with_direct && vsh[lane];
  for (int zi = tid >> 5; zi < p.nz; zi += 4) {
    const double z = p.zo[zi];
    const double zeta = z - p.zpos;
    cd s[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) s[a][b] = cd{0, 0};
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      const cd pf = phase_cl(g(24 + m), z);            // basis element 12 + m: kzf
      const cd pb = phase_cl(g(26 + m), z - p.d_obs);  // basis element 14 + m: kzb
      cd edf{0.0, 0.0}, edb{0.0, 0.0};
      const bool up = dir && zeta > 0, dn = dir && zeta < 0;
      if (up) edf = phase_cl(g(40 + m), zeta);
      if (dn) edb = phase_cl(g(42 + m), zeta);
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        cd tf = g(3 * m + q) * pf, tb = g(6 + 3 * m + q) * pb;
        if (p.with_direct) {
          tf += up ? g(28 + m + 2 * q) * edf : cd{0.0, 0.0};
          tb += dn ? g(34 + m + 2 * q) * edb : cd{0.0, 0.0};
        }
        const cd af = fin0(W * tf), ab = fin0(W * tb);
#pragma unroll
        for (int a = 0; a < 3; ++a) s[a][q] += g(12 + 2 * a + m) * af + g(18 + 2 * a + m) * ab;
      }
    }
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        const long col = zi + (long)p.nz * (cc + 3 * q);
        if (live) S[col * n + nidx] = make_double2(s[cc][q].x, s[cc][q].y);
        if (colmax) {
          double mx = live ? fmax(fabs(s[cc][q].x), fabs(s[cc][q].y)) : 0.0;
          if (live && !(isfinite(s[cc][q].x) && isfinite(s[cc][q].y))) mx = __longlong_as_double(0x7ff0000000000000LL);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
          if (lane == 0 && live)
            atomicMax(colmax + (nidx / kchunk) * (long)(9 * p.nz) + col, (unsigned long long)__double_as_longlong(mx));
        }
      }
  }
}

cudaError_t launch_strengths2d(const SynthParams& p, double2* S, cudaStream_t s, unsigned long long* colmax, long kchunk,
                               double2* amp) {
  if (p.c.n <= 0) return cudaSuccess;
  if (colmax && (kchunk <= 0 || kchunk % 32 != 0)) return cudaErrorInvalidValue;
  if (amp) {
    k_reflect2d<<<(unsigned)((p.c.n + 127) / 128), 128, 0, s>>>(p, amp);
    k_strengths_rows<<<(unsigned)((p.c.n + 31) / 32), 128, 0, s>>>(p, amp, S, colmax, kchunk);
    return cudaGetLastError();
  }
  dim3 grid((unsigned)((p.c.n + 127) / 128), (unsigned)((p.nz + SG_Z - 1) / SG_Z));
  k_strengths2d<<<grid, 128, 0, s>>>(p, S, colmax, kchunk);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// 2D lateral sum: G[pix][col] = Σ_n e^{i(kx_n x_i + ky_n y_j)} S[col][n] (complex FP64)
// Tile: 64 pixels x 32 columns, 16 nodes per stage; 256 threads, 4 pixels x 2 columns each.
// The phase operand is generated per stage in shared memory (sincos per node and
// coordinate, then one complex product per (node, pixel)).
// ------------------------------------------------------------------------------------
constexpr int LP = 64, LC = 32, LK = 16;
__global__ void __launch_bounds__(256) k_lateral(CacheView c, int nx, int ny, const double* __restrict__ xs,
                                                 const double* __restrict__ ys, int ncol, const double2* __restrict__ S,
                                                 double2* __restrict__ Gp, long kchunk) {
  __shared__ double2 Ps[LK][LP];
  __shared__ double2 Ss[LK][LC];
  __shared__ double kxs[LK], kys[LK];
  const long npix = (long)nx * ny;
  const long p0 = (long)blockIdx.x * LP;
  const int c0 = blockIdx.y * LC;
  const int sp = blockIdx.z;
  const long n = c.n;
  const long k0 = (long)sp * kchunk, k1 = min(n, k0 + kchunk);
  const int tid = threadIdx.x;
  const int tp = tid % 16, tc = tid / 16;  // pixels tp + 16 a (a < 4), columns tc + 16 b (b < 2)
  double2 acc[4][2];
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 2; ++b) acc[a][b] = make_double2(0.0, 0.0);
  for (long kk = k0; kk < k1; kk += LK) {
    if (tid < LK) {
      long nn = kk + tid;
      double kx = 0.0, ky = 0.0;
      if (nn < k1) {
        long k = nn % c.Nk, q = nn / c.Nk;
        double s, co;
        sincos(c.phi[q], &s, &co);
        kx = c.kr[k] * co;
        ky = c.kr[k] * s;
      }
      kxs[tid] = kx;
      kys[tid] = ky;
    }
    __syncthreads();
    // phases: LK x LP = 1024 products, 4 per thread
    for (int e = 0; e < 4; ++e) {
      int idx = tid + 256 * e;
      int t = idx / LP, pl = idx % LP;
      long pix = p0 + pl;
      double2 v = make_double2(0.0, 0.0);
      if (pix < npix && kk + t < k1) {
        int i = (int)(pix % nx), j = (int)(pix / nx);
        double sx, cx, sy, cy;
        sincos(kxs[t] * xs[i], &sx, &cx);
        sincos(kys[t] * ys[j], &sy, &cy);
        v = make_double2(cx * cy - sx * sy, cx * sy + sx * cy);
      }
      Ps[t][pl] = v;
    }
    // strengths: LK x LC = 512, 2 per thread
    for (int e = 0; e < 2; ++e) {
      int idx = tid + 256 * e;
      int t = idx % LK, cl = idx / LK;
      long nn = kk + t;
      int col = c0 + cl;
      Ss[t][cl] = (nn < k1 && col < ncol) ? S[(long)col * n + nn] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll 4
    for (int t = 0; t < LK; ++t) {
      double2 pv[4], sv[2];
      for (int a = 0; a < 4; ++a) pv[a] = Ps[t][tp + 16 * a];
      for (int b = 0; b < 2; ++b) sv[b] = Ss[t][tc + 16 * b];
      for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 2; ++b) {
          acc[a][b].x = fma(pv[a].x, sv[b].x, fma(-pv[a].y, sv[b].y, acc[a][b].x));
          acc[a][b].y = fma(pv[a].x, sv[b].y, fma(pv[a].y, sv[b].x, acc[a][b].y));
        }
    }
    __syncthreads();
  }
  double2* G = Gp + (long)sp * npix * ncol;
  for (int a = 0; a < 4; ++a) {
    long pix = p0 + tp + 16 * a;
    if (pix >= npix) continue;
    for (int b = 0; b < 2; ++b) {
      int col = c0 + tc + 16 * b;
      if (col < ncol) G[pix + npix * col] = acc[a][b];
    }
  }
}

__global__ void k_reduce_splits2(long len, int splits, const double2* __restrict__ P, double2* __restrict__ C) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len) return;
  double2 s = make_double2(0.0, 0.0);
  for (int k = 0; k < splits; ++k) {
    double2 v = P[(long)k * len + i];
    s.x += v.x;
    s.y += v.y;
  }
  C[i] = s;
}

int lateral_splits(long n, int splits) {
  long kchunk = (n + splits - 1) / splits;
  kchunk = ((kchunk + LK - 1) / LK) * LK;
  if (kchunk <= 0) return 1;
  return (int)std::max(1L, (n + kchunk - 1) / kchunk);
}

cudaError_t launch_lateral(const CacheView& c, int nx, int ny, const double* xs, const double* ys, int ncol, const double2* S,
                           double2* partial, int splits, cudaStream_t s) {
  long npix = (long)nx * ny;
  splits = lateral_splits(c.n, splits);
  long kchunk = (c.n + splits - 1) / splits;
  kchunk = ((kchunk + LK - 1) / LK) * LK;
  dim3 grid((unsigned)((npix + LP - 1) / LP), (unsigned)((ncol + LC - 1) / LC), (unsigned)splits);
  k_lateral<<<grid, 256, 0, s>>>(c, nx, ny, xs, ys, ncol, S, partial, kchunk);
  return cudaGetLastError();
}

cudaError_t launch_reduce_splits2(long len, int splits, const double2* partial, double2* G, cudaStream_t s) {
  if (len <= 0) return cudaSuccess;
  k_reduce_splits2<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(len, splits, partial, G);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// gl_rule panel expansion (mod_KxGrid.jl:361-384), no FMA contraction: bit-exact with a
// CPU evaluation of the same expressions in IEEE double
// ------------------------------------------------------------------------------------
__global__ void k_gl_nodes(int npanels, const double* pa, const double* pb, const int* sing_side, const double* xi,
                           const double* wx, int order, double* nodes, double* wts) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)npanels * order) return;
  int pi = (int)(t / order), j = (int)(t % order);
  double a = pa[pi], b = pb[pi];
  int sg = sing_side[pi];  // 0 regular, +1 singular at a, -1 singular at b
  if (sg == 0) {
    double h = __dmul_rn(0.5, __dsub_rn(b, a));
    double cc = __dmul_rn(0.5, __dadd_rn(a, b));
    nodes[t] = __dadd_rn(cc, __dmul_rn(h, xi[j]));
    wts[t] = __dmul_rn(h, wx[j]);
  } else {
    double L = sg > 0 ? a : b;
    double U = __dsqrt_rn(__dsub_rn(b, a));
    double hU = __dmul_rn(0.5, U);
    double u = __dmul_rn(hU, __dadd_rn(1.0, xi[j]));
    nodes[t] = __dadd_rn(L, __dmul_rn((double)sg, __dmul_rn(u, u)));
    wts[t] = __dmul_rn(__dmul_rn(hU, wx[j]), __dmul_rn(2.0, u));
  }
}

cudaError_t launch_gl_nodes(int npanels, const double* pa, const double* pb, const int* sing_side, const double* xi,
                            const double* wx, int order, double* nodes, double* wts, cudaStream_t s) {
  long tot = (long)npanels * order;
  if (tot == 0) return cudaSuccess;
  k_gl_nodes<<<(unsigned)((tot + 127) / 128), 128, 0, s>>>(npanels, pa, pb, sing_side, xi, wx, order, nodes, wts);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// Batched synthesis of many small observation sets (uneven batches, one graph launch).
// Work unit = (item, chunk of nodes), pulled by persistent CTAs from a counter. Per
// sub-batch of SYN_SB = 64 nodes, threads 0-63 take one node each and form in shared memory
//   2D: its strengths S[node][col] (col = zi + nz (cc + 3 q)), reflected amplitudes first;
//   1D: its coefficient columns C[node][zi 13 + m] (m: 5 of order 0, 4 of order 1, 4 of
//       order 2);
// while threads 64-127 form for the same nodes
//   2D: the phases P[node][pix] = e^{i kx x} e^{i ky y} (one sincos per x and per y);
//   1D: the tables J_n(kρ ρ_r), n = 0, 1, 2;
// then all threads accumulate the outputs o = row + nrow col of the item's partial sum (2D
// rows: pixels; 1D rows: distinct radii) in shared memory, a strided set of outputs each,
// over the sub-batch's nodes in registers. The shared arrays are laid out with the item's own
// sizes. k_synth_finish sums the chunks of each output in chunk order (2D) or sums them and
// assembles the pixel (1D).
// ------------------------------------------------------------------------------------
constexpr int SYN_SB = 64;

// shared bytes of one item's work unit
__host__ __device__ __forceinline__ size_t synth_item_smem(int is2d, int npix, int nr, int nz) {
  const size_t nout = is2d ? (size_t)npix * 9 * nz : (size_t)nr * 13 * nz;
  if (is2d) return 16 * nout + (size_t)SYN_SB * (npix + 9 * nz) * 16;
  return 16 * nout + (size_t)SYN_SB * 3 * nr * 8 + (size_t)SYN_SB * 13 * nz * 16;
}

size_t synth_small_smem(int is2d, int npix, int nr, int nz) { return synth_item_smem(is2d, npix, nr, nz); }

size_t synth_small_smem() {
  const size_t a = synth_item_smem(1, SYN_MAXPIX, 0, SYN_MAXZ), b = synth_item_smem(0, 0, SYN_MAXR, SYN_MAXZ);
  return a > b ? a : b;
}

__device__ __forceinline__ int find_item(const long* __restrict__ off, int nb, long t) {
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(128, 3) k_synth_small(const SynthItem* __restrict__ items, int nitems,
                                                      const long* __restrict__ w_off, long nwork, unsigned* counter,
                                                      int chunk) {
  extern __shared__ __align__(16) unsigned char syn_smem[];
  __shared__ long wsh;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) wsh = (long)atomicAdd(counter, 1u);
    __syncthreads();
    const long w = wsh;
    __syncthreads();
    if (w >= nwork) return;
    const int it = find_item(w_off, nitems, w);
    const SynthItem& I = items[it];
    const SynthParams& p = I.sp;
    const CacheView& c = p.c;
    const long cid = w - w_off[it];
    const long k0 = cid * chunk, k1 = min(c.n, k0 + chunk);
    const int nz = p.nz, npix = I.nx * I.ny;
    const bool two = I.is2d != 0;
    const int ncol = two ? 9 * nz : 13 * nz;
    const int nrow = two ? npix : I.nr;
    const int nout = nrow * ncol;
    cd* acc = reinterpret_cast<cd*>(syn_smem);                      // [nout]
    cd* Ss = acc + nout;                                            // 2D [SB][ncol]
    cd* Ps = Ss + SYN_SB * ncol;                                    // 2D [SB][npix]
    cd* Cs = acc + nout;                                            // 1D [SB][ncol]
    double* Js = reinterpret_cast<double*>(Cs + SYN_SB * ncol);     // 1D [SB][3][nr]
    for (int o = tid; o < nout; o += 128) acc[o] = cd{0.0, 0.0};
    for (long b0 = k0; b0 < k1; b0 += SYN_SB) {
      const int nb = (int)min((long)SYN_SB, k1 - b0);
      const int j = tid & (SYN_SB - 1);
      const long node = b0 + j;
      if (j < nb) {
        if (tid < SYN_SB) {
          cd Af[2][3], Ab[2][3];
          reflected_amp(p, node, Af, Ab);
          if (two) {
            const long k = node % c.Nk, pp = node / c.Nk;
            const double wt = c.kr[k] * c.wr[k] * c.wphi[pp] / (4.0 * 3.14159265358979323846 * 3.14159265358979323846);
            cd kzf[2], kzb[2], ef[2][3], eb[2][3];
            load_obs_basis(c, node, kzf, kzb, ef, eb);
            for (int zi = 0; zi < nz; ++zi) {
              cd sv[3][3];
              strengths_row(p, node, p.zo[zi], cd{wt, 0.0}, Af, Ab, kzf, kzb, ef, eb, sv);
              for (int q = 0; q < 3; ++q)
                for (int cc = 0; cc < 3; ++cc) Ss[j * ncol + zi + nz * (cc + 3 * q)] = sv[cc][q];
            }
          } else {
            for (int zi = 0; zi < nz; ++zi) {
              cd c0[5], c1[4], c2[4];
              coef1d_row(p, node, p.zo[zi], Af, Ab, c0, c1, c2);
              cd* dst = Cs + j * ncol + 13 * zi;
              for (int m = 0; m < 5; ++m) dst[m] = c0[m];
              for (int m = 0; m < 4; ++m) { dst[5 + m] = c1[m]; dst[9 + m] = c2[m]; }
            }
          }
        } else if (two) {
          const long k = node % c.Nk, pp = node / c.Nk;
          double sn, cs;
          sincos(c.phi[pp], &sn, &cs);
          const double kx = c.kr[k] * cs, ky = c.kr[k] * sn;
          double sy[8], cy[8];
          const int ny8 = min(I.ny, 8);
          for (int jj = 0; jj < ny8; ++jj) sincos(ky * I.ys[jj], &sy[jj], &cy[jj]);
          for (int i = 0; i < I.nx; ++i) {
            double sx, cx;
            sincos(kx * I.xs[i], &sx, &cx);
            for (int jj = 0; jj < I.ny; ++jj) {
              double s2, c2;
              if (jj < 8) { s2 = sy[jj]; c2 = cy[jj]; }
              else sincos(ky * I.ys[jj], &s2, &c2);
              Ps[j * npix + i + I.nx * jj] = cd{cx * c2 - sx * s2, cx * s2 + sx * c2};
            }
          }
        } else {
          const double kx = c.kr[node];
          double* dst = Js + j * 3 * I.nr;
          for (int r = 0; r < I.nr; ++r) {
            double a0, a1, a2;
            bessel_j012(kx * I.rho[r], a0, a1, a2);
            dst[r] = a0;
            dst[I.nr + r] = a1;
            dst[2 * I.nr + r] = a2;
          }
        }
      }
      __syncthreads();
      for (int o = tid; o < nout; o += 128) {
        const int row = o % nrow, cidx = o / nrow;
        cd a = acc[o];
        if (two) {
          const cd* pp = Ps + row;
          const cd* sp = Ss + cidx;
          for (int t = 0; t < nb; ++t) {
            const cd pv = pp[t * npix], sv = sp[t * ncol];
            a.x = fma(pv.x, sv.x, fma(-pv.y, sv.y, a.x));
            a.y = fma(pv.x, sv.y, fma(pv.y, sv.x, a.y));
          }
        } else {
          const int m = cidx % 13;
          const int ord = m < 5 ? 0 : (m < 9 ? 1 : 2);
          const double* jp = Js + ord * I.nr + row;
          const cd* cp = Cs + cidx;
          for (int t = 0; t < nb; ++t) {
            const double jv = jp[t * 3 * I.nr];
            const cd cv = cp[t * ncol];
            a.x = fma(jv, cv.x, a.x);
            a.y = fma(jv, cv.y, a.y);
          }
        }
        acc[o] = a;
      }
      __syncthreads();
    }
    double2* out = I.partial + cid * (long)nout;
    for (int o = tid; o < nout; o += 128) out[o] = make_double2(acc[o].x, acc[o].y);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(128) k_synth_finish(const SynthItem* __restrict__ items, int nitems,
                                                       const long* __restrict__ f_off, long nfin) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nfin) return;
  const int it = find_item(f_off, nitems, t);
  const SynthItem& I = items[it];
  const long u = t - f_off[it];
  const int nz = I.sp.nz;
  const long npix = (long)I.nx * I.ny;
  if (I.is2d) {
    const long nout = npix * 9 * nz;
    double2 s = make_double2(0.0, 0.0);
    for (int k = 0; k < I.nw; ++k) {
      const double2 v = I.partial[(long)k * nout + u];
      s.x += v.x;
      s.y += v.y;
    }
    I.G[u] = s;
    return;
  }
  const long pix = u % npix;
  const int zi = (int)(u / npix);
  const int r = I.rmap[pix];
  const long nout = (long)I.nr * 13 * nz;
  cd g[13];
  for (int m = 0; m < 13; ++m) {
    cd s{0.0, 0.0};
    const long o = r + (long)I.nr * (13 * zi + m);
    for (int k = 0; k < I.nw; ++k) {
      const double2 v = I.partial[(long)k * nout + o];
      s.x += v.x;
      s.y += v.y;
    }
    g[m] = s;
  }
  const int i = (int)(pix % I.nx), j = (int)(pix / I.nx);
  assemble1d_pixel(I.xs[i], I.ys[j], g, g + 5, g + 9, pix, npix, zi, nz, I.G);
}

cudaError_t synth_small_init() {
  return cudaFuncSetAttribute(k_synth_small, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)synth_small_smem());
}

cudaError_t launch_synth_small(const SynthItem* items, int nitems, const long* w_off, long nwork, unsigned* counter,
                               int chunk, int grid, size_t smem, cudaStream_t s) {
  if (nwork <= 0) return cudaSuccess;
  if (grid <= 0 || chunk <= 0 || smem > synth_small_smem()) return cudaErrorInvalidValue;
  k_synth_small<<<grid, 128, smem, s>>>(items, nitems, w_off, nwork, counter, chunk);
  return cudaGetLastError();
}

cudaError_t launch_synth_finish(const SynthItem* items, int nitems, const long* f_off, long nfin, cudaStream_t s) {
  if (nfin <= 0) return cudaSuccess;
  k_synth_finish<<<(unsigned)((nfin + 127) / 128), 128, 0, s>>>(items, nitems, f_off, nfin);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// Grouped 1D synthesis (int8x3 path): the reflected amplitudes, the FP32 coefficient columns
// and the final slice sum + pixel assembly of every item of a group, one launch each. The
// per-node and per-pixel arithmetic is that of k_reflect2d, k_coef1d_amp and k_assemble1d.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 4) k_reflect2d_group(const Synth1DItem* __restrict__ items,
                                                            const long* __restrict__ first, int ni) {
  const int i = group_entry(first, ni, blockIdx.x);
  const Synth1DItem& it = items[i];
  const long n = it.sp.c.n;
  const long node = (long)(blockIdx.x - first[i]) * blockDim.x + threadIdx.x;
  if (node >= n) return;
  cd Af[2][3], Ab[2][3];
  reflected_amp(it.sp, node, Af, Ab);
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      it.amp[(long)(3 * m + q) * n + node] = make_double2(Af[m][q].x, Af[m][q].y);
      it.amp[(long)(6 + 3 * m + q) * n + node] = make_double2(Ab[m][q].x, Ab[m][q].y);
    }
}

// a read-only load the compiler keeps in place (volatile asm: not hoisted out of the row loop),
// so the node's mode fields are re-read from L1 per row instead of held in registers
__device__ __forceinline__ cd ldc_row(const double2* b, long e, long n, long i) {
  double x, y;
  asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(x), "=d"(y) : "l"(b + e * n + i));
  return cd{x, y};
}

// the 13 coefficient columns of one (node, z row) of the scattered terms (no direct term), as
// coef1d_row, from the W-weighted amplitudes (fin0 applied; shared memory, aw[(m 2 + br) 3 + q]
// [thread]) and the four branch phases g[m][br] (phase_cl(kz, z or z - d_obs) kx)
__device__ __forceinline__ void coef_row_scat(const CacheView& c, long k, const double2 (*aw)[128], const cd g[2][2],
                                              cd c0[5], cd c1[4], cd c2[4]) {
  const long n = c.n;
  const cd half_i{0.0, 0.5};
#pragma unroll
  for (int i = 0; i < 5; ++i) c0[i] = cd{0, 0};
#pragma unroll
  for (int i = 0; i < 4; ++i) { c1[i] = cd{0, 0}; c2[i] = cd{0, 0}; }
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int br = 0; br < 2; ++br) {
      const cd ex = ldc_row(c.basis, (br == 0 ? 0 : 6) + m, n, k);
      const cd ey = ldc_row(c.basis, (br == 0 ? 2 : 8) + m, n, k);
      const cd ez = ldc_row(c.basis, (br == 0 ? 4 : 10) + m, n, k);
      const int e0 = (m * 2 + br) * 3;
      const double2 a0 = aw[e0][threadIdx.x], a1 = aw[e0 + 1][threadIdx.x], a2 = aw[e0 + 2][threadIdx.x];
      const cd ax = cd{a0.x, a0.y} * g[m][br], ay = cd{a1.x, a1.y} * g[m][br], az = cd{a2.x, a2.y} * g[m][br];
      c0[0] += half_i * (-(ax * ex) - ay * ey);
      c2[0] += half_i * (ax * ex - ay * ey);
      c0[1] += half_i * (-(ax * ey) + ay * ex);
      c2[1] += half_i * (ax * ey + ay * ex);
      c1[0] += ax * ez;
      c0[2] += half_i * (-(ay * ex) + ax * ey);
      c2[2] += half_i * (ay * ex + ax * ey);
      c0[3] += half_i * (-(ay * ey) - ax * ex);
      c2[3] += half_i * (ay * ey - ax * ex);
      c1[1] += ay * ez;
      c1[2] += az * ex;
      c1[3] += az * ey;
      c0[4] += cd{0.0, -1.0} * (az * ez);
    }
}

// rows z0..z1-1 of a node with the same-layer direct term (coef1d_row), out of line so that its
// registers and local arrays stay out of the scattered path
__device__ __noinline__ void coef_rows_direct(const Synth1DItem& it, long k, int z0, int z1) {
  const SynthParams& p = it.sp;
  const long n = p.c.n;
  const int nz = p.nz;
  const long cst = it.ldc;  // row stride of the coefficient columns
  float* C0 = it.C;
  float* C1 = it.C + (long)C1D_OFF1 * nz * cst;
  float* C2 = it.C + (long)C1D_OFF2 * nz * cst;
  cd Af[2][3], Ab[2][3];
  for (int m = 0; m < 2; ++m)
    for (int q = 0; q < 3; ++q) {
      Af[m][q] = ldc(it.amp, 3 * m + q, n, k);
      Ab[m][q] = ldc(it.amp, 6 + 3 * m + q, n, k);
    }
  for (int zi = z0; zi < z1; ++zi) {
    cd c0[5], c1[4], c2[4];
    coef1d_row(p, k, p.zo[zi], Af, Ab, c0, c1, c2);
    store_coef_row(C0, C1, C2, cst, k, zi, c0, c1, c2);
  }
}

// e^{a + i b}, out of line: the exact phases are the rare case of the recurrence below
__device__ __noinline__ cd cexp_call(double a, double b) { return cexp(cd{a, b}); }

// blocks of an item: ceil(n / 128) node blocks x ceil(nz / COEF1D_ZB_GROUP) height blocks,
// node block fastest. For
// the scattered terms at evenly spaced heights (it.dz != 0) the branch phases of a thread's
// consecutive rows follow by one complex product each, e^{i kz (z + dz)} = e^{i kz z} e^{i kz dz};
// a row whose exponent leaves phase_cl's range (or a step that overflows) takes phase_cl itself.
__global__ void __launch_bounds__(128, 3) k_coef1d_group(const Synth1DItem* __restrict__ items,
                                                      const long* __restrict__ first, int ni) {
  const int i = group_entry(first, ni, blockIdx.x);
  const Synth1DItem& it = items[i];
  const SynthParams& p = it.sp;
  const CacheView& c = p.c;
  const long n = c.n;
  const long nkb = (n + 127) / 128;
  const long b = blockIdx.x - first[i];
  const long k = (b % nkb) * 128 + threadIdx.x;
  if (k >= n) return;
  const int nz = p.nz;
  const long cst = it.ldc;  // row stride of the coefficient columns
  float* C0 = it.C;
  float* C1 = it.C + (long)C1D_OFF1 * nz * cst;
  float* C2 = it.C + (long)C1D_OFF2 * nz * cst;
  const int z0 = (int)(b / nkb) * COEF1D_ZB_GROUP;
  const int z1 = min(nz, z0 + COEF1D_ZB_GROUP);
  if (p.with_direct) {
    coef_rows_direct(it, k, z0, z1);
    return;
  }
  // the node's W-weighted amplitudes and its four kz in shared memory (read once per row and
  // branch; registers hold the row's accumulators and phases)
  __shared__ double2 aw[12][128];
  __shared__ double2 skz[4][128];
  const cd W = cd{0.0, 1.0 / (2.0 * 3.14159265358979323846)} * cd{c.wr[k], 0.0};
  const cd kx{c.kr[k], 0.0};
#pragma unroll
  for (int m = 0; m < 2; ++m) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const cd f = fin0(W * ldc(it.amp, 3 * m + q, n, k)), bk = fin0(W * ldc(it.amp, 6 + 3 * m + q, n, k));
      aw[(m * 2) * 3 + q][threadIdx.x] = make_double2(f.x, f.y);
      aw[(m * 2 + 1) * 3 + q][threadIdx.x] = make_double2(bk.x, bk.y);
    }
    skz[m * 2][threadIdx.x] = c.basis[(12L + m) * n + k];
    skz[m * 2 + 1][threadIdx.x] = c.basis[(14L + m) * n + k];
  }
  const double dz = it.dz;
  cd ph[2][2], step[2][2];
  bool have[2][2];
#pragma unroll
  for (int m = 0; m < 2; ++m)
#pragma unroll
    for (int br = 0; br < 2; ++br) {
      have[m][br] = false;
      ph[m][br] = cd{0, 0};
      const double2 q = skz[m * 2 + br][threadIdx.x];
      step[m][br] = dz != 0.0 ? cexp_call(-q.y * dz, q.x * dz) : cd{0, 0};
      if (!(dz != 0.0 && isfin(step[m][br]))) step[m][br] = cd{0, 0};
    }
  for (int zi = z0; zi < z1; ++zi) {
    const double zf = p.zo[zi], zb = zf - p.d_obs;
    cd g[2][2];
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
      for (int br = 0; br < 2; ++br) {
        const double2 q = skz[m * 2 + br][threadIdx.x];
        const double zz = br == 0 ? zf : zb;
        const double a = -q.y * zz, bb = q.x * zz;
        if (!isfinite(a) || !isfinite(bb) || a > 700.0 || a < -700.0) {
          ph[m][br] = cd{0, 0};
          have[m][br] = false;
        } else if (have[m][br] && (step[m][br].x != 0.0 || step[m][br].y != 0.0)) {
          ph[m][br] = ph[m][br] * step[m][br];
        } else {
          ph[m][br] = cexp_call(a, bb);
          have[m][br] = true;
        }
        g[m][br] = ph[m][br] * kx;
      }
    cd c0[5], c1[4], c2[4];
    coef_row_scat(c, k, aw, g, c0, c1, c2);
    store_coef_row(C0, C1, C2, cst, k, zi, c0, c1, c2);
  }
}

cudaError_t launch_reflect_coef_group(const Synth1DGroup& g, int stage, cudaStream_t s) {
  if (g.ni <= 0) return cudaSuccess;
  if (stage == 0 && g.grid[0] > 0) k_reflect2d_group<<<(unsigned)g.grid[0], 128, 0, s>>>(g.it, g.first_reflect, g.ni);
  if (stage == 1 && g.grid[1] > 0) k_coef1d_group<<<(unsigned)g.grid[1], 128, 0, s>>>(g.it, g.first_coef, g.ni);
  return cudaGetLastError();
}

// one thread per (pixel, height) of an item: P_n(r, c) = Σ_z part_n[z][c][r] (slices in
// order, as k_reduce_transpose), then assemble1d_pixel
__global__ void __launch_bounds__(128) k_assemble1d_group(const Synth1DItem* __restrict__ items,
                                                          const long* __restrict__ first, int ni) {
  const int i = group_entry(first, ni, blockIdx.x);
  const Synth1DItem& it = items[i];
  const long npix = (long)it.nx * it.ny;
  const int nz = it.sp.nz;
  const long t = (long)(blockIdx.x - first[i]) * blockDim.x + threadIdx.x;
  if (t >= npix * nz) return;
  const long pix = t % npix;
  const int zi = (int)(t / npix);
  const int ix = (int)(pix % it.nx), iy = (int)(pix / it.nx);
  const int r = it.rmap[pix];
  const long M = it.nr;
  const int nch = it.nchunk;
  const long N0 = (long)C1D_R0 * nz, N1 = (long)C1D_R1 * nz, N2 = (long)C1D_R2 * nz;
  // the slices' partials summed in order, as k_reduce_transpose
  auto sum = [&](const double* part, long N, long c) {
    double re = 0.0, im = 0.0;
    for (int z = 0; z < nch; ++z) {
      re += part[((long)z * N + c) * M + r];
      im += part[((long)z * N + c + 1) * M + r];
    }
    return cd{re, im};
  };
  cd g0[5], g1[4], g2[4];
  unpack_order_sums([&](int c) { return sum(it.part[0], N0, 2L * (zi * 3 + c)); },
                    [&](int c) { return sum(it.part[1], N1, 2L * (zi * 4 + c)); },
                    [&](int c) { return sum(it.part[2], N2, 2L * (zi * 2 + c)); }, g0, g1, g2);
  assemble1d_pixel(it.xs[ix], it.ys[iy], g0, g1, g2, pix, npix, zi, nz, it.G);
}

cudaError_t launch_assemble1d_group(const Synth1DGroup& g, cudaStream_t s) {
  if (g.ni <= 0 || g.grid[5] <= 0) return cudaSuccess;
  k_assemble1d_group<<<(unsigned)g.grid[5], 128, 0, s>>>(g.it, g.first_asm, g.ni);
  return cudaGetLastError();
}

}  // namespace ytf

// ytf_bessel_i8.cu -- the 1D Bessel synthesis contraction on the int8 tensor cores.
//
// closed_form_G for 1D caches (mod_ClosedFormField.jl:435-487) contracts, per Bessel order n,
//   P_n[r][c] = Σ_k J_n(k_k ρ_r) C_n[c][k]
// (C_n: the real and imaginary parts of the order's coefficient columns, k_coef1d). Both
// operands are fixed point in three signed base-256 digits, as in the 2D lateral kernel:
//   J: X = rint(8355000 J / j_env(k_min ρ))   per (radius, node slice): |J_n| ≤ j_env
//   C: Y = rint(8355000 C / max|C|)   per (node slice, column)
// and the six digit products of weight ≥ 256² are summed exactly in INT32 in tensor memory.
// Unlike the lateral kernel, both operands are prepared once per launch as the exact shared-
// memory image of each 64-node stage (k_aimg_bessel evaluates J_n straight into digits; no
// FP64 table), so the contraction kernel only streams images: warp 0 issues the two bulk
// copies of a stage (one mbarrier, byte-counted), one thread of warp 1 issues the 12 MMAs
// (6 digit products x 2 K-halves; M=128 radii, N ≤ 160 columns, K=32), warps 2-5 read the
// accumulators at the end.
// INT32 headroom: |level-2 sum| ≤ (127·128 + 128·128 + 128·127) K ≤ 48896 · 16384 < 2^30.
#include "ytf_complex.cuh"
#include "ytf_kernels.h"
#include "ytf_tcgen05.cuh"

namespace ytf {

constexpr int BI_M = 128;
constexpr int BI_NODES = 64;  // nodes per stage: one byte each, 64-byte rows (2 MMAs of K = 32)
constexpr int BI_STAGES = 4;
constexpr int BI_THREADS = 192;
constexpr int BI_ACC_STRIDE = 160;
constexpr int BI_TMEM_COLS = 512;
constexpr long BI_WAIT_LIMIT = 1L << 22;  // polls of the drain waits (the pipeline waits: p.wait_limit)
constexpr double BI_SCALE = 8355000.0;

size_t bessel_i8_stage_bytes_a() { return 3ul * BI_M * 64; }
size_t bessel_i8_stage_bytes_b(int Np) { return 3ul * (size_t)Np * 64; }
size_t bessel_i8_smem(int Np) {
  return (size_t)BI_STAGES * (bessel_i8_stage_bytes_a() + bessel_i8_stage_bytes_b(Np)) + 128;
}
int bessel_i8_ctile(int N) {
  int nt = (N + 159) / 160;
  return (N + nt - 1) / nt;
}

// J_2 from J_0, J_1: its power series below |x| = 1 (A&S 9.1.10; exact 0 at x = 0; the term
// ratio -h²/((m + 1)(m + 3)) with the reciprocals as constants) and the three-term recurrence
// above (A&S 9.1.27)
__device__ __forceinline__ double j2_from(double x, double J0, double J1) {
  if (fabs(x) < 1.0) {
    constexpr double inv[12] = {1.0 / 3, 1.0 / 8, 1.0 / 15, 1.0 / 24, 1.0 / 35, 1.0 / 48,
                                1.0 / 63, 1.0 / 80, 1.0 / 99, 1.0 / 120, 1.0 / 143, 1.0 / 168};
    const double h2 = 0.25 * x * x;
    double t = 0.5 * h2, s = t;
#pragma unroll
    for (int m = 0; m < 12; ++m) {
      t *= -h2 * inv[m];
      s += t;
    }
    return s;
  }
  return (2.0 / x) * J1 - J0;
}

// J_0, J_1 (j01_real below: the CUDA math library under x = 25, the asymptotic pair above),
// J_2 from them
__device__ __forceinline__ void j01_real(double x, double& J0, double& J1);
__device__ __forceinline__ double bessel_j012(int order, double x) {
  double J0, J1;
  j01_real(x, J0, J1);
  if (order == 0) return J0;
  if (order == 1) return J1;
  return j2_from(x, J0, J1);
}

// J_0(x) and J_1(x) for x >= 25 (absolute error below 1e-12): Hankel's asymptotic expansions
// (A&S 9.2.5, 9.2.9, 9.2.10), J_n(x) = sqrt(2 / (π x)) (P_n cos χ_n - Q_n sin χ_n) with
// χ_n = x - (2n + 1) π / 4, five terms each of P_n and Q_n in y = 1/x (the coefficient of y^m
// is ±a_m / 8^m, a_m = Π_{j<=m} (4n² - (2j - 1)²) / m!). Both orders share one phase
// (χ_1 = χ_0 - π/2): cos x and sin x from a Cody-Waite reduction by π/2 (a three-part
// constant whose first two parts carry 33 bits, so n π/2 is exact for n < 2^20) and Taylor
// polynomials on |r| <= π/4 (to r^17 and r^18), then cos χ_0 = (cos x + sin x)/√2 and
// sin χ_0 = (sin x - cos x)/√2. The library's j0 and j1 evaluate each order with its own phase.
constexpr double J_ASYM_MIN = 25.0;
__device__ __forceinline__ void j01_large(double x, double& J0, double& J1) {
  const double y = 1.0 / x, y2 = y * y;
  const double p0 = fma(fma(fma(fma(6.074042001273483, y2, -0.5725014209747314), y2, 0.112152099609375), y2,
                            -0.0703125), y2, 1.0);
  const double q0 = y * fma(fma(fma(fma(-24.380529699556064, y2, 1.7277275025844574), y2, -0.22710800170898438), y2,
                                0.0732421875), y2, -0.125);
  const double p1 = fma(fma(fma(fma(-6.883914268109947, y2, 0.6765925884246826), y2, -0.144195556640625), y2,
                            0.1171875), y2, 1.0);
  const double q1 = y * fma(fma(fma(fma(27.248827311268542, y2, -1.993531733751297), y2, 0.2775764465332031), y2,
                                -0.1025390625), y2, 0.375);
  // x = n π/2 + r, |r| <= π/4
  const double n = rint(x * 0.6366197723675814);
  double r = fma(-n, 1.5707963267341256, x);
  r = fma(-n, 6.077100506303966e-11, r);
  r = fma(-n, 2.0222662487959506e-21, r);
  const double r2 = r * r;
  double sr = fma(fma(fma(fma(fma(fma(fma(2.8114572543455206e-15, r2, -7.647163731819816e-13), r2,
                                          1.6059043836821613e-10), r2, -2.505210838544172e-08), r2,
                                  2.7557319223985893e-06), r2, -0.0001984126984126984), r2, 0.008333333333333333), r2,
                  -0.16666666666666666);
  sr = fma(r * r2, sr, r);
  double cr = fma(fma(fma(fma(fma(fma(fma(fma(-1.5619206968586225e-16, r2, 4.779477332387385e-14), r2,
                                          -1.1470745597729725e-11), r2, 2.08767569878681e-09), r2,
                                  -2.755731922398589e-07), r2, 2.48015873015873e-05), r2, -0.001388888888888889), r2,
                  0.041666666666666664), r2, -0.5);
  cr = fma(r2, cr, 1.0);
  const int q = (int)((long long)n & 3);
  const double sx = q == 0 ? sr : q == 1 ? cr : q == 2 ? -sr : -cr;
  const double cx = q == 0 ? cr : q == 1 ? -sr : q == 2 ? -cr : sr;
  const double c0 = (cx + sx) * 0.7071067811865476, s0 = (sx - cx) * 0.7071067811865476;
  const double a = 0.7978845608028654 * sqrt(y);
  J0 = a * (p0 * c0 - q0 * s0);
  J1 = a * (p1 * s0 + q1 * c0);
}
// J_0, J_1 as the int8x3 J images take them: the asymptotic pair from x = 25, the library below
__device__ __forceinline__ void j01_real(double x, double& J0, double& J1) {
  if (fabs(x) >= J_ASYM_MIN) {
    j01_large(fabs(x), J0, J1);
    if (x < 0) J1 = -J1;  // J_1 is odd
  } else {
    J0 = j0(x);
    J1 = j1(x);
  }
}

__global__ void k_bessel_j01(const double* __restrict__ x, long n, double* __restrict__ J0, double* __restrict__ J1) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a, b;
  j01_real(x[i], a, b);
  J0[i] = a;
  J1[i] = b;
}
cudaError_t launch_bessel_j01(const double* x, long n, double* J0, double* J1, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_bessel_j01<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x, n, J0, J1);
  return cudaGetLastError();
}

// |J_n(x)| <= j_env(x) = min(1, 0.9 / sqrt(x)) for n = 0, 1, 2 and x >= 0 (the suprema of
// sqrt(x) |J_n(x)| are 0.798, 0.825, 0.868 for n = 0, 1, 2); non-increasing, so j_env(k_min ρ)
// bounds J_n(k ρ) over a node slice whose smallest node is k_min. The J digits of a (radius,
// slice) are fixed point relative to it, so far radii keep their 24 bits.
__device__ __forceinline__ double j_env(double x) { return x > 0.81 ? 0.9 / sqrt(x) : 1.0; }

// the smallest node of every slice: one block of 256 threads per slice (kmin[z])
__device__ __forceinline__ void slice_kmin_body(const double* kr, long K, long kchunk, int z, double* kmin) {
  __shared__ double red[256];
  const long k0 = (long)z * kchunk, k1 = min(K, k0 + kchunk);
  double m = INFINITY;
  for (long k = k0 + threadIdx.x; k < k1; k += blockDim.x) m = fmin(m, kr[k]);
  red[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = fmin(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) kmin[z] = isfinite(red[0]) ? red[0] : 0.0;
}
__global__ void __launch_bounds__(256) k_slice_kmin(const double* kr, long K, long kchunk, double* kmin) {
  slice_kmin_body(kr, K, kchunk, blockIdx.x, kmin);
}
cudaError_t launch_slice_kmin(const double* kr, long K, long kchunk, int nchunk, double* kmin, cudaStream_t s) {
  if (nchunk <= 0) return cudaSuccess;
  k_slice_kmin<<<(unsigned)nchunk, 256, 0, s>>>(kr, K, kchunk, kmin);
  return cudaGetLastError();
}

__device__ __forceinline__ void digits3b(int Y, uint32_t& d0, uint32_t& d1, uint32_t& d2) {
  d2 = (uint32_t)Y & 255u;
  d1 = (uint32_t)((Y + 128) >> 8) & 255u;
  d0 = (uint32_t)((Y + 32896) >> 16) & 255u;
}

__device__ __forceinline__ double col_scale(unsigned long long bits) {
  const double m = __longlong_as_double((long long)bits);
  return (m > 0.0 && isfinite(m)) ? BI_SCALE / m : 0.0;
}

// per (slice, column) max |C| as IEEE bits (Inf for a non-finite entry); 256 threads, every
// thread of the block calls it
__device__ __forceinline__ void bcolmax_body(const BesselI8& p, int col, int z) {
  const long k0 = (long)z * p.kchunk, k1 = min(p.K, k0 + p.kchunk);
  const float* c = p.C + (long)col * p.K;
  double m = 0.0;
  for (long k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    const double v = c[k];
    m = isfinite(v) ? fmax(m, fabs(v)) : __longlong_as_double(0x7ff0000000000000LL);
  }
  __shared__ double red[256];
  red[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) p.colmax[(long)z * p.N + col] = (unsigned long long)__double_as_longlong(red[0]);
}
__global__ void __launch_bounds__(256) k_bcolmax(BesselI8 p) { bcolmax_body(p, blockIdx.x, blockIdx.y); }

// one thread per (column tile, row slot, slice, 16-node group): 16 bytes of each digit plane
// one thread per 4 consecutive nodes of a column slot (one 32-bit word of each digit plane):
// adjacent threads read adjacent 32-byte runs of C
__device__ __forceinline__ void bimg_real_body(const BesselI8& p, long t) {
  const long words = p.kchunk / 4;
  const long total = (long)p.ntile_n * p.Np * p.nchunk * words;
  if (t >= total) return;
  const long wq = t % words;
  long rest = t / words;
  const int z = (int)(rest % p.nchunk);
  rest /= p.nchunk;
  const int slot = (int)(rest % p.Np);
  const int ct = (int)(rest / p.Np);
  const int col = ct * p.ctile + slot;
  const bool cv = slot < p.ctile && col < p.N;
  const double sB = cv ? col_scale(p.colmax[(long)z * p.N + col]) : 0.0;
  const long g = wq / 4;
  const int q = (int)(wq % 4);
  uint32_t b[3][4];
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const long k = (long)z * p.kchunk + 16 * g + 4 * q + h;
    const double v = (cv && k < p.K) ? (double)p.C[(long)col * p.K + k] : 0.0;
    uint32_t d0, d1, d2;
    digits3b(__double2int_rn(v * sB), d0, d1, d2);
    b[0][h] = d0; b[1][h] = d1; b[2][h] = d2;
  }
  const long nstage = p.kchunk / BI_NODES;
  const int s = (int)(g / 4), kb = (int)(g % 4) * 16;
  const size_t sbytes = 3ul * (size_t)p.Np * 64;
  uint8_t* blk = p.Bimg + (((size_t)ct * p.nchunk + z) * nstage + s) * sbytes;
#pragma unroll
  for (int pl = 0; pl < 3; ++pl)
    *reinterpret_cast<uint32_t*>(blk + (size_t)pl * p.Np * 64 + plane_off(slot, kb) + 4 * q) =
        b[pl][0] | (b[pl][1] << 8) | (b[pl][2] << 16) | (b[pl][3] << 24);
}
__global__ void k_bimg_real(BesselI8 p) { bimg_real_body(p, (long)blockIdx.x * blockDim.x + threadIdx.x); }

// the same digit images with the (slice, column) maxima taken in the same kernel: one block of
// 256 threads per (column tile, 8-slot row group, node slice). Thread (j, r8) = (tid >> 3,
// tid & 7) takes column slot 8 rg + r8 and the slice's 16-node groups j, j + 32, ...: a first
// pass reduces max |C| (IEEE bits into colmax, as k_bcolmax: a non-finite entry counts as Inf),
// a second pass reads the same bytes again (from L2) and writes the digits. Each thread reads
// 64 consecutive bytes of its column per group; a warp (four groups x eight slots) writes each
// digit plane's 512-byte block of a stage whole. Blocks: ntile_n x (Np / 8) x nchunk.
// 16 entries c[k0 .. k0 + 15] (k0 a multiple of 16, c's rows on 16 bytes), zero at k >= K: four
// 16-byte loads when the group lies wholly below K
__device__ __forceinline__ void load16(const float* c, long k0, long K, float v[16]) {
  if (k0 + 16 <= K) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 f = __ldg(reinterpret_cast<const float4*>(c + k0) + q);
      v[4 * q] = f.x; v[4 * q + 1] = f.y; v[4 * q + 2] = f.z; v[4 * q + 3] = f.w;
    }
  } else {
#pragma unroll
    for (int h = 0; h < 16; ++h) v[h] = k0 + h < K ? c[k0 + h] : 0.0f;
  }
}

__device__ __forceinline__ void bimg_slice_body(const BesselI8& p, long b) {
  __shared__ float wmax[8][8];
  const int tid = threadIdx.x, r8 = tid & 7, j = tid >> 3;
  const int rgroups = p.Np / 8;
  const int rg = (int)(b % rgroups);
  const long rest = b / rgroups;
  const int z = (int)(rest % p.nchunk);
  const int ct = (int)(rest / p.nchunk);
  const int slot = rg * 8 + r8;
  const int col = ct * p.ctile + slot;
  const bool cv = slot < p.ctile && col < p.N;
  const float* c = p.C + (long)(cv ? col : 0) * p.ldc;
  const long kbase = (long)z * p.kchunk;
  const int groups = (int)(p.kchunk / 16);
  float m = 0.0f;
  for (int g = j; g < groups; g += 32) {
    float v[16];
    load16(c, kbase + 16L * g, cv ? p.K : 0, v);
#pragma unroll
    for (int h = 0; h < 16; ++h) m = isfinite(v[h]) ? fmaxf(m, fabsf(v[h])) : __int_as_float(0x7f800000);
  }
  // lanes 8 apart share a slot: reduce over them, then over the block's eight warps
  m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 8));
  m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 16));
  if ((tid & 31) < 8) wmax[tid >> 5][r8] = m;
  __syncthreads();
  float mm = wmax[0][r8];
#pragma unroll
  for (int w = 1; w < 8; ++w) mm = fmaxf(mm, wmax[w][r8]);
  const unsigned long long bits = (unsigned long long)__double_as_longlong((double)mm);
  if (j == 0 && cv) p.colmax[(long)z * p.N + col] = bits;
  const double sB = cv ? col_scale(bits) : 0.0;
  const long nstage = p.kchunk / BI_NODES;
  const size_t sbytes = 3ul * (size_t)p.Np * 64;
  uint8_t* base = p.Bimg + ((size_t)ct * p.nchunk + z) * nstage * sbytes;
  for (int g = j; g < groups; g += 32) {
    float v16[16];
    load16(c, kbase + 16L * g, cv ? p.K : 0, v16);
    uint32_t w[3][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t b0 = 0, b1 = 0, b2 = 0;
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const double v = (double)v16[4 * q + h];
        uint32_t d0, d1, d2;
        digits3b(__double2int_rn(v * sB), d0, d1, d2);
        b0 |= d0 << (8 * h);
        b1 |= d1 << (8 * h);
        b2 |= d2 << (8 * h);
      }
      w[0][q] = b0; w[1][q] = b1; w[2][q] = b2;
    }
    uint8_t* blk = base + (size_t)(g / 4) * sbytes;
#pragma unroll
    for (int pl = 0; pl < 3; ++pl)
      *reinterpret_cast<uint4*>(blk + (size_t)pl * p.Np * 64 + plane_off(slot, (g % 4) * 16)) =
          make_uint4(w[pl][0], w[pl][1], w[pl][2], w[pl][3]);
  }
}

// one thread per (radius tile, row, slice, 16-node group): J_n(k ρ) straight into digits
__global__ void k_aimg_bessel(BesselI8 p) {
  const long groups = p.kchunk / 16;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = (long)p.ntile_m * BI_M * p.nchunk * groups;
  if (t >= total) return;
  const long g = t % groups;
  long rest = t / groups;
  const int z = (int)(rest % p.nchunk);
  rest /= p.nchunk;
  const int row = (int)(rest % BI_M);
  const int mt = (int)(rest / BI_M);
  const int r = mt * BI_M + row;
  const bool rv = r < p.M;
  const double rho = rv ? p.rho[r] : 0.0;
  const double sA = BI_SCALE / j_env(p.kmin[z] * rho);
  uint32_t w[3][4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t b[3][4];
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const long k = (long)z * p.kchunk + 16 * g + 4 * q + h;
      const double v = (rv && k < p.K) ? bessel_j012(p.order, p.kr[k] * rho) : 0.0;
      uint32_t d0, d1, d2;
      digits3b(__double2int_rn(v * sA), d0, d1, d2);
      b[0][h] = d0; b[1][h] = d1; b[2][h] = d2;
    }
#pragma unroll
    for (int pl = 0; pl < 3; ++pl) w[pl][q] = b[pl][0] | (b[pl][1] << 8) | (b[pl][2] << 16) | (b[pl][3] << 24);
  }
  const long nstage = p.kchunk / BI_NODES;
  const int s = (int)(g / 4), kb = (int)(g % 4) * 16;
  const size_t sbytes = 3ul * BI_M * 64;
  uint8_t* blk = p.Aimg + (((size_t)mt * p.nchunk + z) * nstage + s) * sbytes;
#pragma unroll
  for (int pl = 0; pl < 3; ++pl)
    *reinterpret_cast<uint4*>(blk + (size_t)pl * BI_M * 64 + plane_off(row, kb)) =
        make_uint4(w[pl][0], w[pl][1], w[pl][2], w[pl][3]);
}

// k_aimg_bessel for all three orders at once: J_0 and J_1 once per (ρ, k), J_2 from them
// (series below |x| = 1, recurrence above, as bessel_j012), three images in the same layout.
// One thread per 4 consecutive nodes of a radius (one 32-bit word of each digit plane): the
// FP64 Bessel chains are latency-bound, so short chains and many threads.
__device__ __forceinline__ void aimg_bessel3_body(const BesselI8& p, long t, uint8_t* __restrict__ A0,
                                                  uint8_t* __restrict__ A1, uint8_t* __restrict__ A2) {
  const long words = p.kchunk / 4;
  const long total = (long)p.ntile_m * BI_M * p.nchunk * words;
  if (t >= total) return;
  const long wq = t % words;
  long rest = t / words;
  const int z = (int)(rest % p.nchunk);
  rest /= p.nchunk;
  const int row = (int)(rest % BI_M);
  const int mt = (int)(rest / BI_M);
  const int r = mt * BI_M + row;
  const bool rv = r < p.M;
  const double rho = rv ? p.rho[r] : 0.0;
  const double sA = BI_SCALE / j_env(p.kmin[z] * rho);
  const long g = wq / 4;
  const int q = (int)(wq % 4);
  uint32_t b[3][3][4];  // [order][plane][node]
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const long k = (long)z * p.kchunk + 16 * g + 4 * q + h;
    double v[3] = {0.0, 0.0, 0.0};
    if (rv && k < p.K) {
      const double x = p.kr[k] * rho;
      j01_real(x, v[0], v[1]);
      v[2] = j2_from(x, v[0], v[1]);
    }
#pragma unroll
    for (int o = 0; o < 3; ++o) {
      uint32_t d0, d1, d2;
      digits3b(__double2int_rn(v[o] * sA), d0, d1, d2);
      b[o][0][h] = d0; b[o][1][h] = d1; b[o][2][h] = d2;
    }
  }
  const long nstage = p.kchunk / BI_NODES;
  const int s = (int)(g / 4), kb = (int)(g % 4) * 16;
  const size_t sbytes = 3ul * BI_M * 64;
  const size_t off = (((size_t)mt * p.nchunk + z) * nstage + s) * sbytes;
  uint8_t* out[3] = {A0 + off, A1 + off, A2 + off};
#pragma unroll
  for (int o = 0; o < 3; ++o)
#pragma unroll
    for (int pl = 0; pl < 3; ++pl)
      *reinterpret_cast<uint32_t*>(out[o] + (size_t)pl * BI_M * 64 + plane_off(row, kb) + 4 * q) =
          b[o][pl][0] | (b[o][pl][1] << 8) | (b[o][pl][2] << 16) | (b[o][pl][3] << 24);
}
__global__ void __launch_bounds__(256) k_aimg_bessel3(BesselI8 p, uint8_t* __restrict__ A0, uint8_t* __restrict__ A1,
                                                       uint8_t* __restrict__ A2) {
  aimg_bessel3_body(p, (long)blockIdx.x * blockDim.x + threadIdx.x, A0, A1, A2);
}

cudaError_t launch_bessel_i8_aimg3(const BesselI8& p, uint8_t* A0, uint8_t* A1, uint8_t* A2, cudaStream_t s) {
  if (p.M <= 0 || p.K <= 0) return cudaSuccess;
  const long total = (long)p.ntile_m * BI_M * p.nchunk * (p.kchunk / 4);
  k_aimg_bessel3<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(p, A0, A1, A2);
  return cudaGetLastError();
}

struct BiShared {
  uint64_t full[BI_STAGES], empty[BI_STAGES], done;
  uint32_t tmem;
  int abort_flag;
};

__device__ __forceinline__ bool bi_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, unsigned* err,
                                        long limit) {
  for (long it = 0; it < limit; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 255) == 255 && *abort_flag) return false;
  }
  *abort_flag = 1;
  atomicOr(err, 1u);
  return false;
}
__device__ __forceinline__ void bi_drain_wait(uint32_t bar, uint32_t parity) {
  for (long it = 0; it < BI_WAIT_LIMIT; ++it)
    if (mbar_try(bar, parity)) return;
}

// one CTA's (radius tile mt, column tile ct, node slice z) contraction; every thread calls it
__device__ __forceinline__ void gemm_i8_img_body(const BesselI8& p, int mt, int ct, int z, uint8_t* smem) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int c0 = ct * p.ctile;
  const int nct = min(p.ctile, p.N - c0);
  const long k0 = (long)z * p.kchunk, k1 = min(p.K, k0 + p.kchunk);
  const int nst = k1 > k0 ? (int)((k1 - k0 + BI_NODES - 1) / BI_NODES) : 0;
  const long nstage_chunk = p.kchunk / BI_NODES;
  const uint32_t planeA = BI_M * 64u, planeB = (uint32_t)p.Np * 64u;
  const uint32_t stageA = 3u * planeA, stageB = 3u * planeB;
  uint8_t* smA = smem;
  uint8_t* smB = smem + BI_STAGES * stageA;
  BiShared* sh = reinterpret_cast<BiShared*>(smB + BI_STAGES * stageB);
  volatile int* abort_flag = &sh->abort_flag;
  if (tid == 0) {
    for (int s = 0; s < BI_STAGES; ++s) {
      mbar_init(smem_u32(&sh->full[s]), 1);
      mbar_init(smem_u32(&sh->empty[s]), 1);
    }
    mbar_init(smem_u32(&sh->done), 1);
    sh->abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem)),
                 "r"(BI_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem;

  if (warp == 0) {
    if (lane == 0) {
      const uint8_t* gA = p.Aimg + ((size_t)mt * p.nchunk + z) * nstage_chunk * stageA;
      const uint8_t* gB = p.Bimg + ((size_t)ct * p.nchunk + z) * nstage_chunk * stageB;
      int issued = 0;
      for (int s = 0; s < nst; ++s) {
        const int slot = s % BI_STAGES;
        if (s >= BI_STAGES && !bi_wait(smem_u32(&sh->empty[slot]), ((s / BI_STAGES) - 1) & 1, abort_flag, p.err, p.wait_limit))
          break;
        const uint32_t bar = smem_u32(&sh->full[slot]);
        mbar_arrive_tx(bar, stageA + stageB);
        bulk_g2s(smem_u32(smA + slot * stageA), gA + (size_t)s * stageA, stageA, bar);
        bulk_g2s(smem_u32(smB + slot * stageB), gB + (size_t)s * stageB, stageB, bar);
        issued = s + 1;
      }
      for (int s = max(0, issued - BI_STAGES); s < issued; ++s)
        bi_drain_wait(smem_u32(&sh->full[s % BI_STAGES]), (s / BI_STAGES) & 1);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc =
          (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(p.Np >> 3) << 17) | ((uint32_t)(BI_M >> 4) << 24);
      const int pa[6] = {0, 0, 1, 0, 1, 2}, pb[6] = {0, 1, 0, 2, 1, 0};
      for (int s = 0; s < nst; ++s) {
        const int slot = s % BI_STAGES;
        if (!bi_wait(smem_u32(&sh->full[slot]), (s / BI_STAGES) & 1, abort_flag, p.err, p.wait_limit)) break;
        tc_fence_after();
        const uint32_t a0 = smem_u32(smA + slot * stageA), b0 = smem_u32(smB + slot * stageB);
#pragma unroll
        for (int t = 0; t < 2; ++t)
#pragma unroll
          for (int pr = 0; pr < 6; ++pr) {
            const uint64_t ad = umma_desc(a0 + pa[pr] * planeA + t * 256u);
            const uint64_t bd = umma_desc(b0 + pb[pr] * planeB + t * 256u);
            const bool first = s == 0 && t == 0 && (pr == 0 || pr == 1 || pr == 3);
            asm volatile(
                "{\n\t.reg .pred PD;\n\t"
                "setp.ne.b32 PD, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, PD;\n\t}" ::"r"(
                    tmem + (uint32_t)((pa[pr] + pb[pr]) * BI_ACC_STRIDE)),
                "l"(ad), "l"(bd), "r"(idesc), "r"(first ? 0u : 1u)
                : "memory");
          }
        tc_commit(smem_u32(&sh->empty[slot]));
      }
      tc_commit(smem_u32(&sh->done));
      if (*abort_flag) bi_drain_wait(smem_u32(&sh->done), 0);
    }
  } else {
    // epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. +31 (rows of the radius tile)
    bool ok = bi_wait(smem_u32(&sh->done), 0, abort_flag, p.err, p.wait_limit);
    ok = __all_sync(0xffffffffu, ok) && !*abort_flag;
    if (ok && nst > 0) {
      tc_fence_after();
      const int q = warp & 3;
      const uint32_t lanebase = (uint32_t)(32 * q) << 16;
      const int r = mt * BI_M + 32 * q + lane;
      const double eA = r >= p.M ? 1.0 : p.rowscale ? p.rowscale[(long)z * p.M + r]
                                                     : j_env(p.kmin[z] * p.rho[r]);  // the row's J digit scale
      double* out = p.partial + (long)z * p.N * p.M;
      const unsigned long long* cmax = p.colmax + (long)z * p.N;
      for (int e0 = 0; e0 < p.Np; e0 += 8) {
        uint32_t v0[8], v1[8], v2[8];
        tmem_ld8(tmem + lanebase + e0, v0);
        tmem_ld8(tmem + lanebase + BI_ACC_STRIDE + e0, v1);
        tmem_ld8(tmem + lanebase + 2 * BI_ACC_STRIDE + e0, v2);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int cl = e0 + e;
          if (cl < nct && r < p.M) {
            const long long v = (long long)(int)v0[e] * 65536 + (long long)(int)v1[e] * 256 + (long long)(int)v2[e];
            const unsigned long long bits = cmax[c0 + cl];
            const double m = __longlong_as_double((long long)bits);
            double f;
            if (!isfinite(m)) f = __longlong_as_double(0x7ff8000000000000LL);
            else f = m > 0.0 ? 65536.0 / (BI_SCALE * col_scale(bits)) : 0.0;
            out[(long)(c0 + cl) * p.M + r] = (double)v * f * eA;
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    // after a timeout the epilogue may have stopped waiting for `done` while MMAs still run:
    // the MMA thread has committed `done` (it is past its loop), so wait for it before the
    // tensor memory is released
    if (*abort_flag && lane == 0) bi_drain_wait(smem_u32(&sh->done), 0);
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BI_TMEM_COLS) : "memory");
  }
}
__global__ void __launch_bounds__(BI_THREADS, 1) k_gemm_i8_img(BesselI8 p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  gemm_i8_img_body(p, blockIdx.x, blockIdx.y, blockIdx.z, smem);
}

// P[r][c] = Σ_z partial[z][c][r] through a 32 x 32 shared-memory transpose
__global__ void k_reduce_transpose(int M, int N, int nz, const double* __restrict__ part, double* __restrict__ P) {
  __shared__ double tile[32][33];
  const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + j, r = r0 + threadIdx.x;
    double s = 0.0;
    if (c < N && r < M)
      for (int z = 0; z < nz; ++z) s += part[((long)z * N + c) * M + r];
    tile[j][threadIdx.x] = s;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = r0 + j, c = c0 + threadIdx.x;
    if (r < M && c < N) P[(long)r * N + c] = tile[threadIdx.x][j];
  }
}

// per (order, slice, radius): max(|Re J|, |Im J|) over the slice's nodes (1 where it is 0)
__global__ void __launch_bounds__(256) k_jtab_max(BesselI8 p, const double* __restrict__ J, double* __restrict__ rs) {
  const int z = blockIdx.x, r = blockIdx.y, o = blockIdx.z;
  const long plane = (long)p.M * p.K;
  const double* re = J + (2L * o) * plane + (long)r * p.K;
  const double* im = re + plane;
  const long k0 = (long)z * p.kchunk, k1 = min(p.K, k0 + p.kchunk);
  double m = 0.0;
  for (long k = k0 + threadIdx.x; k < k1; k += blockDim.x) m = fmax(m, fmax(fabs(re[k]), fabs(im[k])));
  __shared__ double red[256];
  red[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) rs[((long)o * p.nchunk + z) * p.M + r] = red[0] > 0.0 && isfinite(red[0]) ? red[0] : 1.0;
}

// one thread per (image, radius tile, row, slice, 4-node word): the digits of Re or Im J_o
// relative to the row's slice maximum, written as one 32-bit word of each digit plane
struct Img6 {
  uint8_t* p[6];
};
__global__ void __launch_bounds__(256) k_jtab_img(BesselI8 p, const double* __restrict__ J,
                                                  const double* __restrict__ rs, Img6 img) {
  const long words = p.kchunk / 4;
  const long per = (long)p.ntile_m * BI_M * p.nchunk * words;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 6 * per) return;
  const int im = (int)(t / per);  // 2 o + part
  long u = t % per;
  const long wq = u % words;
  u /= words;
  const int z = (int)(u % p.nchunk);
  u /= p.nchunk;
  const int row = (int)(u % BI_M);
  const int mt = (int)(u / BI_M);
  const int r = mt * BI_M + row;
  const bool rv = r < p.M;
  const int o = im / 2;
  const double sA = rv ? BI_SCALE / rs[((long)o * p.nchunk + z) * p.M + r] : 0.0;
  const double* tab = J + (long)im * p.M * p.K + (long)(rv ? r : 0) * p.K;
  const long g = wq / 4;
  const int q = (int)(wq % 4);
  uint32_t w[3] = {0u, 0u, 0u};
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const long k = (long)z * p.kchunk + 16 * g + 4 * q + h;
    const double v = (rv && k < p.K) ? tab[k] : 0.0;
    uint32_t d0, d1, d2;
    digits3b(__double2int_rn(v * sA), d0, d1, d2);
    w[0] |= d0 << (8 * h);
    w[1] |= d1 << (8 * h);
    w[2] |= d2 << (8 * h);
  }
  const long nstage = p.kchunk / BI_NODES;
  const int s = (int)(g / 4), kb = (int)(g % 4) * 16;
  const size_t sbytes = 3ul * BI_M * 64;
  uint8_t* blk = img.p[im] + (((size_t)mt * p.nchunk + z) * nstage + s) * sbytes;
#pragma unroll
  for (int pl = 0; pl < 3; ++pl)
    *reinterpret_cast<uint32_t*>(blk + (size_t)pl * BI_M * 64 + plane_off(row, kb) + 4 * q) = w[pl];
}

cudaError_t launch_jtable_images(const BesselI8& bp, const double* Jtab, double* rowscale, uint8_t* const img[6],
                                 cudaStream_t s) {
  if (bp.M <= 0 || bp.K <= 0) return cudaSuccess;
  k_jtab_max<<<dim3((unsigned)bp.nchunk, (unsigned)bp.M, 3), 256, 0, s>>>(bp, Jtab, rowscale);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long tot = 6L * bp.ntile_m * BI_M * bp.nchunk * (bp.kchunk / 4);
  Img6 im6;
  for (int i = 0; i < 6; ++i) im6.p[i] = img[i];
  k_jtab_img<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(bp, Jtab, rowscale, im6);
  return cudaGetLastError();
}

cudaError_t launch_bessel_i8(const BesselI8& p, double* P, cudaStream_t s) {
  if (p.M <= 0 || p.N <= 0 || p.K <= 0) return cudaSuccess;
  if ((!p.kmin && !p.rowscale) || p.kchunk % BI_NODES != 0 || p.kchunk > 16384 || p.Np % 16 != 0 || p.Np > BI_ACC_STRIDE || p.Np < p.ctile ||
      (long)p.nchunk * p.kchunk < p.K)
    return cudaErrorInvalidValue;
  cudaError_t e;
  k_bcolmax<<<dim3((unsigned)p.N, (unsigned)p.nchunk), 256, 0, s>>>(p);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  {
    const long total = (long)p.ntile_n * p.Np * p.nchunk * (p.kchunk / 4);
    k_bimg_real<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(p);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (!p.aimg_ready) {
    const long total = (long)p.ntile_m * BI_M * p.nchunk * (p.kchunk / 16);
    k_aimg_bessel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(p);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  const size_t sm = bessel_i8_smem(p.Np);
  if ((e = cudaFuncSetAttribute(k_gemm_i8_img, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)) != cudaSuccess)
    return e;
  k_gemm_i8_img<<<dim3((unsigned)p.ntile_m, (unsigned)p.ntile_n, (unsigned)p.nchunk), BI_THREADS, sm, s>>>(p);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_reduce_transpose<<<dim3((unsigned)((p.M + 31) / 32), (unsigned)((p.N + 31) / 32)), dim3(32, 8), 0, s>>>(
      p.M, p.N, p.nchunk, p.partial, P);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// Grouped launches: every (item, order) entry of a group in one grid per stage. Entry
// e = 3 i + o holds item i's order-o parameters; its J_n images share item i's node slicing
// (bp[3 i] gives the layout), so one Bessel evaluation per (ρ, k) serves the three orders.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_aimg_bessel3_group(const BesselI8* __restrict__ bp, const long* __restrict__ first,
                                                          int ni) {
  const int i = group_entry(first, ni, blockIdx.x);
  const BesselI8& p = bp[3 * i];
  aimg_bessel3_body(p, (long)(blockIdx.x - first[i]) * blockDim.x + threadIdx.x, bp[3 * i].Aimg, bp[3 * i + 1].Aimg,
                    bp[3 * i + 2].Aimg);
}

// nchunk blocks per item: the slices' smallest nodes (bp[3 i].kmin, shared by the orders)
__global__ void __launch_bounds__(256) k_slice_kmin_group(const BesselI8* __restrict__ bp,
                                                        const long* __restrict__ first, int ni) {
  const int i = group_entry(first, ni, blockIdx.x);
  const BesselI8& p = bp[3 * i];
  slice_kmin_body(p.kr, p.K, p.kchunk, (int)(blockIdx.x - first[i]), p.kmin);
}

// ntile_n x (Np / 8) x nchunk blocks per entry (bimg_slice_body)
__global__ void __launch_bounds__(256) k_bimg_real_group(const BesselI8* __restrict__ bp, const long* __restrict__ first,
                                                       int ne) {
  const int e = group_entry(first, ne, blockIdx.x);
  bimg_slice_body(bp[e], blockIdx.x - first[e]);
}

// ntile_m x ntile_n x nchunk CTAs per entry, radius tile fastest (the CTAs that share a
// column tile's B images run side by side)
__global__ void __launch_bounds__(BI_THREADS, 1) k_gemm_i8_img_group(const BesselI8* __restrict__ bp,
                                                                     const long* __restrict__ first, int ne) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int e = group_entry(first, ne, blockIdx.x);
  const BesselI8& p = bp[e];
  const long b = blockIdx.x - first[e];
  const int mt = (int)(b % p.ntile_m);
  const long rest = b / p.ntile_m;
  gemm_i8_img_body(p, mt, (int)(rest % p.ntile_n), (int)(rest / p.ntile_n), smem);
}

cudaError_t launch_bessel_i8_group(const Synth1DGroup& g, int stage, cudaStream_t s) {
  if (g.ni <= 0) return cudaSuccess;
  const int ne = 3 * g.ni;
  cudaError_t e;
  if (stage == 0 && g.grid[6] > 0) {
    k_slice_kmin_group<<<(unsigned)g.grid[6], 256, 0, s>>>(g.bp, g.first_kmin, g.ni);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (stage == 0 && g.grid[2] > 0) {
    k_aimg_bessel3_group<<<(unsigned)g.grid[2], 256, 0, s>>>(g.bp, g.first_aimg, g.ni);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (stage == 1 && g.grid[3] > 0) {
    k_bimg_real_group<<<(unsigned)g.grid[3], 256, 0, s>>>(g.bp, g.first_bimg, ne);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (stage == 2 && g.grid[4] > 0) {
    const size_t sm = bessel_i8_smem(BI_ACC_STRIDE);
    if ((e = cudaFuncSetAttribute(k_gemm_i8_img_group, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm)) !=
        cudaSuccess)
      return e;
    k_gemm_i8_img_group<<<(unsigned)g.grid[4], BI_THREADS, sm, s>>>(g.bp, g.first_gemm, ne);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace ytf

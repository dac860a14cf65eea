// ytf_lateral_i8.cu -- the 2D lateral synthesis on the int8 tensor cores (tcgen05 kind::i8).
//
// G[pix, col] = Σ_n e^{i(kx_n x_i + ky_n y_j)} S[col, n]   (closed_form_G, lateral=:direct,
// mod_ClosedFormField.jl:743-753) as one real GEMM per tile, as in the split-BF16 kernel:
//   A'[pix, 2n + {0,1}] = (Re P, Im P),  P = Px[n, i] · Py[n, j]
//   B'[(col, re), 2n + {0,1}] = (Sr, -Si),  B'[(col, im), 2n + {0,1}] = (Si, Sr)
// but in fixed point: A' as X = rint(sA · a) with sA = 4194000 (|P| = 1, so |X| < 2^22: the
// range of the magic-number rounding below), and B' per (column, node slice) as
// Y = rint(sB · b) with sB = 8355000 / max|S| over the slice (|Y| ≤ 8355000 < 2^23).
// X and Y are written in three signed base-256 digits (X = 65536 d0 + 256 d1 + d2, top digit
// in [-64, 64] for X and [-127, 127] for Y, d1, d2 in [-128, 127]) and the six digit products
// of weight ≥ 256^2 are summed exactly by the tensor cores in INT32: level L = i + j in
// tensor-memory accumulator L. The dropped products (weight ≤ 256) are ~2^-23 of the leading
// one and dominate the error (a fourth accumulator would not fit: 4 x 144 columns > 512).
// Integer accumulation is exact, so the result depends on no accumulation order; the only
// roundings are the FP32 phase product, the two fixed-point quantisations and the FP64
// combination at the end:
//   X·Y / 2^16 = 65536 acc0 + 256 acc1 + acc2,   G = that · 2^16 / (sA · sB).
// Overflow: per real term |level-2 product sum| ≤ 64·128 + 128·128 + 128·127 = 40832; the
// host keeps each CTA's node slice ≤ 16384 nodes (K ≤ 32768 real terms), so |acc| < 1.4e9.
//
// Kernels:
//   (k_strengths2d reduces max|S| per (node slice, column) while it writes S)
//   k_bslice : B' digits, written once per launch in the exact shared-memory image of each
//              32-node stage (3 planes x Np rows x 64 B, canonical K-major core matrices)
//   k_lateral_i8 : one CTA per (128-pixel tile, column tile, node slice); 8 producer warps
//              build A' digits from the FP32 phase tables (zero-padded to the slice grid)
//              into a 4-deep ring, warp 8 copies
//              each stage's B' image with one bulk copy, one thread of warp 9 issues the
//              12 MMAs of a stage (6 digit products x 2 K-halves, M=128, N=Np, K=32) and
//              commits them to the stage's "empty" barrier. At the end all 8 producer warps
//              read the three INT32 accumulators and write the FP64 partial sums.
// Every wait is bounded and checks a shared abort flag; a timeout sets the error word, the
// CTA lets its issued copies and MMAs finish (bounded) and frees its tensor memory. No TMA
// tensor maps and no multicast.
#include "ytf_complex.cuh"
#include "ytf_kernels.h"
#include "ytf_tcgen05.cuh"

namespace ytf {

constexpr int I8_M = 128;            // pixels per tile (MMA M)
constexpr int I8_NODES = 32;         // nodes per stage (real K = 64 bytes per row)
constexpr int I8_STAGES = 4;         // ring depth
constexpr int I8_PRODUCERS = 256;    // warps 0-7
constexpr int I8_THREADS = 320;      // + warp 8 (bulk copies) + warp 9 (MMA issue)
constexpr int I8_ACC_STRIDE = 160;   // tensor-memory columns per accumulator (max N)
constexpr int I8_TMEM_COLS = 512;
constexpr long I8_WAIT_LIMIT = 1L << 22;  // polls of the drain waits (the pipeline waits: p.wait_limit)
constexpr float I8_SA = 4194000.0f;      // fixed-point scale of the phase operand
constexpr float I8_MAGIC = 12582912.0f;  // 1.5 * 2^23: fl(t + MAGIC) has rint(t) in its low 23 bits

size_t lateral_i8_stage_bytes(int Np) { return 3ul * (size_t)Np * 64; }

size_t lateral_i8_smem(int Np) {
  return (size_t)I8_STAGES * (3ul * I8_M * 64 + lateral_i8_stage_bytes(Np)) + 128;
}

// balanced column tiles of at most 80 complex columns (MMA N ≤ 160, three accumulators)
int lateral_i8_ctile(int ncol) {
  int ntiles = (ncol + 79) / 80;
  return (ncol + ntiles - 1) / ntiles;
}

// ------------------------------------------------------------------------------------
// FP32 phase tables Px[n][i] = e^{i kx_n x_i}, Py[n][j] = e^{i ky_n y_j}, zero for the padding
// nodes n <= node < n_pad. The arguments are formed and reduced to [-π, π] in FP64 (2π as a
// double plus its remainder; the FMAs subtract k·2π with one rounding each, so the reduced
// argument is good to a few FP64 ulp of the argument), then FP32 sincosf of the reduced
// argument: the FP32 values the int8 digits are made from, within ~1 FP32 ulp. The block's
// nodes get their cos φ, sin φ once, in shared memory.
// ------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_phase_tables_pad(CacheView c, int nx, int ny, const double* xs,
                                                          const double* ys, long n_pad, float2* Px, float2* Py) {
  __shared__ double kxs[256], kys[256];
  const int m = nx + ny;
  const long t0 = (long)blockIdx.x * blockDim.x;
  const long tot = n_pad * (long)m;
  const long nn0 = tot <= 0x7fffffffL ? (long)((unsigned)t0 / (unsigned)m) : t0 / m;
  const long last = min(tot, t0 + (long)blockDim.x) - 1;
  const int nodes = (int)(last / m - nn0 + 1);
  if ((int)threadIdx.x < nodes) {
    const long nn = nn0 + threadIdx.x;
    double kx = 0.0, ky = 0.0;
    if (nn < c.n) {
      const long k = nn % c.Nk, q = nn / c.Nk;
      double s, co;
      sincos(c.phi[q], &s, &co);
      kx = c.kr[k] * co;
      ky = c.kr[k] * s;
    }
    kxs[threadIdx.x] = kx;
    kys[threadIdx.x] = ky;
  }
  __syncthreads();
  const long t = t0 + threadIdx.x;
  if (t >= tot) return;
  // 32-bit division when the table fits (a 64-bit one costs tens of instructions)
  const long nn = tot <= 0x7fffffffL ? (long)((unsigned)t / (unsigned)m) : t / m;
  const int e = (int)(t - nn * m);
  float2 v = make_float2(0.f, 0.f);
  if (nn < c.n) {
    const int b = (int)(nn - nn0);
    const double arg = e < nx ? kxs[b] * xs[e] : kys[b] * ys[e - nx];
    // arg - 2π rint(arg / 2π), 2π = TWO_PI_HI + TWO_PI_LO
    const double TWO_PI_HI = 6.28318530717958623200e+00, TWO_PI_LO = 2.44929359829470635445e-16;
    const double kq = rint(arg * 0.15915494309189533577);
    const double r = fma(-kq, TWO_PI_LO, fma(-kq, TWO_PI_HI, arg));
    float sn, cs;
    sincosf((float)r, &sn, &cs);
    v = make_float2(cs, sn);
  }
  if (e < nx) Px[nn * nx + e] = v;
  else Py[nn * ny + (e - nx)] = v;
}

// The same tables when the pixel coordinates are evenly spaced (x_i = x_0 + i dx, y_j = y_0 +
// j dy): one thread per (node, axis) forms e^{i k x_0} and e^{i k dx} in FP64 and steps along
// the row, e(x + dx) = e(x) e^{i k dx} (unit-modulus factors: a few FP64 ulp after a row of
// 64, far below the FP32 rounding of the stored value); rows go through shared memory so the
// stores are coalesced.
__global__ void __launch_bounds__(128) k_phase_tables_even(CacheView c, int nx, int ny, double x0, double dx, double y0,
                                                           double dy, long n_pad, float2* Px, float2* Py) {
  // 64 nodes per block: threads 0-63 step their node's x row, 64-127 its y row, into shared
  // memory (32 entries of each row per pass), then the block writes them coalesced
  __shared__ float2 rows[2][64][33];
  const long nb0 = (long)blockIdx.x * 64;
  const int tid = threadIdx.x, ax = tid >> 6, r = tid & 63;
  const int cnt = ax ? ny : nx;
  const long nn = nb0 + r;
  double er = 0.0, ei = 0.0, cd_ = 1.0, sd = 0.0;
  if (nn < c.n) {
    const long k = nn % c.Nk, q = nn / c.Nk;
    double sp, cp;
    sincos(c.phi[q], &sp, &cp);
    const double kk = c.kr[k] * (ax ? sp : cp);
    sincos(kk * (ax ? y0 : x0), &ei, &er);
    sincos(kk * (ax ? dy : dx), &sd, &cd_);
  }
  const long nrows = min(64L, n_pad - nb0);
  for (int base = 0; base < max(nx, ny); base += 32) {
    const int m = min(32, cnt - base);
    for (int i = 0; i < m; ++i) {
      rows[ax][r][i] = nn < c.n ? make_float2((float)er, (float)ei) : make_float2(0.f, 0.f);
      const double nr = er * cd_ - ei * sd, ni = er * sd + ei * cd_;
      er = nr;
      ei = ni;
    }
    __syncthreads();
    for (int a = 0; a < 2; ++a) {
      const int ca = a ? ny : nx;
      const int ma = min(32, ca - base);
      if (ma <= 0) continue;
      float2* out = a ? Py : Px;
      for (int e = tid; e < nrows * ma; e += 128) {
        const int rr = e / ma, i = e - rr * ma;
        out[(nb0 + rr) * ca + base + i] = rows[a][rr][i];
      }
    }
    __syncthreads();
  }
}

cudaError_t launch_phase_tables_pad(const CacheView& c, int nx, int ny, const double* xs, const double* ys, long n_pad,
                                    float2* Px, float2* Py, cudaStream_t s, const double* even) {
  long tot = n_pad * (long)(nx + ny);
  if (tot <= 0) return cudaSuccess;
  if (even) {
    k_phase_tables_even<<<(unsigned)((n_pad + 63) / 64), 128, 0, s>>>(c, nx, ny, even[0], even[1], even[2], even[3],
                                                                     n_pad, Px, Py);
    return cudaGetLastError();
  }
  k_phase_tables_pad<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(c, nx, ny, xs, ys, n_pad, Px, Py);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------
// B' preparation
// ------------------------------------------------------------------------------------
// fixed-point scale of one (node slice, column) of strengths from its max(|Re|, |Im|):
// |S sB| ≤ 8355000 (one rounding of the product above it is still below 8355000.5), so the
// top digit (Y + 32896) >> 16 stays in [-127, 127]. 0 for an all-zero column; a non-finite
// maximum poisons the column's output (fac = NaN), as the FP64 contraction would.
__device__ __forceinline__ double slice_scale(unsigned long long bits) {
  const double m = __longlong_as_double((long long)bits);
  return (m > 0.0 && isfinite(m)) ? 8355000.0 / m : 0.0;
}
__device__ __forceinline__ double slice_factor(unsigned long long bits) {
  const double m = __longlong_as_double((long long)bits);
  if (!isfinite(m)) return __longlong_as_double(0x7ff8000000000000LL);
  return m > 0.0 ? 65536.0 / ((double)I8_SA * slice_scale(bits)) : 0.0;
}

// three signed base-256 digits of Y (|Y| ≤ 8355000), most significant first, as bytes
__device__ __forceinline__ void digits3(int Y, uint32_t& d0, uint32_t& d1, uint32_t& d2) {
  d2 = (uint32_t)Y & 255u;
  d1 = (uint32_t)((Y + 128) >> 8) & 255u;
  d0 = (uint32_t)((Y + 32896) >> 16) & 255u;
}

// one thread per (column tile, column slot, node slice, 8-node group): 16 bytes of each of
// the two rows of the column in each of the three digit planes. Grid: x over the slice's
// 8-node groups, y = column slot, z = column tile x node slice (no index division).
__global__ void __launch_bounds__(256) k_bslice(LateralI8 p) {
  const int groups = (int)(p.kchunk / 8);
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= groups) return;
  const int cl = blockIdx.y;
  const int z = (int)(blockIdx.z % (unsigned)p.nchunk), ct = (int)(blockIdx.z / (unsigned)p.nchunk);
  const int col = ct * p.ctile + cl;
  const bool cv = cl < p.ctile && col < p.ncol;
  const long o = (long)z * p.ncol + (cv ? col : 0);
  const double sB = cv ? slice_scale(p.colmax[o]) : 0.0;
  const long nstage = p.kchunk / I8_NODES;
  const int s = (int)(g / 4), kb = (int)(g % 4) * 16;
  uint32_t w[2][3][4];  // [row re/im][plane][word]
#pragma unroll
  for (int q2 = 0; q2 < 4; ++q2) {
    uint32_t b[2][3][4];  // bytes of this word: [row][plane][byte]
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long nn = (long)z * p.kchunk + 8 * g + 2 * q2 + h;
      double2 v = make_double2(0.0, 0.0);
      if (cv && nn < p.n) v = p.S[(long)col * p.n + nn];
      const int yr = __double2int_rn(v.x * sB), yi = __double2int_rn(v.y * sB);
      uint32_t r0, r1, r2, i0, i1, i2, n0, n1, n2;
      digits3(yr, r0, r1, r2);
      digits3(yi, i0, i1, i2);
      digits3(-yi, n0, n1, n2);
      // row 2c: (Sr, -Si); row 2c+1: (Si, Sr)
      b[0][0][2 * h] = r0; b[0][1][2 * h] = r1; b[0][2][2 * h] = r2;
      b[0][0][2 * h + 1] = n0; b[0][1][2 * h + 1] = n1; b[0][2][2 * h + 1] = n2;
      b[1][0][2 * h] = i0; b[1][1][2 * h] = i1; b[1][2][2 * h] = i2;
      b[1][0][2 * h + 1] = r0; b[1][1][2 * h + 1] = r1; b[1][2][2 * h + 1] = r2;
    }
#pragma unroll
    for (int rr = 0; rr < 2; ++rr)
#pragma unroll
      for (int pl = 0; pl < 3; ++pl)
        w[rr][pl][q2] = b[rr][pl][0] | (b[rr][pl][1] << 8) | (b[rr][pl][2] << 16) | (b[rr][pl][3] << 24);
  }
  const size_t sbytes = 3ul * (size_t)p.Np * 64;
  uint8_t* blk = p.Bq + (((size_t)ct * p.nchunk + z) * nstage + s) * sbytes;
#pragma unroll
  for (int rr = 0; rr < 2; ++rr)
#pragma unroll
    for (int pl = 0; pl < 3; ++pl) {
      const int row = 2 * cl + rr;
      *reinterpret_cast<uint4*>(blk + (size_t)pl * p.Np * 64 + plane_off(row, kb)) =
          make_uint4(w[rr][pl][0], w[rr][pl][1], w[rr][pl][2], w[rr][pl][3]);
    }
}

// ------------------------------------------------------------------------------------
// the tensor-core contraction
// ------------------------------------------------------------------------------------
struct I8Shared {
  uint64_t full_a[I8_STAGES], full_b[I8_STAGES], empty[I8_STAGES], done;
  uint32_t tmem;
  int abort_flag;
};

// bounded wait (limit polls); gives up early when another thread of the CTA has already given up
__device__ __forceinline__ bool i8_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, unsigned* err,
                                        long limit) {
  for (long it = 0; it < limit; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 255) == 255 && *abort_flag) return false;
  }
  *abort_flag = 1;
  atomicOr(err, 1u);
  return false;
}
// bounded wait that ignores the abort flag: lets issued copies and MMAs finish
__device__ __forceinline__ void i8_drain_wait(uint32_t bar, uint32_t parity) {
  for (long it = 0; it < I8_WAIT_LIMIT; ++it)
    if (mbar_try(bar, parity)) return;
}

__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred PD;\n\t"
      "setp.ne.b32 PD, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, PD;\n\t}" ::"r"(tmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
      : "memory");
}

// the phase operands of one thread for one stage: 16 nodes of one pixel, from the zero-padded
// phase tables [n_pad][nx], [n_pad][ny] (no bounds checks: a warp's lanes read consecutive
// pixels of one node row, so each load is one or two cache lines)
struct PhaseRegs {
  float2 px[16], py[16];
};

__device__ __forceinline__ void i8_load(const float2* px, const float2* py, long sx, long sy, PhaseRegs& R) {
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    R.px[q] = __ldg(px + q * sx);
    R.py[q] = __ldg(py + q * sy);
  }
}

// fixed-point bits of one phase component: fl(a·sA + MAGIC) = MAGIC + rint(a·sA)
__device__ __forceinline__ uint32_t fx_bits(float a) { return __float_as_uint(fmaf(a, I8_SA, I8_MAGIC)); }

__global__ void __launch_bounds__(I8_THREADS, 1) k_lateral_i8(LateralI8 p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long p0 = (long)blockIdx.x * I8_M;
  const int ct = blockIdx.y;
  const int c0 = ct * p.ctile;
  const int nct = min(p.ctile, p.ncol - c0);
  const int z = blockIdx.z;
  const long k0 = (long)z * p.kchunk;
  const long k1 = min(p.n, k0 + p.kchunk);
  const int nst = k1 > k0 ? (int)((k1 - k0 + I8_NODES - 1) / I8_NODES) : 0;
  const long nstage_chunk = p.kchunk / I8_NODES;
  const uint32_t planeA = I8_M * 64u, planeB = (uint32_t)p.Np * 64u;
  const uint32_t stageA = 3u * planeA, stageB = 3u * planeB;
  uint8_t* smA = smem;
  uint8_t* smB = smem + I8_STAGES * stageA;
  I8Shared* sh = reinterpret_cast<I8Shared*>(smB + I8_STAGES * stageB);
  volatile int* abort_flag = &sh->abort_flag;

  if (tid == 0) {
    for (int s = 0; s < I8_STAGES; ++s) {
      mbar_init(smem_u32(&sh->full_a[s]), I8_PRODUCERS / 32);
      mbar_init(smem_u32(&sh->full_b[s]), 1);
      mbar_init(smem_u32(&sh->empty[s]), 1);
    }
    mbar_init(smem_u32(&sh->done), 1);
    sh->abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem)),
                 "r"(I8_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sh->tmem;

  if (warp < I8_PRODUCERS / 32) {
    // ---------------- producers: A' digits ----------------
    // pixel r of the tile, nodes 16h..16h+15 of each stage; a pixel beyond npix reads pixel 0
    // (its output row is never stored, and each A' row only reaches its own output row)
    const int r = tid & 127, h = tid >> 7;
    const long pix = p0 + r;
    const bool pv = pix < p.npix;
    const int i = pv ? (int)(pix % p.nx) : 0, j = pv ? (int)(pix / p.nx) : 0;
    const long sx = p.nx, sy = p.ny;
    const float2* pxb = p.Px + (k0 + 16 * h) * sx + i;
    const float2* pyb = p.Py + (k0 + 16 * h) * sy + j;
    // one stage from `use` while `pre` receives the next stage's loads; false = give up
    auto stage = [&](int s, PhaseRegs& use, PhaseRegs& pre) -> bool {
      const int slot = s % I8_STAGES;
      if (s + 1 < nst) i8_load(pxb + (s + 1) * I8_NODES * sx, pyb + (s + 1) * I8_NODES * sy, sx, sy, pre);
      bool ok = true;
      if (s >= I8_STAGES) ok = i8_wait(smem_u32(&sh->empty[slot]), ((s / I8_STAGES) - 1) & 1, abort_flag, p.err, p.wait_limit);
      if (!__all_sync(0xffffffffu, ok)) return false;
      uint8_t* A = smA + slot * stageA;
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        uint32_t w0[4], w1[4], w2[4];
#pragma unroll
        for (int wd = 0; wd < 4; ++wd) {
          // word wd of this 16-byte chunk: nodes 2wd, 2wd+1 of the half, (re, im) each
          uint32_t u0[2], u1[2], u2[2];
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const float2 a = use.px[8 * half + 2 * wd + e], b = use.py[8 * half + 2 * wd + e];
            const float re = fmaf(a.x, b.x, -a.y * b.y), im = fmaf(a.x, b.y, a.y * b.x);
            const uint32_t xr = fx_bits(re), xi = fx_bits(im);
            // digit bytes: d2 = byte 0 of X, d1 = byte 1 of X + 128, d0 = byte 2 of X + 32896
            // (the magic's own bits sit above bit 15 except its 0x40 in byte 2, removed here)
            u2[e] = __byte_perm(xr, xi, 0x0040);
            u1[e] = __byte_perm(xr + 128u, xi + 128u, 0x0051);
            u0[e] = __byte_perm(xr + 32896u - 0x400000u, xi + 32896u - 0x400000u, 0x0062);
          }
          w2[wd] = __byte_perm(u2[0], u2[1], 0x5410);
          w1[wd] = __byte_perm(u1[0], u1[1], 0x5410);
          w0[wd] = __byte_perm(u0[0], u0[1], 0x5410);
        }
        const uint32_t off = plane_off(r, 32 * h + 16 * half);
        *reinterpret_cast<uint4*>(A + off) = make_uint4(w0[0], w0[1], w0[2], w0[3]);
        *reinterpret_cast<uint4*>(A + planeA + off) = make_uint4(w1[0], w1[1], w1[2], w1[3]);
        *reinterpret_cast<uint4*>(A + 2 * planeA + off) = make_uint4(w2[0], w2[1], w2[2], w2[3]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&sh->full_a[slot]));
      return true;
    };
    PhaseRegs ra, rb;
    if (nst > 0) i8_load(pxb, pyb, sx, sy, ra);
    for (int s = 0; s < nst; s += 2) {
      if (!stage(s, ra, rb)) break;
      if (s + 1 < nst && !stage(s + 1, rb, ra)) break;
    }
  } else if (warp == 8) {
    // ---------------- bulk copies of the prepared B' stage images ----------------
    if (lane == 0) {
      const uint8_t* gB = p.Bq + ((size_t)ct * p.nchunk + z) * nstage_chunk * stageB;
      int issued = 0;
      for (int s = 0; s < nst; ++s) {
        const int slot = s % I8_STAGES;
        if (s >= I8_STAGES && !i8_wait(smem_u32(&sh->empty[slot]), ((s / I8_STAGES) - 1) & 1, abort_flag, p.err, p.wait_limit))
          break;
        const uint32_t bar = smem_u32(&sh->full_b[slot]);
        mbar_arrive_tx(bar, stageB);
        bulk_g2s(smem_u32(smB + slot * stageB), gB + (size_t)s * stageB, stageB, bar);
        issued = s + 1;
      }
      // every issued copy lands before the CTA can exit
      for (int s = max(0, issued - I8_STAGES); s < issued; ++s)
        i8_drain_wait(smem_u32(&sh->full_b[s % I8_STAGES]), (s / I8_STAGES) & 1);
    }
  } else {
    // ---------------- MMA issue ----------------
    if (lane == 0) {
      // kind::i8: D S32 (bits 4-5 = 2), A and B signed 8-bit (bits 7-9 = 1, 10-12 = 1), both
      // K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
      const uint32_t idesc =
          (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(p.Np >> 3) << 17) | ((uint32_t)(I8_M >> 4) << 24);
      const int pa[6] = {0, 0, 1, 0, 1, 2}, pb[6] = {0, 1, 0, 2, 1, 0};
      for (int s = 0; s < nst; ++s) {
        const int slot = s % I8_STAGES;
        const uint32_t par = (s / I8_STAGES) & 1;
        if (!i8_wait(smem_u32(&sh->full_b[slot]), par, abort_flag, p.err, p.wait_limit)) break;
        if (!i8_wait(smem_u32(&sh->full_a[slot]), par, abort_flag, p.err, p.wait_limit)) break;
        tc_fence_after();
        const uint32_t a0 = smem_u32(smA + slot * stageA), b0 = smem_u32(smB + slot * stageB);
#pragma unroll
        for (int t = 0; t < 2; ++t)
#pragma unroll
          for (int pr = 0; pr < 6; ++pr) {
            const uint64_t ad = umma_desc(a0 + pa[pr] * planeA + t * 256u);
            const uint64_t bd = umma_desc(b0 + pb[pr] * planeB + t * 256u);
            // the first MMA into each level accumulator overwrites it
            const bool first = s == 0 && t == 0 && (pr == 0 || pr == 1 || pr == 3);
            mma_i8(tmem + (uint32_t)((pa[pr] + pb[pr]) * I8_ACC_STRIDE), ad, bd, idesc, first ? 0u : 1u);
          }
        tc_commit(smem_u32(&sh->empty[slot]));
      }
      // all MMAs issued so far (possibly none) complete before `done` arrives
      tc_commit(smem_u32(&sh->done));
      if (*abort_flag) i8_drain_wait(smem_u32(&sh->done), 0);
    }
  }

  // ---------------- epilogue: INT32 accumulators -> FP64 partial sums ----------------
  if (warp < I8_PRODUCERS / 32) {
    bool ok = i8_wait(smem_u32(&sh->done), 0, abort_flag, p.err, p.wait_limit);
    ok = __all_sync(0xffffffffu, ok) && !*abort_flag;
    if (ok && nst > 0) {
      tc_fence_after();
      const int q = warp & 3, hh = warp >> 2, half = p.Np / 2;
      const uint32_t lanebase = (uint32_t)(32 * q) << 16;
      const long pix = p0 + 32 * q + lane;
      double2* out = p.partial + (long)z * p.npix * p.ncol;
      const unsigned long long* cmax = p.colmax + (long)z * p.ncol;
      for (int e0 = 0; e0 < half; e0 += 8) {
        uint32_t v0[8], v1[8], v2[8];
        const uint32_t col = (uint32_t)(hh * half + e0);
        tmem_ld8(tmem + lanebase + col, v0);
        tmem_ld8(tmem + lanebase + I8_ACC_STRIDE + col, v1);
        tmem_ld8(tmem + lanebase + 2 * I8_ACC_STRIDE + col, v2);
        tmem_wait_ld();
#pragma unroll
        for (int e = 0; e < 8; e += 2) {
          const int cc = (int)(col + e) / 2;
          if (cc < nct && pix < p.npix) {
            const long long re =
                (long long)(int)v0[e] * 65536 + (long long)(int)v1[e] * 256 + (long long)(int)v2[e];
            const long long im =
                (long long)(int)v0[e + 1] * 65536 + (long long)(int)v1[e + 1] * 256 + (long long)(int)v2[e + 1];
            const double f = slice_factor(cmax[c0 + cc]);
            out[pix + p.npix * (long)(c0 + cc)] = make_double2((double)re * f, (double)im * f);
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
    if (*abort_flag && lane == 0) i8_drain_wait(smem_u32(&sh->done), 0);
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(I8_TMEM_COLS) : "memory");
  }
}

cudaError_t launch_lateral_i8(const LateralI8& p, cudaStream_t s) {
  if (p.npix <= 0 || p.ncol <= 0 || p.n <= 0) return cudaSuccess;
  if (p.kchunk % I8_NODES != 0 || p.kchunk > 16384 || p.Np % 16 != 0 || p.Np > I8_ACC_STRIDE || p.Np < 2 * p.ctile ||
      p.n_pad != (long)p.nchunk * p.kchunk || p.n_pad < p.n)
    return cudaErrorInvalidValue;
  {
    const dim3 grid((unsigned)((p.kchunk / 8 + 255) / 256), (unsigned)(p.Np / 2), (unsigned)(p.ntile * p.nchunk));
    k_bslice<<<grid, 256, 0, s>>>(p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  size_t sm = lateral_i8_smem(p.Np);
  cudaError_t e = cudaFuncSetAttribute(k_lateral_i8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((p.npix + I8_M - 1) / I8_M), (unsigned)p.ntile, (unsigned)p.nchunk);
  k_lateral_i8<<<grid, I8_THREADS, sm, s>>>(p);
  return cudaGetLastError();
}

}  // namespace ytf

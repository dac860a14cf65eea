// ytf_lateral_tc.cu -- the 2D lateral synthesis on the 5th-generation tensor cores.
//
// G[pix, col] = Σ_n e^{i(kx_n x_i + ky_n y_j)} S[col, n]   (closed_form_G, lateral=:direct,
// mod_ClosedFormField.jl:743-753) as one real GEMM per tile:
//   A'[pix, 2n + {0,1}] = (Re P, Im P),  P = Px[n, i] · Py[n, j]
//   B'[(col, re), 2n + {0,1}] = (Sr, -Si),  B'[(col, im), 2n + {0,1}] = (Si, Sr)
//   C'[pix, (col, re|im)] = A' · B'^T
// Both operands are split in three BF16 terms (x = h + m + l, ~26 significant bits) and the
// six products hh, hm, mh, hl, mm, lh accumulate in FP32 in tensor memory (the dropped
// ml, lm, ll terms are O(2^-26)). The tensor core's FP32 accumulation truncates, so its
// error grows with the number of additions into one accumulator: the dominant hh product
// has an accumulator of its own, the five cross products (2^-8 smaller) share a second,
// and every 8 stages (128 nodes) both are folded into FP64 registers and restarted.
// Each CTA owns a 128-pixel x N' tile (N' = 2 x columns ≤ 96) and one slice of the nodes;
// slices are summed in FP64 by k_reduce_splits2.
//
// Per CTA: 256 threads produce the operands of a 16-node stage straight into shared memory
// in the canonical K-major no-swizzle layout (8-row x 16-byte core matrices), double
// buffered; one thread issues 12 tcgen05.mma (M=128, N=N', K=16) per stage and commits them
// to the stage's mbarrier; the producers of stage s+2 wait on it. The global loads of stage
// s+1 are issued before stage s is converted, so their latency overlaps the conversion.
// At each drain all 8 warps read the accumulators (tcgen05.ld 32x32b; warp w reads lanes
// 32(w%4).. and half w/4 of the columns) into FP64 registers; the last drain's values are
// the CTA's partial sums.
// Every wait is bounded; a timeout sets the error word and the CTA still frees its tensor
// memory and returns. No TMA and no multicast: operands are generated, not copied.
#include <cuda_bf16.h>

#include "ytf_complex.cuh"
#include "ytf_kernels.h"
#include "ytf_tcgen05.cuh"

namespace ytf {

constexpr int TC_M = 128;        // pixels per tile (MMA M)
constexpr int TC_NODES = 16;     // nodes per pipeline stage (real K = 32)
constexpr int TC_THREADS = 256;
constexpr int TC_TMEM_COLS = 256;
constexpr long TC_WAIT_LIMIT = 1L << 22;
constexpr int TC_NMAX = 96;      // largest MMA N (2 x 48 complex columns per tile)
constexpr int TC_XCOL = 128;     // tensor-memory column of the cross-product accumulator
constexpr int TC_PERIOD = 8;     // stages (8 x 16 nodes) between FP64 drains
constexpr int TC_SMAX = 3;       // (column, node) strength pairs per thread and stage: 48 x 16 / 256

// byte offset of element (row r, k) in an R x 32 bf16 plane
__device__ __forceinline__ uint32_t plane_off_bf(int r, int k) { return plane_off(r, 2 * k); }

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
  for (long i = 0; i < TC_WAIT_LIMIT; ++i)
    if (mbar_try(addr, parity)) return true;
  return false;
}

__device__ __forceinline__ void split3(float v, __nv_bfloat16& h, __nv_bfloat16& m, __nv_bfloat16& l) {
  h = __float2bfloat16_rn(v);
  float r = v - __bfloat162float(h);
  m = __float2bfloat16_rn(r);
  l = __float2bfloat16_rn(r - __bfloat162float(m));
}
__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred PD;\n\t"
      "setp.ne.b32 PD, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, PD;\n\t}"
      ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
      : "memory");
}

// Operands of one 16-node stage, held in registers between the global loads (issued one
// stage ahead) and their conversion into shared memory.
struct StageRegs {
  float2 px[8], py[8];
  double2 sv[TC_SMAX];
};

__device__ __forceinline__ void load_stage(const LateralTC& p, long nbase, long k1, int r, int hh, bool pv, int i, int j,
                                           int c0, int nct, int tid, StageRegs& R) {
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const long nn = nbase + 8 * hh + q;
    if (pv && nn < k1) {
      R.px[q] = p.Px[nn * p.nx + i];
      R.py[q] = p.Py[nn * p.ny + j];
    } else {
      R.px[q] = make_float2(0.f, 0.f);
      R.py[q] = make_float2(0.f, 0.f);
    }
  }
#pragma unroll
  for (int e = 0; e < TC_SMAX; ++e) {
    const int idx = tid + TC_THREADS * e;
    const int c = idx / TC_NODES, q = idx % TC_NODES;
    const long nn = nbase + q;
    R.sv[e] = (c < nct && nn < k1) ? p.S[(long)(c0 + c) * p.n + nn] : make_double2(0.0, 0.0);
  }
}

__global__ void __launch_bounds__(TC_THREADS, 1) k_lateral_tc(LateralTC p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long p0 = (long)blockIdx.x * TC_M;
  const int c0 = blockIdx.y * p.ctile;
  const int nct = min(p.ctile, p.ncol - c0);
  const long k0 = (long)blockIdx.z * p.kchunk;
  const long k1 = min(p.n, k0 + p.kchunk);
  const int nstages = k1 > k0 ? (int)((k1 - k0 + TC_NODES - 1) / TC_NODES) : 0;
  const uint32_t planeA = TC_M * 64u, planeB = (uint32_t)p.Np * 64u;
  const uint32_t stageBytes = 3u * planeA + 3u * planeB;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + 2 * stageBytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 2);

  // padding rows of B (rows 2*nct .. Np-1) are zero in both stages and never rewritten
  for (int s = 0; s < 2; ++s)
    for (int pl = 0; pl < 3; ++pl) {
      uint8_t* Bp = smem + s * stageBytes + 3 * planeA + pl * planeB;
      for (int idx = tid; idx < (p.Np - 2 * nct) * 16; idx += TC_THREADS) {
        int r = 2 * nct + idx / 16, kk = 2 * (idx % 16);
        *reinterpret_cast<uint32_t*>(Bp + plane_off_bf(r, kk)) = 0u;
      }
    }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(TC_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t tm_hh = tmem, tm_x = tmem + TC_XCOL;  // hh products / the five cross products
  // kind::f16: D F32 (bit 4), A BF16 (bits 7-9 = 1), B BF16 (bits 10-12 = 1), both K-major,
  // N >> 3 at bits 17-22, M >> 4 at bits 24-28
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(p.Np >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);

  // this thread's producer coordinates and its share of the drained accumulator
  const int r = tid & 127, hh = tid >> 7;
  const long pix = p0 + r;
  const bool pv = pix < p.npix;
  const int i = pv ? (int)(pix % p.nx) : 0, j = pv ? (int)(pix / p.nx) : 0;
  const int drow = 32 * (warp & 3) + lane, dhalf = warp >> 2, dcols = p.Np / 2;
  double acc[TC_NMAX / 2];
#pragma unroll
  for (int e = 0; e < TC_NMAX / 2; ++e) acc[e] = 0.0;

  bool failed = false;
  int committed = -1;  // last stage whose MMAs were committed (uniform across the CTA)
  StageRegs cur, nxt;
  if (nstages > 0) load_stage(p, k0, k1, r, hh, pv, i, j, c0, nct, tid, cur);
  for (int s = 0; s < nstages; ++s) {
    const int buf = s & 1;
    uint8_t* A = smem + buf * stageBytes;
    uint8_t* B = A + 3 * planeA;
    const long nbase = k0 + (long)s * TC_NODES;
    if (s + 1 < nstages) load_stage(p, nbase + TC_NODES, k1, r, hh, pv, i, j, c0, nct, tid, nxt);
    // buffer `buf` was read by the MMAs of stage s-2 (a completed phase returns at once)
    bool ok = true;
    if (s >= 2) ok = mbar_wait(smem_u32(&mbar[buf]), ((s - 2) >> 1) & 1);
    if (__syncthreads_or(!ok)) { failed = true; break; }
    // ---- A: phase products for 128 pixels x 16 nodes (8 nodes per thread) ----
    {
      uint32_t w[3][2][4];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float2 a = cur.px[q], b = cur.py[q];
        const float re = fmaf(a.x, b.x, -a.y * b.y), im = fmaf(a.x, b.y, a.y * b.x);
        __nv_bfloat16 rh, rm, rl, ih, imm, il;
        split3(re, rh, rm, rl);
        split3(im, ih, imm, il);
        w[0][q >> 2][q & 3] = pack2(rh, ih);
        w[1][q >> 2][q & 3] = pack2(rm, imm);
        w[2][q >> 2][q & 3] = pack2(rl, il);
      }
#pragma unroll
      for (int pl = 0; pl < 3; ++pl)
#pragma unroll
        for (int half = 0; half < 2; ++half) {
          uint4 v = make_uint4(w[pl][half][0], w[pl][half][1], w[pl][half][2], w[pl][half][3]);
          *reinterpret_cast<uint4*>(A + pl * planeA + plane_off_bf(r, 16 * hh + 8 * half)) = v;
        }
    }
    // ---- B: strengths of nct columns x 16 nodes ----
#pragma unroll
    for (int e = 0; e < TC_SMAX; ++e) {
      const int idx = tid + TC_THREADS * e;
      const int c = idx / TC_NODES, q = idx % TC_NODES;
      if (c < nct) {
        __nv_bfloat16 rh, rm, rl, ih, imm, il;
        split3((float)cur.sv[e].x, rh, rm, rl);
        split3((float)cur.sv[e].y, ih, imm, il);
        const __nv_bfloat16 rs[3] = {rh, rm, rl}, is[3] = {ih, imm, il};
#pragma unroll
        for (int pl = 0; pl < 3; ++pl) {
          uint8_t* Bp = B + pl * planeB;
          *reinterpret_cast<uint32_t*>(Bp + plane_off_bf(2 * c, 2 * q)) = pack2(rs[pl], __hneg(is[pl]));
          *reinterpret_cast<uint32_t*>(Bp + plane_off_bf(2 * c + 1, 2 * q)) = pack2(is[pl], rs[pl]);
        }
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    const bool period_start = (s % TC_PERIOD) == 0;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(A), b0 = smem_u32(B);
      const int pa[6] = {0, 0, 1, 0, 1, 2}, pb[6] = {0, 1, 0, 2, 1, 0};
#pragma unroll
      for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int pr = 0; pr < 6; ++pr) {
          const uint64_t ad = umma_desc(a0 + pa[pr] * planeA + t * 256u);
          const uint64_t bd = umma_desc(b0 + pb[pr] * planeB + t * 256u);
          // the first MMA of a drain period into each accumulator overwrites it
          const uint32_t accum = (period_start && t == 0 && (pr == 0 || pr == 1)) ? 0u : 1u;
          mma_f16(pr == 0 ? tm_hh : tm_x, ad, bd, idesc, accum);
        }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mbar[buf]))
                   : "memory");
    }
    committed = s;
    // ---- period end: fold both FP32 accumulators into the FP64 registers ----
    if ((s % TC_PERIOD) == TC_PERIOD - 1 || s == nstages - 1) {
      bool okd = mbar_wait(smem_u32(&mbar[buf]), (s >> 1) & 1);
      if (!okd) okd = mbar_wait(smem_u32(&mbar[buf]), (s >> 1) & 1);
      if (__syncthreads_or(!okd)) { failed = true; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t lanebase = (uint32_t)(32 * (warp & 3)) << 16;
#pragma unroll
      for (int e0 = 0; e0 < TC_NMAX / 2; e0 += 8) {
        if (e0 < dcols) {
          uint32_t vh[8], vx[8];
          const uint32_t col = (uint32_t)(dhalf * dcols + e0);
          tmem_ld8(tm_hh + lanebase + col, vh);
          tmem_ld8(tm_x + lanebase + col, vx);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int e = 0; e < 8; ++e) acc[e0 + e] += (double)__uint_as_float(vh[e]) + (double)__uint_as_float(vx[e]);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
    }
    cur = nxt;
  }
  if (failed) {
    // let any committed MMAs finish before the tensor memory is released
    if (committed >= 0) {
      bool ok = mbar_wait(smem_u32(&mbar[committed & 1]), (committed >> 1) & 1);
      (void)ok;
    }
    if (tid == 0) atomicOr(p.err, 1u);
  } else {
    const long pixd = p0 + drow;
    double2* out = p.partial + (long)blockIdx.z * p.npix * p.ncol;
    if (pixd < p.npix) {
#pragma unroll
      for (int e = 0; e < TC_NMAX / 2; e += 2) {
        if (e < dcols) {
          const int col = (dhalf * dcols + e) / 2;
          if (col < nct) out[pixd + p.npix * (long)(c0 + col)] = make_double2(acc[e], acc[e + 1]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS) : "memory");
}

// FP32 phase tables: Px[n][i] = e^{i kx_n x_i}, Py[n][j] = e^{i ky_n y_j} (computed in FP64)
__global__ void k_phase_tables(CacheView c, int nx, int ny, const double* xs, const double* ys, float2* Px, float2* Py) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int m = nx + ny;
  if (t >= c.n * m) return;
  long nn = t / m;
  int e = (int)(t % m);
  long k = nn % c.Nk, q = nn / c.Nk;
  double s, co;
  sincos(c.phi[q], &s, &co);
  double sn, cs;
  if (e < nx) {
    sincos(c.kr[k] * co * xs[e], &sn, &cs);
    Px[nn * nx + e] = make_float2((float)cs, (float)sn);
  } else {
    sincos(c.kr[k] * s * ys[e - nx], &sn, &cs);
    Py[nn * ny + (e - nx)] = make_float2((float)cs, (float)sn);
  }
}

cudaError_t launch_phase_tables(const CacheView& c, int nx, int ny, const double* xs, const double* ys, float2* Px,
                                float2* Py, cudaStream_t s) {
  long tot = c.n * (long)(nx + ny);
  if (tot <= 0) return cudaSuccess;
  k_phase_tables<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(c, nx, ny, xs, ys, Px, Py);
  return cudaGetLastError();
}

size_t lateral_tc_smem(int Np) {
  size_t stage = 3ul * TC_M * 64 + 3ul * (size_t)Np * 64;
  size_t b = 2 * stage + 64;
  return b;
}

// balanced column tiles of at most 48 complex columns (MMA N ≤ 96)
int lateral_tc_ctile(int ncol) {
  int ntiles = (ncol + 47) / 48;
  return (ncol + ntiles - 1) / ntiles;
}

cudaError_t launch_lateral_tc(const LateralTC& p, int splits, cudaStream_t s) {
  size_t sm = lateral_tc_smem(p.Np);
  cudaError_t e = cudaFuncSetAttribute(k_lateral_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((p.npix + TC_M - 1) / TC_M), (unsigned)((p.ncol + p.ctile - 1) / p.ctile), (unsigned)splits);
  k_lateral_tc<<<grid, TC_THREADS, sm, s>>>(p);
  return cudaGetLastError();
}

}  // namespace ytf

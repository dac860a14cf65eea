// ytf_mlp.cu -- the small MLP of the learned node placement: forward, backward and Adam
// kernels, and its C ABI.
//
// Network: L linear layers (sizes n_0 -> n_1 -> ... -> n_L), GELU after every layer but the
// last. Master parameters are FP32 (W_l [n_l x n_{l-1}] row-major, then b_l [n_l], layer by
// layer); every forward/backward pass first rounds the weights to BF16 and multiplies with
// those, accumulating in FP32 ("BF16 weights, FP32 accumulation"). Activations and gradients
// are FP32. Loss over a batch of B samples with targets (t0, t1):
//   ℓ = mean_b (o0 - t0)^2 + mean_b [softplus(o1) - t1 o1]
// (o0: the log-response prediction, o1: the logit of the pole-proximity score).
//
// One strided GEMM serves the three products of a layer:
//   forward  Z[b][o]  = Σ_i H[b][i] W[o][i] + bias[o]   (then GELU)
//   input    dH[b][i] = Σ_o dZ[b][o] W[o][i]
//   weights  dW[o][i] = Σ_b dZ[b][o] H[b][i]
// C[m][n] = Σ_k A(m, k) B(k, n), A(m, k) = A[m sam + k sak], B(k, n) = B[k sbk + n sbn], on the
// tensor cores (tcgen05.mma kind::f16, BF16 operands, FP32 accumulation in tensor memory). The
// BF16 weights enter as they are; an FP32 operand (activations, gradients) is split into two
// BF16 terms hi = bf16(v), lo = bf16(v - hi), and the products hi·hi, hi·lo, lo·hi are summed,
// so an FP32 operand keeps about 16 significant bits (the dropped lo·lo is below 2^-16 of it).
// A CTA computes a 128 x Np tile (Np = N rounded up to 16, at most 256) over K in blocks of
// 128: its 128 threads convert the block's operands into shared memory (planes of 64-byte rows,
// 32 BF16 each, the canonical no-swizzle K-major layout), one thread issues the block's MMAs,
// their commit frees the buffers for the next block; the 4 warps then drain the accumulator
// (warp w: tensor-memory lanes 32w..32w+31 = the tile's rows) with bias, accumulation and GELU.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/ytf.h"
#include "ytf_tcgen05.cuh"

namespace ytf {
namespace mlp {

constexpr int GM = 128;          // tile rows (MMA M)
constexpr int GNMAX = 256;       // largest tile width (MMA N)
constexpr int GKB = 128;         // K per block: 4 planes of 32
constexpr long GWAIT = 1L << 24; // polls of the bounded commit wait

__device__ __forceinline__ uint32_t plane_bf(int r, int k) { return plane_off(r, 2 * k); }

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred PD;\n\t"
      "setp.ne.b32 PD, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, PD;\n\t}" ::"r"(tmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
      : "memory");
}

// the two BF16 terms of a source value (the second is 0 for a BF16 source)
__device__ __forceinline__ void split_bf(float v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(v);
  lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

// tn: the tile width (128 or 256). With ksl > 0 the K range is split: CTA (x, y, z) sums
// K in [z ksl, (z + 1) ksl) and writes its raw sums to part[z][M][N] (k_splitk_finish adds
// the slices, the bias, the accumulation and GELU); otherwise it finishes the tile itself.
template <class TA, class TB>
__global__ void __launch_bounds__(128, 1) k_gemm_tc(int M, int N, int K, const TA* __restrict__ A, long sam, long sak,
                                                     const TB* __restrict__ B, long sbk, long sbn,
                                                     float* __restrict__ C, long ldc, const float* __restrict__ bias,
                                                     float* __restrict__ H, int act, int accumulate, int tn, int ksl,
                                                     float* __restrict__ part, unsigned* __restrict__ err) {
  constexpr bool SA = std::is_same<TA, float>::value;  // split A into two terms
  constexpr bool SB = std::is_same<TB, float>::value;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint64_t done;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * GM, n0 = blockIdx.x * tn;
  const int nt = min(tn, N - n0);
  const int kbeg = ksl > 0 ? (int)blockIdx.z * ksl : 0;
  const int kend = ksl > 0 ? min(K, kbeg + ksl) : K;
  const int Np = ((nt + 15) / 16) * 16;
  const uint32_t planeA = GM * 64u, planeB = (uint32_t)Np * 64u;
  constexpr int NPL = GKB / 32;
  uint8_t* Ahi = smem;
  uint8_t* Alo = Ahi + NPL * planeA;
  uint8_t* Bhi = Alo + (SA ? NPL * planeA : 0);
  uint8_t* Blo = Bhi + NPL * planeB;
  if (tid == 0) {
    mbar_init(smem_u32(&done), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(GNMAX)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base;
  // kind::f16: D F32 (bit 4), A BF16 (bits 7-9 = 1), B BF16 (bits 10-12 = 1), both K-major
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(Np >> 3) << 17) | ((uint32_t)(GM >> 4) << 24);
  bool ok = true;
  int round = 0;
  for (int k0 = kbeg; k0 < kend; k0 += GKB, ++round) {
    if (round > 0) {
      // the previous block's MMAs have read the buffers before they are overwritten
      bool got = false;
      for (long it = 0; it < GWAIT && !got; ++it) got = mbar_try(smem_u32(&done), (round - 1) & 1);
      if (!got) { ok = false; if (tid == 0) atomicOr(err, 1u); break; }
    }
    for (int e = tid; e < GM * GKB; e += 128) {
      int r, k;
      if (sak == 1) { r = e / GKB; k = e % GKB; } else { k = e / GM; r = e % GM; }
      const int m = m0 + r, kk = k0 + k;
      const float v = (m < M && kk < kend) ? (float)A[(long)m * sam + (long)kk * sak] : 0.f;
      __nv_bfloat16 hi, lo;
      split_bf(v, hi, lo);
      const uint32_t off = (k >> 5) * planeA + plane_bf(r, k & 31);
      *reinterpret_cast<__nv_bfloat16*>(Ahi + off) = hi;
      if (SA) *reinterpret_cast<__nv_bfloat16*>(Alo + off) = lo;
    }
    for (int e = tid; e < Np * GKB; e += 128) {
      int r, k;
      if (sbk == 1) { r = e / GKB; k = e % GKB; } else { k = e / Np; r = e % Np; }
      const int n = n0 + r, kk = k0 + k;
      const float v = (r < nt && kk < kend) ? (float)B[(long)kk * sbk + (long)n * sbn] : 0.f;
      __nv_bfloat16 hi, lo;
      split_bf(v, hi, lo);
      const uint32_t off = (k >> 5) * planeB + plane_bf(r, k & 31);
      *reinterpret_cast<__nv_bfloat16*>(Bhi + off) = hi;
      if (SB) *reinterpret_cast<__nv_bfloat16*>(Blo + off) = lo;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int pl = 0; pl < NPL; ++pl)
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const uint32_t oa = pl * planeA + t * 256u, ob = pl * planeB + t * 256u;
          // the first MMA of the tile overwrites the accumulator, every other one adds to it
          mma_bf16(tmem, umma_desc(smem_u32(Ahi + oa)), umma_desc(smem_u32(Bhi + ob)), idesc,
                   (k0 > kbeg || pl > 0 || t > 0) ? 1u : 0u);
          if (SB) mma_bf16(tmem, umma_desc(smem_u32(Ahi + oa)), umma_desc(smem_u32(Blo + ob)), idesc, 1u);
          if (SA) mma_bf16(tmem, umma_desc(smem_u32(Alo + oa)), umma_desc(smem_u32(Bhi + ob)), idesc, 1u);
        }
      tc_commit(smem_u32(&done));
    }
  }
  // the last block's MMAs (and with them every earlier one) complete before the drain
  if (round > 0) {
    bool got = false;
    for (long it = 0; it < GWAIT && !got; ++it) got = mbar_try(smem_u32(&done), (round - 1) & 1);
    if (!got) { ok = false; if (tid == 0) atomicOr(err, 1u); }
  }
  ok = __all_sync(0xffffffffu, ok);
  tc_fence_after();
  if (ok && round > 0) {
    const int m = m0 + 32 * warp + lane;
    const uint32_t lanebase = (uint32_t)(32 * warp) << 16;
    for (int c0 = 0; c0 < Np; c0 += 8) {
      uint32_t v[8];
      tmem_ld8(tmem + lanebase + c0, v);
      tmem_wait_ld();
      if (m < M) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int n = n0 + c0 + j;
          if (c0 + j >= nt) break;
          if (part) {
            part[((long)blockIdx.z * M + m) * N + n] = __uint_as_float(v[j]);
            continue;
          }
          float z = __uint_as_float(v[j]) + (bias ? bias[n] : 0.f);
          if (accumulate) z += C[(long)m * ldc + n];
          C[(long)m * ldc + n] = z;
          if (H) H[(long)m * ldc + n] = act ? 0.5f * z * (1.f + erff(z * 0.70710678118654752f)) : z;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(GNMAX) : "memory");
}

// the K slices of a split GEMM summed in slice order, then bias, accumulation and GELU
__global__ void k_splitk_finish(int M, int N, int S, const float* __restrict__ part, float* __restrict__ C, long ldc,
                                const float* __restrict__ bias, float* __restrict__ H, int act, int accumulate) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)M * N) return;
  const int m = (int)(t / N), n = (int)(t % N);
  float z = 0.f;
  for (int sl = 0; sl < S; ++sl) z += part[(long)sl * M * N + t];
  z += bias ? bias[n] : 0.f;
  if (accumulate) z += C[(long)m * ldc + n];
  C[(long)m * ldc + n] = z;
  if (H) H[(long)m * ldc + n] = act ? 0.5f * z * (1.f + erff(z * 0.70710678118654752f)) : z;
}

template <class TA, class TB>
size_t gemm_tc_smem(int Np) {
  constexpr bool SA = std::is_same<TA, float>::value, SB = std::is_same<TB, float>::value;
  return (size_t)(GKB / 32) * ((SA ? 2 : 1) * GM * 64 + (SB ? 2 : 1) * (size_t)Np * 64);
}

// dZ = dH * GELU'(Z), GELU'(z) = Φ(z) + z φ(z)
__global__ void k_gelu_back(long n, const float* __restrict__ Z, const float* __restrict__ dH, float* __restrict__ dZ) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float z = Z[t];
  const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
  dZ[t] = dH[t] * (cdf + z * pdf);
}

// column sums: db[o] = Σ_b dZ[b][o]
__global__ void k_colsum(int B, int N, const float* __restrict__ dZ, float* __restrict__ db) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= N) return;
  float s = 0.f;
  for (int b = 0; b < B; ++b) s += dZ[(long)b * N + o];
  db[o] = s;
}

// loss terms and the output gradient; out: [B][2], T: [B][2]; per-sample loss into lb
__global__ void k_loss(int B, const float* __restrict__ out, const float* __restrict__ T, float* __restrict__ dout,
                       float* __restrict__ lb) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const float o0 = out[2 * b], o1 = out[2 * b + 1], t0 = T[2 * b], t1 = T[2 * b + 1];
  const float e = o0 - t0;
  const float sp = o1 > 0 ? o1 + log1pf(expf(-o1)) : log1pf(expf(o1));
  lb[b] = e * e + (sp - t1 * o1);
  const float sig = 1.f / (1.f + expf(-o1));
  dout[2 * b] = 2.f * e / B;
  dout[2 * b + 1] = (sig - t1) / B;
}

// a mini-batch drawn with replacement from the device-resident set: sample index from a
// counter-based hash (splitmix64) of (seed, step, row)
__global__ void k_gather(int B, int d, long n, unsigned long long seed, long step, const float* __restrict__ X,
                         const float* __restrict__ T, float* __restrict__ Xb, float* __restrict__ Tb) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)B * (d + 2)) return;
  const int b = (int)(t / (d + 2)), c = (int)(t % (d + 2));
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(step * B + b + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const long i = (long)(z % (unsigned long long)n);
  if (c < d) Xb[(long)b * d + c] = X[i * d + c];
  else Tb[2L * b + (c - d)] = T[2 * i + (c - d)];
}

__global__ void k_to_bf16(long n, const float* __restrict__ a, __nv_bfloat16* __restrict__ b) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) b[t] = __float2bfloat16_rn(a[t]);
}

__global__ void k_adam(long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t];
  const float mt = b1 * m[t] + (1.f - b1) * gt;
  const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
}

}  // namespace mlp
}  // namespace ytf

using namespace ytf::mlp;

struct ytf_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<int> sizes;          // n_0 .. n_L
  std::vector<long> woff, boff;    // offsets of W_l and b_l in the parameter vector
  long nparam = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  __nv_bfloat16* wb = nullptr;     // BF16 copy of the parameters (weights used from here)
  long step = 0;
  // activations for the largest batch seen: Z_l and H_l per layer, gradients, loss terms
  long cap = 0;
  std::vector<float*> Z, H, dZ, dH;
  float *T = nullptr, *lb = nullptr, *X = nullptr;
  unsigned* tc_err = nullptr;      // set by a tensor-core GEMM whose commit wait ran out
  float* part = nullptr;           // K-slice sums of split GEMMs
  size_t part_cap = 0;
  std::string err;
  ~ytf_mlp() {
    cudaFree(p); cudaFree(g); cudaFree(m); cudaFree(v); cudaFree(wb);
    for (auto* q : Z) cudaFree(q);
    for (auto* q : H) cudaFree(q);
    for (auto* q : dZ) cudaFree(q);
    for (auto* q : dH) cudaFree(q);
    cudaFree(T); cudaFree(lb); cudaFree(X); cudaFree(tc_err); cudaFree(part);
  }
};

namespace {

int mfail(ytf_mlp* n, int code, const std::string& msg) {
  if (n) n->err = msg;
  return code;
}
#define MCK(call)                                                                    \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) return mfail(net, YTF_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)

template <class TA, class TB>
cudaError_t gemm(ytf_mlp* net, int M, int N, int K, const TA* A, long sam, long sak, const TB* B, long sbk, long sbn,
                 float* C, long ldc, const float* bias, float* H, int act, int accumulate) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  // fill the 148 SMs: 128-wide tiles when 256-wide ones are too few, then K slices
  const int mt = (M + GM - 1) / GM;
  const int tn = (long)mt * ((N + GNMAX - 1) / GNMAX) < 148 && N > 128 ? 128 : GNMAX;
  const int tiles = mt * ((N + tn - 1) / tn);
  int S = 1, ksl = 0;
  if (tiles < 74 && K >= 2 * GKB) {
    S = std::min((148 + tiles - 1) / tiles, (K + GKB - 1) / GKB);
    ksl = (((K + S - 1) / S + GKB - 1) / GKB) * GKB;
    S = (K + ksl - 1) / ksl;
  }
  float* part = nullptr;
  if (S > 1) {
    const size_t need = (size_t)S * M * N;
    if (need > net->part_cap) {
      cudaFree(net->part);
      net->part = nullptr;
      net->part_cap = 0;
      cudaError_t e = cudaMalloc(&net->part, sizeof(float) * need);
      if (e != cudaSuccess) return e;
      net->part_cap = need;
    }
    part = net->part;
  } else {
    ksl = 0;
  }
  const int Np = ((std::min(N, tn) + 15) / 16) * 16;
  const size_t sm = gemm_tc_smem<TA, TB>(Np);
  cudaError_t e = cudaFuncSetAttribute(k_gemm_tc<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  dim3 grid((N + tn - 1) / tn, mt, S);
  k_gemm_tc<TA, TB><<<grid, 128, sm, net->stream>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc, bias, H, act, accumulate,
                                                   tn, ksl, part, net->tc_err);
  if ((e = cudaGetLastError()) != cudaSuccess || S == 1) return e;
  k_splitk_finish<<<(unsigned)(((long)M * N + 255) / 256), 256, 0, net->stream>>>(M, N, S, part, C, ldc, bias, H, act,
                                                                              accumulate);
  return cudaGetLastError();
}

int ensure(ytf_mlp* net, long B) {
  if (B <= net->cap) return YTF_OK;
  for (auto* q : net->Z) cudaFree(q);
  for (auto* q : net->H) cudaFree(q);
  for (auto* q : net->dZ) cudaFree(q);
  for (auto* q : net->dH) cudaFree(q);
  cudaFree(net->T); cudaFree(net->lb); cudaFree(net->X);
  const int L = (int)net->sizes.size() - 1;
  net->Z.assign(L + 1, nullptr); net->H.assign(L + 1, nullptr);
  net->dZ.assign(L + 1, nullptr); net->dH.assign(L + 1, nullptr);
  for (int l = 0; l <= L; ++l) {
    const size_t bytes = sizeof(float) * B * net->sizes[l];
    MCK(cudaMalloc(&net->H[l], bytes));
    MCK(cudaMalloc(&net->dH[l], bytes));
    if (l > 0) {
      MCK(cudaMalloc(&net->Z[l], bytes));
      MCK(cudaMalloc(&net->dZ[l], bytes));
    }
  }
  MCK(cudaMalloc(&net->T, sizeof(float) * 2 * B));
  MCK(cudaMalloc(&net->lb, sizeof(float) * B));
  MCK(cudaMalloc(&net->X, sizeof(float) * B * net->sizes[0]));
  net->cap = B;
  return YTF_OK;
}

// forward pass of B samples already in H[0]
int forward(ytf_mlp* net, int B) {
  const int L = (int)net->sizes.size() - 1;
  const long n = net->nparam;
  k_to_bf16<<<(unsigned)((n + 255) / 256), 256, 0, net->stream>>>(n, net->p, net->wb);
  MCK(cudaGetLastError());
  for (int l = 1; l <= L; ++l) {
    const int in = net->sizes[l - 1], out = net->sizes[l];
    MCK((gemm<float, __nv_bfloat16>(net, B, out, in, net->H[l - 1], in, 1, net->wb + net->woff[l - 1], 1, in,
                                   net->Z[l], out, net->p + net->boff[l - 1], net->H[l], l < L ? 1 : 0, 0)));
  }
  return YTF_OK;
}

// backward from the targets in T; gradients into g
int backward(ytf_mlp* net, int B) {
  const int L = (int)net->sizes.size() - 1;
  k_loss<<<(B + 255) / 256, 256, 0, net->stream>>>(B, net->H[L], net->T, net->dZ[L], net->lb);
  MCK(cudaGetLastError());
  for (int l = L; l >= 1; --l) {
    const int in = net->sizes[l - 1], out = net->sizes[l];
    if (l < L) {
      const long cnt = (long)B * out;
      k_gelu_back<<<(unsigned)((cnt + 255) / 256), 256, 0, net->stream>>>(cnt, net->Z[l], net->dH[l], net->dZ[l]);
      MCK(cudaGetLastError());
    }
    // dW = dZ^T H, db = Σ dZ
    MCK((gemm<float, float>(net, out, in, B, net->dZ[l], 1, out, net->H[l - 1], in, 1, net->g + net->woff[l - 1],
                           in, nullptr, nullptr, 0, 0)));
    k_colsum<<<(out + 255) / 256, 256, 0, net->stream>>>(B, out, net->dZ[l], net->g + net->boff[l - 1]);
    MCK(cudaGetLastError());
    if (l > 1)
      MCK((gemm<float, __nv_bfloat16>(net, B, in, out, net->dZ[l], out, 1, net->wb + net->woff[l - 1], in, 1,
                                     net->dH[l - 1], in, nullptr, nullptr, 0, 0)));
  }
  return YTF_OK;
}

}  // namespace

extern "C" {

int ytf_mlp_create(int device, int nlayers, const int* sizes, unsigned long long seed, ytf_mlp** out) {
  if (!out || nlayers < 1 || !sizes) return YTF_ERR_ARG;
  *out = nullptr;
  for (int l = 0; l <= nlayers; ++l)
    if (sizes[l] < 1) return YTF_ERR_ARG;
  if (sizes[nlayers] != 2) return YTF_ERR_ARG;  // (log-response, pole-score logit)
  if (cudaSetDevice(device) != cudaSuccess) return YTF_ERR_CUDA;
  ytf_mlp* net = new ytf_mlp();
  net->device = device;
  net->sizes.assign(sizes, sizes + nlayers + 1);
  long o = 0;
  for (int l = 1; l <= nlayers; ++l) {
    net->woff.push_back(o);
    o += (long)sizes[l] * sizes[l - 1];
    net->boff.push_back(o);
    o += sizes[l];
  }
  net->nparam = o;
  // He-style initialisation from a seeded 64-bit LCG (uniform, variance 2 / fan_in), zero bias
  std::vector<float> h(o, 0.f);
  unsigned long long st = seed * 6364136223846793005ull + 1442695040888963407ull;
  for (int l = 1; l <= nlayers; ++l) {
    const float a = std::sqrt(6.0f / sizes[l - 1]) * (l == nlayers ? 0.5f : 1.0f);
    for (long i = 0; i < (long)sizes[l] * sizes[l - 1]; ++i) {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      const double u = (double)(st >> 11) * (1.0 / 9007199254740992.0);
      h[net->woff[l - 1] + i] = (float)((2 * u - 1) * a);
    }
  }
  int rc = YTF_OK;
  if (cudaMalloc(&net->p, 4 * o) != cudaSuccess || cudaMalloc(&net->g, 4 * o) != cudaSuccess ||
      cudaMalloc(&net->m, 4 * o) != cudaSuccess || cudaMalloc(&net->v, 4 * o) != cudaSuccess ||
      cudaMalloc(&net->wb, 2 * o) != cudaSuccess || cudaMalloc(&net->tc_err, sizeof(unsigned)) != cudaSuccess)
    rc = YTF_ERR_NOMEM;
  if (!rc && (cudaMemcpy(net->p, h.data(), 4 * o, cudaMemcpyHostToDevice) != cudaSuccess ||
              cudaMemset(net->m, 0, 4 * o) != cudaSuccess || cudaMemset(net->v, 0, 4 * o) != cudaSuccess ||
              cudaMemset(net->g, 0, 4 * o) != cudaSuccess || cudaMemset(net->tc_err, 0, sizeof(unsigned)) != cudaSuccess))
    rc = YTF_ERR_CUDA;
  if (rc) { delete net; return rc; }
  *out = net;
  return YTF_OK;
}

int ytf_mlp_destroy(ytf_mlp* net) {
  if (net) { cudaSetDevice(net->device); cudaStreamSynchronize(net->stream); delete net; }
  return YTF_OK;
}

const char* ytf_mlp_last_error(const ytf_mlp* net) { return net ? net->err.c_str() : "null network"; }

long ytf_mlp_num_params(const ytf_mlp* net) { return net ? net->nparam : 0; }

int ytf_mlp_set_stream(ytf_mlp* net, void* stream) {
  if (!net) return YTF_ERR_ARG;
  net->stream = (cudaStream_t)stream;
  return YTF_OK;
}

int ytf_mlp_params(ytf_mlp* net, float* get, const float* set) {
  if (!net) return YTF_ERR_ARG;
  MCK(cudaSetDevice(net->device));
  if (set) MCK(cudaMemcpyAsync(net->p, set, 4 * net->nparam, cudaMemcpyHostToDevice, net->stream));
  if (get) MCK(cudaMemcpyAsync(get, net->p, 4 * net->nparam, cudaMemcpyDeviceToHost, net->stream));
  MCK(cudaStreamSynchronize(net->stream));
  return YTF_OK;
}

int ytf_mlp_forward(ytf_mlp* net, int B, const float* X, float* out, int on_device) {
  if (!net || B < 0 || (B > 0 && (!X || !out))) return YTF_ERR_ARG;
  if (B == 0) return YTF_OK;
  MCK(cudaSetDevice(net->device));
  int rc = ensure(net, B);
  if (rc) return rc;
  const size_t xb = sizeof(float) * B * net->sizes[0];
  MCK(cudaMemcpyAsync(net->H[0], X, xb, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, net->stream));
  if ((rc = forward(net, B))) return rc;
  const int L = (int)net->sizes.size() - 1;
  MCK(cudaMemcpyAsync(out, net->H[L], sizeof(float) * 2 * B, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                      net->stream));
  MCK(cudaStreamSynchronize(net->stream));
  return YTF_OK;
}

int ytf_mlp_gradients(ytf_mlp* net, int B, const float* X, const float* T, float* grad, float* loss, int on_device) {
  if (!net || B < 1 || !X || !T) return YTF_ERR_ARG;
  MCK(cudaSetDevice(net->device));
  int rc = ensure(net, B);
  if (rc) return rc;
  const auto kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  MCK(cudaMemcpyAsync(net->H[0], X, sizeof(float) * B * net->sizes[0], kind, net->stream));
  MCK(cudaMemcpyAsync(net->T, T, sizeof(float) * 2 * B, kind, net->stream));
  if ((rc = forward(net, B)) || (rc = backward(net, B))) return rc;
  if (grad) MCK(cudaMemcpyAsync(grad, net->g, 4 * net->nparam, cudaMemcpyDeviceToHost, net->stream));
  if (loss) {
    std::vector<float> lb(B);
    MCK(cudaMemcpyAsync(lb.data(), net->lb, 4 * (size_t)B, cudaMemcpyDeviceToHost, net->stream));
    MCK(cudaStreamSynchronize(net->stream));
    double s = 0;
    for (float x : lb) s += x;
    *loss = (float)(s / B);
  }
  MCK(cudaStreamSynchronize(net->stream));
  return YTF_OK;
}

int ytf_mlp_train(ytf_mlp* net, long n, const float* X, const float* T, int batch, int steps, float lr,
                  unsigned long long seed, float* losses) {
  if (!net || n < 1 || !X || !T || batch < 1 || steps < 0) return YTF_ERR_ARG;
  MCK(cudaSetDevice(net->device));
  int rc = ensure(net, batch);
  if (rc) return rc;
  const int d = net->sizes[0];
  // mini-batches drawn from the device-resident set (X: [n][d], T: [n][2]) on the device
  float* dl = nullptr;
  MCK(cudaMalloc(&dl, sizeof(float) * batch));
  std::vector<float> lb(batch);
  for (int s = 0; s < steps; ++s) {
    const long cnt = (long)batch * (d + 2);
    k_gather<<<(unsigned)((cnt + 255) / 256), 256, 0, net->stream>>>(batch, d, n, seed, net->step, X, T, net->H[0],
                                                                      net->T);
    if (cudaGetLastError() != cudaSuccess) { cudaFree(dl); return mfail(net, YTF_ERR_CUDA, "gather launch"); }
    if ((rc = forward(net, batch)) || (rc = backward(net, batch))) { cudaFree(dl); return rc; }
    net->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)net->step), c2 = 1.f - std::pow(b2, (float)net->step);
    k_adam<<<(unsigned)((net->nparam + 255) / 256), 256, 0, net->stream>>>(net->nparam, net->p, net->g, net->m, net->v,
                                                                           lr, b1, b2, 1e-8f, c1, c2);
    if (cudaGetLastError() != cudaSuccess) { cudaFree(dl); return mfail(net, YTF_ERR_CUDA, "adam launch"); }
    if (losses) {
      cudaMemcpyAsync(lb.data(), net->lb, 4 * (size_t)batch, cudaMemcpyDeviceToHost, net->stream);
      cudaStreamSynchronize(net->stream);
      double a = 0;
      for (float x : lb) a += x;
      losses[s] = (float)(a / batch);
    }
  }
  cudaFree(dl);
  MCK(cudaStreamSynchronize(net->stream));
  return YTF_OK;
}

}  // extern "C"

// ytf_kernels.h -- parameter blocks and launchers shared by the libytf kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ytf {

constexpr int MAXL = 32;  // layers per stack (bit masks below are 32 wide)

// per-node status bits (the reference's numerical guards, as data instead of exceptions)
enum : uint8_t {
  ST_VALID = 1,        // node contributes (valid[k] of the reference)
  ST_EIGEN = 2,        // 4x4 QR did not converge
  ST_SORT = 4,         // more than two modes in one direction (reference: BoundsError)
  ST_SINGULAR = 8,     // exact zero pivot in the source projection solve (interfaces fall back to QR)
  ST_SEEDS = 16,       // non-finite point seeds (reference: `continue`)
  ST_TNONFINITE = 32,  // some T^o non-finite (Tvalid[o][k] = false)
};

// one layer: kinds (0 iso, 1 uniaxial, 2 biaxial, 3 general), column-major 3x3 ε and μ
// (interleaved re/im), thickness
struct LayerDev {
  int ekind, mkind;
  double eps[18];
  double mu[18];
  double d;
};

struct TransferParams {
  const LayerDev* layers;  // device, nL entries
  int nL, src, nobs;       // src, obs[] are 1-based
  int obs[MAXL];
  uint32_t needL, needR;   // layers (bit l-1) whose SLeft / SRight are kept in scratch
  double omega;
  int mode;                // 0: 1D nodes; 1: 2D full solve; 2: 2D rotation base (φ = 0)
  long n;                  // nodes solved by k_layer_modes / k_chain (this chunk)
  long off;                // global index of the chunk's first node
  long nout;               // nodes of the output cache (== n except the rotation fill)
  int Nk, Np;
  const double* kr;        // 1D: kx nodes; 2D: kρ nodes
  const double* kr_im;     // 1D nodes on a deformed contour: imaginary parts (else NULL)
  const double* phi;       // 2D: φ nodes
  // scratch
  double2* modes;          // [nL][20][n]
  uint8_t* lstat;          // [nL][n]
  double2* sint;           // [nL-1][16][n]
  double2* sleft;          // [nL][16][n]
  double2* sright;         // [nL][16][n]
  uint8_t* dec;            // [nL-1][n] matching decisions per interface (forward-only chain)
  // outputs
  uint8_t* status;         // [nout] (rotation base: [n])
  uint8_t* valid;          // [nout]
  uint8_t* tvalid;         // [nobs][nout]
  double2* Tout;           // [nobs][16][nout], column-major 4x4 per node
  double2* Qf;             // [2][nout]
  double2* Qb;             // [2][nout]
  double2* sf;             // [6][nout], column-major 2x3
  double2* sb;             // [6][nout]
  double2* basis;          // [nobs][16][nout]: exf0 exf1 eyf0 eyf1 ezf0 ezf1 exb.. eyb.. ezb.. kzf0 kzf1 kzb0 kzb1
  // response mode of the forward-only chain (_cavity_response): when set, k_scan writes
  // resp[node] and the status only (no T^o, seeds, basis, valid flags)
  double* resp;            // [nout]
};

cudaError_t launch_layer_modes(const TransferParams& p, cudaStream_t stream);
cudaError_t launch_layer_modes_qr(const TransferParams& p, cudaStream_t stream);
cudaError_t launch_chain(const TransferParams& p, cudaStream_t stream);
// k_chain when every observation layer is the source layer, as three kernels: part 0..2 =
// k_iface, k_seeds, k_scan, launched in that order (needs the sint and dec scratch)
cudaError_t launch_chain_part(int part, const TransferParams& p, cudaStream_t stream);
// batched transfer kernels over nb problems (device arrays probs[nb], off[nb + 1]; total =
// off[nb]): kernel 0 = layer modes, 1 = general QR pass, 3 = chain, 5-7 = the forward-only
// chain (seeds, iface (off over (nL - 1) n interface-node pairs), scan; iface first)
cudaError_t launch_transfer_batch(int kernel, const TransferParams* probs, const long* off, int nb, long total,
                                  cudaStream_t stream);
cudaError_t launch_rotate_fill(const TransferParams& p, const uint8_t* base_status, const uint8_t* base_tvalid,
                               const double2* Tbase, cudaStream_t stream);

// persistent transfer kernels: tiles of units of one problem each, pulled from a counter
struct TileQueue {
  const int* prob;    // [ntiles] problem index into the parameter array
  const long* start;  // [ntiles] first unit of the tile
  const long* end;    // [ntiles] one past its last unit
  int ntiles;
  unsigned* counter;  // next tile; zero before the launch
};
// stage: 0 modes, 1 QR pass, 3 general chain, 6 iface, 5 seeds, 7 scan (units as the batched
// kernels, iface before seeds); block 128 or 256 threads; grid CTAs (persistent)
cudaError_t launch_persist(int stage, int block, int grid, const TransferParams* probs, const TileQueue& q,
                           cudaStream_t s);

// read-only view of a device transfer cache for the synthesis kernels
struct CacheView {
  long n;
  int Nk, Np;
  int src;          // 1-based
  double d_src;
  const double* kr;    // [Nk]
  const double* wr;    // [Nk]
  const double* kri;   // [Nk] imaginary parts of complex 1D nodes (deformed contour), else NULL
  const double* wri;   // [Nk] imaginary parts of their weights
  const double* phi;   // [Np]
  const double* wphi;  // [Np]
  const uint8_t* valid;
  const uint8_t* tvalid;  // of the obs layer in use: [n]
  const double2* T;       // of the obs layer: [16][n]
  const double2* Qf;
  const double2* Qb;
  const double2* sf;
  const double2* sb;
  const double2* basis;   // of the obs layer: [16][n]
};

struct SynthParams {
  CacheView c;
  int same;          // obs layer == source layer
  int with_direct;   // add the same-layer direct term
  double uf_F, ub_F, uf_B, ub_B;  // seed masks of the reflected amplitudes (terms)
  double zpos;       // source position in the cavity frame
  double d_obs;
  int nz;
  const double* zo;  // [nz] device
};

// 1D coefficient columns per height: of the 13 complex coefficients (order 0: xx yx xy yy zz;
// order 1: zx zy xz yz; order 2: xx yx xy yy) the synthesis stores the 9 independent ones,
// order 0: xx yx zz, order 1: zx zy xz yz, order 2: xx yx, because in the azimuthally
// symmetric 1D integrand yy = xx and xy = -yx of order 0, xy = yx and yy = -xx of order 2
// exactly (the same products summed in swapped order, or negated: bit for bit); the pixel
// assembly restores them. Real columns per height of orders 0, 1, 2 and the orders' offsets.
constexpr int C1D_R0 = 6, C1D_R1 = 8, C1D_R2 = 4;
constexpr int C1D_OFF1 = C1D_R0, C1D_OFF2 = C1D_R0 + C1D_R1, C1D_RT = C1D_R0 + C1D_R1 + C1D_R2;
constexpr int C1D_RMAX = C1D_R1;  // the widest order

// 1D Jacobi-Anger synthesis
cudaError_t launch_coef1d(const SynthParams& p, double* C0, double* C1, double* C2, cudaStream_t s);
// the same through per-node reflected amplitudes in amp ([12][n] complex scratch)
cudaError_t launch_coef1d_amp(const SynthParams& p, double2* amp, double* C0, double* C1, double* C2, cudaStream_t s);
// the same columns rounded to FP32 (the int8x3 contraction's input)
cudaError_t launch_coef1d_amp(const SynthParams& p, double2* amp, float* C0, float* C1, float* C2, cudaStream_t s);
cudaError_t launch_bessel_c(const double* kr, const double* kri, long nk, const double* rho, int nr, double* J,
                            cudaStream_t s);
cudaError_t launch_combine_complex(long M, int N2, const double* A, const double* B, double* P, cudaStream_t s);
cudaError_t launch_bessel_eval(long n, int order, const double* zr, const double* zi, double* outr, double* outi,
                               cudaStream_t s);
cudaError_t launch_bessel(const double* kr, long nk, const double* rho, int nr, double* J0, double* J1, double* J2,
                          cudaStream_t s);
int dgemm_splits(int K, int splits);  // effective split count of launch_dgemm_nt
cudaError_t launch_dgemm_nt(int M, int N, int K, const double* A, const double* B, double* partial, int splits,
                            cudaStream_t s);
cudaError_t launch_reduce_splits(long len, int splits, const double* partial, double* C, cudaStream_t s);
// acc[i] += x[i], i < len
cudaError_t launch_add(long len, const double* x, double* acc, cudaStream_t s);
cudaError_t launch_assemble1d(int nx, int ny, int nz, const double* xs, const double* ys, const int* rmap, int nr,
                              const double* P0, const double* P1, const double* P2, double2* G, cudaStream_t s);
// 2D direct lateral synthesis
// colmax (optional, zeroed by the caller): [n / kchunk][9 nz] IEEE bits of max(|Re|, |Im|);
// amp (optional scratch, [12][n] complex): the two-kernel form (k_reflect2d, k_strengths_rows)
cudaError_t launch_strengths2d(const SynthParams& p, double2* S, cudaStream_t s, unsigned long long* colmax = nullptr,
                               long kchunk = 0, double2* amp = nullptr);
int lateral_splits(long n, int splits);  // effective split count of launch_lateral
cudaError_t launch_lateral(const CacheView& c, int nx, int ny, const double* xs, const double* ys, int ncol, const double2* S,
                           double2* partial, int splits, cudaStream_t s);
cudaError_t launch_reduce_splits2(long len, int splits, const double2* partial, double2* G, cudaStream_t s);

// batched synthesis of small observation sets (uneven batches): per item the partial sums
// of each node chunk, then a per-output sum over the chunks (2D) or sum and pixel assembly (1D)
constexpr int SYN_MAXOUT = 2304;  // partial outputs per item: 2D nx ny 9 nz, 1D nr 13 nz
constexpr int SYN_MAXPIX = 64;    // 2D pixels per item
constexpr int SYN_MAXR = 32;      // 1D distinct radii per item
constexpr int SYN_MAXZ = 8;       // z rows per item
struct SynthItem {
  SynthParams sp;          // cache view, term masks, source position, z rows (device)
  const double* xs;        // [nx] device
  const double* ys;        // [ny] device
  int nx, ny;
  int is2d;
  const double* rho;       // 1D: [nr] distinct radii (device)
  const int* rmap;         // 1D: [nx ny] pixel -> radius (device)
  int nr;
  int nw;                  // node chunks of this item
  double2* partial;        // [nw][outputs]
  double2* G;              // [nx ny nz 9] Julia layout (device)
};
size_t synth_small_smem();                                      // the largest item's
size_t synth_small_smem(int is2d, int npix, int nr, int nz);    // one item's
cudaError_t synth_small_init();  // shared-memory attribute of k_synth_small (before any capture)
// w_off[nitems + 1]: prefix of the items' chunk counts; counter zeroed before the launch;
// smem: the largest synth_small_smem(item) of the batch
cudaError_t launch_synth_small(const SynthItem* items, int nitems, const long* w_off, long nwork, unsigned* counter,
                               int chunk, int grid, size_t smem, cudaStream_t s);
// f_off[nitems + 1]: prefix of the items' finish units (2D: nx ny 9 nz, 1D: nx ny nz)
cudaError_t launch_synth_finish(const SynthItem* items, int nitems, const long* f_off, long nfin, cudaStream_t s);

// 2D lateral synthesis on the tensor cores (split-BF16, FP32 accumulation)
struct LateralTC {
  long npix, n;
  int nx, ny, ncol;
  int ctile;  // complex columns per CTA tile (≤ 128)
  int Np;     // 2 * ctile rounded up to a multiple of 16 (MMA N)
  const float2* Px;   // [n][nx]
  const float2* Py;   // [n][ny]
  const double2* S;   // [ncol][n]
  double2* partial;   // [splits][npix * ncol]
  long kchunk;        // nodes per split
  unsigned* err;      // set to nonzero if a wait timed out
};
cudaError_t launch_phase_tables(const CacheView& c, int nx, int ny, const double* xs, const double* ys, float2* Px,
                                float2* Py, cudaStream_t s);
size_t lateral_tc_smem(int Np);
int lateral_tc_ctile(int ncol);
cudaError_t launch_lateral_tc(const LateralTC& p, int splits, cudaStream_t s);

// 2D lateral synthesis on the int8 tensor cores (three base-256 digits per operand, exact
// INT32 accumulation)
struct LateralI8 {
  long npix, n;
  int nx, ny, ncol;
  int ctile;         // complex columns per column tile (≤ 80)
  int Np;            // 2 * ctile rounded up to a multiple of 16 (MMA N, ≤ 160)
  int ntile;         // column tiles
  long kchunk;       // nodes per slice: a multiple of 32, ≤ 16384
  int nchunk;        // slices = ceil(n / kchunk)
  long n_pad;        // nchunk * kchunk: node rows of the phase tables
  const float2* Px;  // [n_pad][nx], zero beyond n
  const float2* Py;  // [n_pad][ny]
  const double2* S;  // [ncol][n]
  uint8_t* Bq;       // [ntile][nchunk][kchunk/32][3 planes][Np rows x 64 B] digit images
  const unsigned long long* colmax;  // [nchunk][ncol] bits of max(|Re S|, |Im S|) (k_strengths2d)
  double2* partial;  // [nchunk][npix * ncol]
  unsigned* err;     // nonzero if a pipeline wait timed out
  long wait_limit;   // polls of each bounded pipeline wait before it gives up
};
size_t lateral_i8_stage_bytes(int Np);
size_t lateral_i8_smem(int Np);
int lateral_i8_ctile(int ncol);
cudaError_t launch_lateral_i8(const LateralI8& p, cudaStream_t s);
// even (optional, host): {x_0, dx, y_0, dy} of evenly spaced pixel coordinates: the tables by
// recurrence along each row
cudaError_t launch_phase_tables_pad(const CacheView& c, int nx, int ny, const double* xs, const double* ys, long n_pad,
                                    float2* Px, float2* Py, cudaStream_t s, const double* even = nullptr);

// 1D Bessel synthesis contraction on the int8 tensor cores: P[r][c] = Σ_k J_order(k ρ_r) C[c][k]
struct BesselI8 {
  int M, N;          // radii, real coefficient columns
  long K;            // nodes
  int order;         // Bessel order 0, 1 or 2
  int ctile, Np;     // columns per tile, ctile rounded up to 16 (MMA N ≤ 160)
  int ntile_m, ntile_n;
  long kchunk;       // nodes per slice: a multiple of 64, ≤ 16384
  int nchunk;
  const double* kr;  // [K]
  const double* rho; // [M]
  const float* C;    // [N][ldc] coefficient columns (FP32)
  long ldc;          // row stride of C: K on the per-item path; K rounded up to 4 (16-byte rows) in groups
  uint8_t* Aimg;     // [ntile_m][nchunk][kchunk/64][3][128 x 64 B]
  uint8_t* Bimg;     // [ntile_n][nchunk][kchunk/64][3][Np x 64 B]
  unsigned long long* colmax;  // [nchunk][N]
  double* partial;   // [nchunk][N][M]
  unsigned* err;
  long wait_limit;   // polls of each bounded pipeline wait before it gives up
  int aimg_ready;    // Aimg already holds this order's J_n digits (launch_bessel_i8_aimg3)
  double* kmin;      // [nchunk] smallest node of each slice (the J digits' scale, launch_slice_kmin)
  const double* rowscale;  // [nchunk][M] the J digits' scale per (slice, radius) when set (digits
                           // rint(J 8355000 / rowscale)); else j_env(kmin[z] ρ_r)
};
// complex J_n tables ([6][nr][nk]: Re J_0, Im J_0, Re J_1, ... from launch_bessel_c) into the
// int8x3 layout: rowscale[o][z][r] = max over slice z of max(|Re J_o|, |Im J_o|) at radius r
// (1 where it is 0), then for each order o and part (0 Re, 1 Im) the digit image
// img[2 o + part] in bp's A layout (ntile_m x nchunk x stages); bp gives M, K, ntile_m, kchunk,
// nchunk
cudaError_t launch_jtable_images(const BesselI8& bp, const double* Jtab, double* rowscale, uint8_t* const img[6],
                                 cudaStream_t s);
// J_0(x), J_1(x) as the int8x3 1D synthesis evaluates them (library below 25, asymptotic above)
cudaError_t launch_bessel_j01(const double* x, long n, double* J0, double* J1, cudaStream_t s);
// kmin[z] = min over slice z of kr (a slice of kchunk nodes, the last one up to K)
cudaError_t launch_slice_kmin(const double* kr, long K, long kchunk, int nchunk, double* kmin, cudaStream_t s);
// the J_0, J_1, J_2 digit images of all three orders in one pass (one Bessel evaluation per
// (ρ, k)); p gives the shared layout (M, K, ntile_m, kchunk, nchunk, kr, rho)
cudaError_t launch_bessel_i8_aimg3(const BesselI8& p, uint8_t* A0, uint8_t* A1, uint8_t* A2, cudaStream_t s);
size_t bessel_i8_stage_bytes_a();
size_t bessel_i8_stage_bytes_b(int Np);
size_t bessel_i8_smem(int Np);
int bessel_i8_ctile(int N);
cudaError_t launch_bessel_i8(const BesselI8& p, double* P, cudaStream_t s);

// ------------------------------------------------------------------------------------
// Grouped 1D int8x3 synthesis: the items of a batch (each a 1D cache of real nodes with its
// own radii, heights and output) through one launch per stage for the whole group. A
// stage's blocks are the concatenation of every item's (or every (item, order) entry's)
// blocks; `first[e]` is the first block of entry e (first[ne] = the grid), and a block finds
// its entry by binary search.
// ------------------------------------------------------------------------------------
struct Synth1DItem {
  SynthParams sp;          // the item's node data (real nodes), term masks, heights (device)
  double2* amp;            // [12][nk] reflected amplitudes
  float* C;                // [26 nz][ldc] coefficient columns: orders 0, 1, 2 at rows 0, 10 nz, 18 nz
  long ldc;                // row stride of C: nk rounded up to 4, so every row starts on 16 bytes
  int nx, ny, nr;          // pixel grid, distinct radii
  const double* xs;        // [nx] device
  const double* ys;        // [ny] device
  const int* rmap;         // [nx ny] pixel -> radius index
  double2* G;              // [nx][ny][nz][3][3] output (Julia's column-major layout)
  int nchunk;              // node slices of the contraction
  long kchunk;             // nodes per slice (a multiple of 64)
  double dz;               // spacing of evenly spaced heights (to 4 ulp), else 0
  const double* part[3];   // [nchunk][N_o][nr] slice partials of order o (N_0 = 10 nz, N_1 = N_2 = 8 nz)
};
// every stage of the group, in order, on stream s; `it`/`bp` and the `first_*` tables are
// device arrays (bp: 3 entries per item, orders 0, 1, 2; bp[3i] also carries the layout of
// item i's J_n images). Host copies (ni, grid sizes) come in `grid`: {reflect, coef, aimg,
// bimg, gemm, assemble, slice minima}.
struct Synth1DGroup {
  int ni;
  const Synth1DItem* it;
  const BesselI8* bp;
  const long* first_reflect;   // [ni + 1]
  const long* first_coef;      // [ni + 1]
  const long* first_aimg;      // [ni + 1]
  const long* first_bimg;      // [3 ni + 1]
  const long* first_gemm;      // [3 ni + 1]
  const long* first_asm;       // [ni + 1]
  const long* first_kmin;      // [ni + 1]
  long grid[7];
};
// the entry whose block range holds block b: the last e with first[e] <= b (first ascending)
__device__ __forceinline__ int group_entry(const long* first, int ne, long b) {
  int lo = 0, hi = ne;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (first[mid] <= b) lo = mid;
    else hi = mid;
  }
  return lo;
}
// stage 0: reflected amplitudes, 1: FP32 coefficient columns
cudaError_t launch_reflect_coef_group(const Synth1DGroup& g, int stage, cudaStream_t s);
// stage 0: slice minima and J_n digit images, 1: coefficient digit images with their slice
// maxima, 2: contraction
cudaError_t launch_bessel_i8_group(const Synth1DGroup& g, int stage, cudaStream_t s);
cudaError_t launch_assemble1d_group(const Synth1DGroup& g, cudaStream_t s);    // slice sum + pixel assembly
constexpr int COEF1D_ZB_GROUP = 8;   // heights per thread of the grouped coefficient kernel

// Gauss-Legendre panels -> nodes/weights, bit-exact with the CPU restatement
cudaError_t launch_gl_nodes(int npanels, const double* pa, const double* pb, const int* sing_side, const double* xi,
                            const double* wx, int order, double* nodes, double* wts, cudaStream_t s);

}  // namespace ytf

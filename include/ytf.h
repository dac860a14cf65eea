/* ytf.h -- C ABI of libytf, the B200 (sm_100a) implementation of YellowThinFilms'
 * spectral Green's-function path: per-k-node Berreman mode solve, S-matrix cascade and
 * cavity transfer maps, Sommerfeld k-quadrature nodes, and the synthesis of
 * G(ρ, z, z') on a lateral grid.
 *
 * Conventions
 *   - Every entry point returns an int status: YTF_OK (0) or a YTF_ERR_* code; the
 *     message is in ytf_last_error(ctx). No C++ exception crosses this boundary.
 *   - Layer indices are 1-based, as in the reference's Julia API (source_layer,
 *     obs_layers, obs_layer). The last layer is semi-infinite and hosts no source.
 *   - Complex arrays are interleaved (re, im) doubles. 3x3 tensors are column-major
 *     (Julia's order). Output G has Julia's Array{ComplexF64,5} layout
 *     (Nx, Ny, Nz, 3 field components, 3 moments), column-major.
 *   - Node, weight and coordinate inputs are host pointers (copied). `out` of
 *     ytf_green is a host pointer unless out_is_device != 0.
 *   - Calls are synchronous on the context's stream (ytf_ctx_set_stream).
 *   - One context per host thread; handles are owned by the library and freed by the
 *     matching *_destroy.
 *   - Per-node numerical failures are data (valid / Tvalid / status arrays), never
 *     errors, as in the reference (mod_CavityTransfer.jl:226-251).
 */
#ifndef YTF_H
#define YTF_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ytf_ctx ytf_ctx;
typedef struct ytf_stack ytf_stack;
typedef struct ytf_cache ytf_cache;

enum {
  YTF_OK = 0,
  YTF_ERR_ARG = 1,   /* argument error; message mirrors the reference's `error(...)` text */
  YTF_ERR_CUDA = 2,  /* CUDA runtime error (no device, launch failure, ...) */
  YTF_ERR_NOMEM = 3, /* device allocation failed */
  YTF_ERR_STATE = 4  /* handle used with the wrong context or kind */
};
/* `terms` of closed_form_G (mod_ClosedFormField.jl:143-160) */
enum { YTF_TERMS_ALL = 0, YTF_TERMS_DIRECT = 1, YTF_TERMS_SCATTERED = 2, YTF_TERMS_TOEPLITZ = 3, YTF_TERMS_HANKEL = 4 };
/* arithmetic of the synthesis contraction */
enum { YTF_PREC_FP64 = 0, YTF_PREC_SPLIT_BF16 = 1, YTF_PREC_INT8X3 = 2 };
/* `rotation` of build_cavity_transfer_2d (mod_CavityTransfer.jl:307-318) */
enum { YTF_ROT_AUTO = -1, YTF_ROT_OFF = 0, YTF_ROT_ON = 1 };
/* material kinds (the reference's material TYPES, mod_ModeSolver.jl:28-65) */
enum { YTF_ISOTROPIC = 0, YTF_UNIAXIAL = 1, YTF_BIAXIAL = 2, YTF_GENERAL = 3 };

int ytf_version(void);

/* Context: one CUDA device and stream, plus the library's reusable device workspace. */
int ytf_ctx_create(ytf_ctx** out, int device);
int ytf_ctx_destroy(ytf_ctx* ctx);
int ytf_ctx_set_stream(ytf_ctx* ctx, void* cuda_stream);

/* Polls of each bounded mbarrier wait inside the int8 tensor-core pipelines (the Bessel and
 * lateral contractions) before the wait gives up; 0 restores the default 2^22 (about a
 * second). No counterpart in the reference (its loops have no waits). A wait that runs out
 * ends its kernel early without touching its output: the kernel lets its issued copies and
 * MMAs finish, releases its tensor memory and sets an error word, and the call returns
 * YTF_ERR_CUDA with "a tensor-core pipeline wait timed out"; the context stays usable.
 * Tests set a tiny limit to drive that path. */
int ytf_ctx_set_wait_limit(ytf_ctx* ctx, long polls);
/* Workspace bound, in bytes, of one group of ytf_green_batch's grouped 1D int8x3 synthesis
 * (about 14 KB per node at 64 heights); 0 restores the default 4 GiB. No counterpart in the
 * reference. A smaller bound gives more groups (more launches), never a different item set. */
int ytf_ctx_set_group_bytes(ytf_ctx* ctx, long bytes);
int ytf_ctx_sync(ytf_ctx* ctx);
const char* ytf_last_error(const ytf_ctx* ctx);

/* Per-kernel accounting of this library's own launches (no counterpart in the reference;
 * it serves the measurement). ytf_ctx_profile resets the counters and turns CUDA-event
 * timing of every launch on the context's stream on or off. ytf_ctx_profile_read
 * returns, per kernel name (32-byte slots), the summed event time (ms) and the number
 * of launches since the reset; *n receives the number of distinct kernels. */
int ytf_ctx_profile(ytf_ctx* ctx, int enable);
int ytf_ctx_profile_read(ytf_ctx* ctx, int max_entries, char* names, double* total_ms, long* launches, int* n);

/* Stack (replaces Vector{<:AbstractLayer} of FlatOpticalLayer / FlatLayer,
 * mod_ModeSolver.jl:71-80). eps, mu: nL x 9 complex, column-major 3x3; mu may be NULL
 * (μ = 1, FlatOpticalLayer); mu_kind may be NULL (isotropic). */
int ytf_stack_create(ytf_ctx* ctx, int nL, const int* eps_kind, const int* mu_kind, const double* eps,
                     const double* mu, const double* d, ytf_stack** out);
int ytf_stack_destroy(ytf_stack* stack);

/* build_cavity_transfer_1d(stack, ω, source_layer, kx_nodes, wt_nodes; obs_layers,
 * check_symmetry) (mod_CavityTransfer.jl:196-258). obs_layers == NULL means 1:nL. */
int ytf_transfer_1d(ytf_ctx* ctx, const ytf_stack* stack, double omega, int source_layer, int nk,
                    const double* kx_nodes, const double* wt_nodes, int nobs, const int* obs_layers,
                    int check_symmetry, ytf_cache** out);

/* build_cavity_transfer_2d(stack, ω, source_layer, kρ, wρ, φ, wφ; obs_layers, rotation)
 * (mod_CavityTransfer.jl:307-398). Nodes are (kρ_k, φ_p), flat index k + nkr * p. */
int ytf_transfer_2d(ytf_ctx* ctx, const ytf_stack* stack, double omega, int source_layer, int nkr,
                    const double* kr_nodes, const double* kr_weights, int nphi, const double* phi_nodes,
                    const double* phi_weights, int nobs, const int* obs_layers, int rotation, ytf_cache** out);

int ytf_cache_destroy(ytf_cache* cache);

/* Sizes of a cache: flat node count, obs layers (up to 32), 2D flag, rotation flag. */
int ytf_cache_info(const ytf_cache* cache, long* n_nodes, int* n_obs, int* obs_layers, int* is2d, int* rotation);

/* valid[k] and Tvalid[o][k] of CavityTransferCache1D/2D (mod_CavityTransfer.jl:160-178),
 * plus the per-node status bit mask (1 valid, 2 eigen non-convergence, 4 mode-sort
 * overflow, 8 singular solve, 16 non-finite seeds, 32 non-finite T). Host buffers;
 * any may be NULL. tvalid is [n_obs][n_nodes]. */
int ytf_cache_status(ytf_ctx* ctx, const ytf_cache* cache, unsigned char* valid, unsigned char* tvalid,
                     unsigned char* status);

/* The cache's per-node arrays (CavityTransferCache1D/2D fields T, Qf_src, Qb_src, sf,
 * sb, basis), host buffers, any may be NULL: T [n_obs][n][4x4 col-major], Qf/Qb [n][2],
 * sf/sb [n][2x3 col-major], basis [n_obs][n][8 fields x 2 modes] in the order
 * Exf Eyf Ezf Exb Eyb Ezb KZf KZb. All complex. */
int ytf_cache_export(ytf_ctx* ctx, const ytf_cache* cache, double* T, double* Qf, double* Qb, double* sf, double* sb,
                     double* basis);

/* _cavity_response(stack, ω, s, kρ, φ) (mod_KSpaceFeatures.jl:109-127) at n values of kρ
 * (host arrays): the largest singular value of the source-layer reflections RL, RR and,
 * below the top layer, of the cavity resolvent (I - ΦF RL ΦB RR)^-1; 0 where the node
 * solve fails or is not finite. The pole scan of kspace_features evaluates it on a
 * logarithmic kρ grid; one call solves all n nodes on the device. */
int ytf_cavity_response(ytf_ctx* ctx, const ytf_stack* stack, double omega, int source_layer, long n,
                        const double* kr, double phi, double* out);

/* ytf_cavity_response for many (stack, ω, source layer) items with one synchronisation
 * (_cavity_response, mod_KSpaceFeatures.jl:109-127, per item): item i's counts[i] kρ values
 * are kr[o_i : o_i + counts[i]] with o_i = counts[0] + ... + counts[i-1]; its responses go to
 * the same places of out. The exact window sampling of the learned node placement calls it
 * once for all problems. An argument error names the item. */
int ytf_cavity_response_batch(ytf_ctx* ctx, int nitems, const ytf_stack* const* stacks, const double* omega,
                              const int* source_layer, const long* counts, const double* kr, double phi, double* out);

/* build_cavity_transfer_1d on a deformed integration contour: complex nodes kρ = k_re + i k_im
 * with complex weights (w_re + i w_im), e.g. kρ(t) = t - i h s(t) with s(0) = s(L) = 0 below
 * the real axis. No counterpart in the reference, whose rules stay on the real axis
 * (mod_KxGrid.jl:361-394); with lossy layers every pole and branch point lies above the real
 * axis, so by Cauchy's theorem the contour integral equals the real-axis one with the same
 * end points. Azimuthally symmetric (closed-form) stacks only, as the 1D path; the mode
 * solve, S-matrices and projections are the analytic continuation in kρ (principal square
 * roots: ω²ε - kρ² stays in the upper half plane below the axis). closed_form_G on such a
 * cache uses complex J_n(kρ ρ) in an FP64 contraction (INT8X3 falls back to it). */
int ytf_transfer_1d_contour(ytf_ctx* ctx, const ytf_stack* stack, double omega, int source_layer, int nk,
                            const double* k_re, const double* k_im, const double* w_re, const double* w_im, int nobs,
                            const int* obs_layers, ytf_cache** out);

/* J_0(x) and J_1(x) of real x exactly as the int8x3 1D synthesis evaluates them for its J
 * digit images: the CUDA math library's j0/j1 below |x| = 25, Hankel's asymptotic expansions
 * with one shared phase above (absolute error below 1e-12). For tests and callers that want
 * the same values; no counterpart in the reference (SpecialFunctions.besselj). */
int ytf_bessel_j01(ytf_ctx* ctx, long n, const double* x, double* j0, double* j1);

/* J_order(z) (order 0, 1, 2) at n complex points z = z_re + i z_im, evaluated by the device
 * functions of the contour synthesis (power series, Miller recurrence, Hankel expansion). */
int ytf_bessel_j(ytf_ctx* ctx, int order, long n, const double* z_re, const double* z_im, double* out_re,
                 double* out_im);

/* layer_light_lines(layer, ω, φ) (mod_KxGrid.jl:41-59) of one layer given as raw arrays
 * (column-major 3x3 ε and μ, interleaved re/im; mu NULL = identity): up to 2 values into
 * out (ascending), their count in *n. Host arithmetic; needs no context or GPU. */
int ytf_layer_light_lines(const double* eps, const double* mu, double omega, double phi, double* out, int* n);

/* Parameters of the point rule (kspace_features dims=1 + fixed_kρ_rule). */
typedef struct {
  double h_min;        /* smallest |z - z'| (or source-image distance) to resolve: Kcut >= target_decay / h_min */
  double rho_max;      /* largest lateral distance (flat-region width 4 / rho_max); 0: none */
  double target_decay; /* e-folds of evanescent decay at the cut (the reference's 25) */
  double kr_cap;       /* absolute cap on Kcut; 0: 1e5 x the largest light line */
  int scan;            /* 1: scan the real axis for guided-mode poles (log step 1e-3) */
  int order;           /* Gauss-Legendre order per panel (8) */
  double rtol;         /* relative accuracy the pole panels are sized for (1e-6) */
} ytf_grid_params;

#define YTF_GRID_MAX_POLES 256
#define YTF_GRID_MAX_LINES 64
typedef struct {
  double Kcut, kmax;
  long n_panels;
  int n_poles, n_light_lines;
  double poles[YTF_GRID_MAX_POLES][2]; /* (q, Γ) of the first poles found */
  double light_lines[YTF_GRID_MAX_LINES];
  double* panels;   /* optional, set by the caller: receives the panels (a, b) pairs ... */
  long panels_cap;  /* ... when panels_cap >= n_panels */
} ytf_grid_info;

/* point_kx_grid (mod_ClosedFormGrid.jl:381-424) with the :fixed engine: kspace_features for
 * a point rule at φ = 0 (light lines of every layer, Kcut, the real-axis pole scan of the
 * source layer's cavity response (mod_KSpaceFeatures.jl:151-204) with golden-section peaks
 * and half-power widths, clusters) and fixed_kρ_rule (:396-419): graded panels between the
 * light lines, u² substitution at the half-space light lines, Gauss-Legendre nodes. The
 * cavity response is evaluated on the device (ytf_cavity_response), the panels on the host,
 * the nodes by ytf_gl_rule. k = w = NULL: size query (*n, info). cap: capacity of k and w. */
int ytf_nodes_1d(ytf_ctx* ctx, const ytf_stack* stack, double omega, int source_layer, const ytf_grid_params* params,
                 long cap, double* k, double* w, long* n, ytf_grid_info* info);

/* The same rule with the real-axis poles (q, Γ) given by the caller instead of scanned (the
 * learned node placement proposes them): light lines, Kcut, clusters of the given poles,
 * fixed_kρ_rule panels, Gauss-Legendre nodes. No counterpart in the reference, whose
 * kspace_features always scans (mod_KSpaceFeatures.jl:295-360). */
int ytf_nodes_from_poles(ytf_ctx* ctx, const ytf_stack* stack, double omega, int source_layer,
                         const ytf_grid_params* params, int npoles, const double* q, const double* G, long cap,
                         double* k, double* w, long* n, ytf_grid_info* info);

/* The panels of ytf_nodes_1d (scan = 0: no pole knowledge, npoles[j] < 0) or of
 * ytf_nodes_from_poles (npoles[j] >= 0 poles) for many 1D problems at once, on the host
 * threads: problem j has stacks[j], omega[j], source_layer[j], prm[j] and its poles at
 * q/G[sum of the earlier npoles (negative counted as 0) ...]. counts[j] receives its panel
 * count and panels (pairs a, b) receive every problem's panels in problem order. *total is
 * the sum; when it exceeds cap (panel pairs) nothing is written and YTF_ERR_ARG returned, so
 * the caller can retry with a larger buffer. Each problem's panels equal its own call's
 * (ytf_grid_info.panels). No counterpart in the reference (one grid per call). */
int ytf_rule_panels_batch(ytf_ctx* ctx, int nprob, const ytf_stack* const* stacks, const double* omega,
                          const int* source_layer, const ytf_grid_params* prm, const int* npoles, const double* q,
                          const double* G, long cap, double* panels, long* counts, long* total);

/* The peak rule of real_axis_poles (mod_KSpaceFeatures.jl:151-204) on sampled responses,
 * without its refinement rounds: for each of nwin log-uniform grids of npts points (ks,
 * logR: nwin x npts, row-major) the local maxima at or above max + log(floor_rel) that stand
 * `prominence` (log) above the higher valley within a factor 4 in k, positioned by a
 * parabola in log k, with Γ from the nearer half-power crossing. counts[w] peaks per window;
 * their (q, Γ) concatenated into q, G (capacity cap; q = G = NULL: counting only), *total
 * peaks in all. Host arithmetic; needs no context. The learned node placement reads the
 * exact windows it samples around the network's candidates through it. */
int ytf_peaks_batch(int nwin, int npts, const double* ks, const double* logR, double prominence, double floor_rel,
                    long cap, int* counts, double* q, double* G, long* total);

/* adaptive_seeds(kspace_features(...; dims=1); rtol) (mod_KSpaceFeatures.jl:421-445): the
 * starting breakpoints of the reference's adaptive engine for a point rule -- light lines,
 * geometric grading L (1 ± 2^-j), j = 1..min(50, ceil(2 log2(10/rtol))), onto the half-space
 * light lines, each pole cluster's [a - 4Γ, a, b, b + 4Γ], and 2 kmax, 4 kmax, ... below Kcut --
 * sorted and unique within (0, Kcut). The features (and the pole scan, if params->scan) as
 * ytf_nodes_1d. seeds = NULL: size query. */
int ytf_adaptive_seeds(ytf_ctx* ctx, const ytf_stack* stack, double omega, int source_layer,
                       const ytf_grid_params* params, long cap, double* seeds, long* n);

/* point_kρ_grid_2d (mod_ClosedFormGrid.jl:536-585) with the :fixed engine and an explicit
 * h_min: kspace_features with dims = 2 (mod_KSpaceFeatures.jl:295-360) -- the scanned
 * directions (φ = 0 for an azimuthally symmetric stack; N_φ_scan/4 + 1 over [0, π/2] when
 * every tensor is diagonal; N_φ_scan over [0, 2π) otherwise), light lines at every scanned
 * direction, the pole scan along each of them on the device, clusters merged at the φ step,
 * N_φ from the lateral factor (2.5 Kcut ρ_max) and the pole tracks (_pole_track_η, :243-259),
 * at least 64, even -- then fixed_kρ_rule: one kρ rule shared by every φ. Returns the kρ
 * nodes/weights as ytf_nodes_1d and in *n_phi the size of the uniform φ trapezoid
 * (build_kphi_grid: φ_p = 2π p / N_φ, weights 2π / N_φ). k = w = NULL: size query. */
int ytf_nodes_2d(ytf_ctx* ctx, const ytf_stack* stack, double omega, int source_layer, const ytf_grid_params* params,
                 int n_phi_scan, long cap, double* k, double* w, long* n, long* n_phi, ytf_grid_info* info);

/* One problem of a batched transfer build: the arguments of build_cavity_transfer_1d
 * (is2d = 0: k_nodes/k_weights are kx nodes and weights, check_symmetry applies) or of
 * build_cavity_transfer_2d (is2d = 1 or nphi > 0: kρ nodes/weights and φ nodes/weights,
 * rotation applies). */
typedef struct {
  const ytf_stack* stack;
  double omega;
  int source_layer;
  int nk;
  const double* k_nodes;
  const double* k_weights;
  int nphi;
  const double* phi_nodes;
  const double* phi_weights;
  int nobs;
  const int* obs_layers; /* NULL or nobs <= 0: every layer */
  int check_symmetry;
  int rotation;          /* YTF_ROT_* */
  int is2d;
  int nodes_on_device;   /* 1D items: k_nodes/k_weights are device pointers (this context's GPU),
                            read on the context's stream during the call (e.g. from
                            ytf_gl_rule_batch_device); not accepted by ytf_plan_create */
} ytf_transfer_desc;

/* Many independent builds (stacks, frequencies, source layers, grids of any sizes) in one
 * call: out[i] is the cache build_cavity_transfer_1d/2d(desc[i]) would return, bit for bit.
 * The reference builds one cache per call and threads over the nodes inside it
 * (mod_CavityTransfer.jl:224, :330); its callers loop over stacks and frequencies
 * (e.g. chunked_2d, mod_ClosedFormGrid.jl:457-467). Here the node solves of all items run
 * in the same kernel launches (grouped under a 6 GiB scratch budget); azimuthally symmetric
 * 2D items with rotation take the rotation path. Argument errors name the item; on any
 * error no cache is returned. */
int ytf_transfer_batch(ytf_ctx* ctx, int nb, const ytf_transfer_desc* desc, ytf_cache** out);

/* One item of ytf_green_batch: the arguments of ytf_green. */
typedef struct {
  const ytf_cache* cache;
  int obs_layer;
  double zsrc_local;
  int nz;
  const double* z_obs;
  int nx;
  const double* xs;
  int ny;
  const double* ys;
  int terms;
  int precision;
  double* out;
  int out_is_device;
} ytf_green_desc;

/* closed_form_G(cache, obs_layer, zsrc_local, z_obs, xs, ys; terms)
 * (1D: mod_ClosedFormField.jl:435-487; 2D, lateral=:direct: :711-753). out: Nx*Ny*Nz*9
 * complex, Julia layout. precision: YTF_PREC_FP64 (CUDA-core FP64 contraction),
 * YTF_PREC_SPLIT_BF16 (tensor-core contraction, split-BF16 operands, FP32 accumulation) or
 * YTF_PREC_INT8X3 (int8 tensor-core contraction: operands in three fixed-point base-256
 * digits, exact INT32 accumulation). INT8X3 applies to the 2D lateral sum and to the 1D Bessel
 * contraction (J_n(kρ) and the coefficient columns in digits; on a deformed contour the complex
 * J_n's real and imaginary parts, two contractions per order); SPLIT_BF16 to the 2D lateral
 * sum only (1D: FP64). */
int ytf_green(ytf_ctx* ctx, const ytf_cache* cache, int obs_layer, double zsrc_local, int nz, const double* z_obs,
              int nx, const double* xs, int ny, const double* ys, int terms, int precision, double* out,
              int out_is_device);

/* closed_form_G over many (cache, observation set) items with one synchronisation: the
 * same results as ytf_green per item, in order, on the context's stream; the coordinates of
 * all items go up in one copy and the items' kernels queue back to back. 1D items of real
 * nodes (at most 1048576) at YTF_PREC_INT8X3 are synthesised together, seven launches per
 * group of items (ytf_ctx_set_group_bytes): each such item's G equals ytf_green's to the
 * int8x3 tolerance (the contraction's node slices, and so the slices' fixed-point scales,
 * differ); every other item's G is ytf_green's bit for bit. The reference
 * calls closed_form_G once per cache (mod_ClosedFormField.jl:435, :711); its callers loop
 * (e.g. build_closed_form_green, mod_ClosedFormAssembly.jl:114). */
int ytf_green_batch(ytf_ctx* ctx, int nb, const ytf_green_desc* desc);

/* FastGaussQuadrature.gausslegendre(n) (used at mod_KxGrid.jl:362): ascending nodes on
 * [-1, 1] and weights, correctly rounded. */
int ytf_gauss_legendre(int n, double* x, double* w);

/* gl_rule(panels; order, singular) (mod_KxGrid.jl:361-384), expanded on the device:
 * composite Gauss-Legendre with the u² substitution on panels that end on a singular
 * value. nodes/weights: npanels*order, host buffers. Bit-exact with an IEEE-double CPU
 * evaluation of the same expressions. */
int ytf_gl_rule(ytf_ctx* ctx, int npanels, const double* pa, const double* pb, int order, int nsing,
                const double* singular, double* nodes, double* weights);

/* ytf_gl_rule for many panel sets with one synchronisation (gl_rule, mod_KxGrid.jl:361-384,
 * per set): set j has npanels[j] panels (pa, pb concatenated over the sets) and nsing[j]
 * singular points (concatenated likewise); its npanels[j] x order nodes and weights go to the
 * same places of nodes and weights. Every set's rule equals its own ytf_gl_rule call. */
int ytf_gl_rule_batch(ytf_ctx* ctx, int nsets, const int* npanels, const double* pa, const double* pb, int order,
                      const int* nsing, const double* singular, double* nodes, double* weights);

/* ytf_gl_rule_batch with the nodes and weights left in device memory: d_nodes/d_weights are
 * device pointers (this context's GPU, npanels-sum x order doubles each), written on the
 * context's stream; the call returns without synchronising, so work queued after it on that
 * stream (ytf_transfer_batch with nodes_on_device) sees the rule. No counterpart in the
 * reference. */
int ytf_gl_rule_batch_device(ytf_ctx* ctx, int nsets, const int* npanels, const double* pa, const double* pb, int order,
                             const int* nsing, const double* singular, double* d_nodes, double* d_weights);

/* Allocation-free variant of ytf_green for 2D caches (no counterpart in the reference).
 * For callers that must not have the library allocate device memory: a host that owns all
 * device memory through its own pool (e.g. a Julia CUDA.jl session or a caching
 * allocator), or code that cannot afford cudaMalloc's device-wide synchronisation. The
 * strengths and the split-k partial sums use a fixed 64 MiB array inside the library
 * (held on every GPU that loads it until exit) instead of cudaMalloc'd workspace. Limit:
 * 9*nz*(n_nodes + nx*ny) <= 4,194,304 complex values; larger requests return YTF_ERR_ARG.
 * z_obs_dev, xs_dev, ys_dev and out_dev are DEVICE pointers (out: nx*ny*nz*9 complex,
 * Julia layout). As ytf_green: an empty grid returns YTF_OK, an empty rule writes zeros.
 * The first call on a device looks up the array's device address and keeps it for the life
 * of the process; make that first call before any stream capture, and do not call this entry
 * point on a device after cudaDeviceReset (the kept address is then stale). The call
 * synchronises the context's stream before it returns. All calls share the array: calls that
 * overlap on the GPU (other streams, other host threads) race and must be serialised by the
 * caller. */
int ytf_green_noalloc(ytf_ctx* ctx, const ytf_cache* cache, int obs_layer, double zsrc_local, int nz,
                      const double* z_obs_dev, int nx, const double* xs_dev, int ny, const double* ys_dev, int terms,
                      double* out_dev);

/* ---------------------------------------------------------------------------------------
 * Uneven-batch plans. No counterpart in the reference, whose callers loop over stacks,
 * frequencies and grids, one build_cavity_transfer_1d/2d and one closed_form_G per item
 * (mod_CavityTransfer.jl:224, :330; mod_ClosedFormField.jl:435, :711; e.g. chunked_2d,
 * mod_ClosedFormGrid.jl:457-467). A plan takes nb (transfer, green) item pairs, allocates
 * everything once and records the whole computation as one CUDA graph: the upload of every
 * item's nodes and coordinates, the node solve as persistent kernels that pull tiles of
 * (item, nodes) from a device counter (scratch reused pass by pass under 6 GiB), the
 * synthesis of every item's G (FP64, node chunks of all items as the work units of one
 * persistent kernel), and the download of the host outputs. ytf_plan_run stages the inputs
 * and launches the graph; ytf_plan_wait synchronises and delivers the host outputs.
 *
 * Item i: tr[i] as for ytf_transfer_batch (rotation is ignored: 2D items take the full (kρ, φ)
 * solve, which the rotation reproduces to rounding) and gr[i] as for ytf_green_batch, where
 * gr[i].cache is ignored (item i synthesises from the cache of tr[i]). Small observation sets
 * (nz <= 8, 2D nx*ny <= 64 and 9*nz*nx*ny <= 2304, FP64) share one batched synthesis kernel;
 * other 2D items run closed_form_G's own kernels (any precision) inside the same graph, from
 * workspaces the plan owns (sized by one eager pass at creation). 1D items must be small
 * sets: FP64, nz <= 8, at most 32 distinct radii and 13*nz*(distinct radii) <= 2304, real
 * nodes. The descriptors' host arrays are read again by every ytf_plan_run (their sizes, and
 * for 1D items the pattern of equal radii, are fixed at creation) and gr[i].out receives G at
 * ytf_plan_wait (from the graph itself when it is device memory (out_is_device) or page-locked
 * host memory). Results: the caches equal
 * ytf_transfer_batch's bit for bit; G equals ytf_green_batch's bit for bit for the large 2D
 * items and to rounding for the small sets (the node sums run in another order). */
typedef struct ytf_plan ytf_plan;
typedef struct {
  int block;             /* threads per CTA of the persistent node-solve kernels: 128 or 256 */
  int ctas_per_sm;       /* node-solve grid: ctas_per_sm x SM count (1..32) */
  int tile;              /* units per node-solve tile (nodes; (node, layer) pairs for the mode solve) */
  int chunk;             /* nodes per synthesis work unit (multiple of 16) */
  int synth_ctas_per_sm; /* synthesis grid: synth_ctas_per_sm x SM count (1..8) */
} ytf_tune;
/* tune NULL: block 128, 4 CTAs per SM, tile 1024, chunk 2048, 2 synthesis CTAs per SM */
int ytf_plan_create(ytf_ctx* ctx, int nb, const ytf_transfer_desc* tr, const ytf_green_desc* gr,
                    const ytf_tune* tune, ytf_plan** out);
/* re-record the graph with other tiles (the caches, scratch and staging are kept) */
int ytf_plan_retune(ytf_plan* plan, const ytf_tune* tune);
int ytf_plan_run(ytf_plan* plan);
/* device_ms (optional): CUDA-event time of the last run's graph on the context's stream */
int ytf_plan_wait(ytf_plan* plan, float* device_ms);
/* the cache of item i (owned by the plan, valid until ytf_plan_destroy; do not destroy it) */
int ytf_plan_cache(const ytf_plan* plan, int item, const ytf_cache** out);
/* nodes of all items, node-solve passes, kernel launches per run, bytes staged in and out */
int ytf_plan_info(const ytf_plan* plan, long* nodes, int* passes, int* kernels, long* h2d_bytes, long* d2h_bytes);
int ytf_plan_destroy(ytf_plan* plan);

/* ---------------------------------------------------------------------------------------
 * The small MLP of the learned node placement. No counterpart in the reference: the
 * reference places quadrature nodes from a pole scan of solved responses
 * (mod_KSpaceFeatures.jl:151-204); this network predicts the scanned quantity (the log
 * cavity response and a pole-proximity score) from a stack descriptor, the frequency and k,
 * so a node placement can be proposed without the scan. Every proposed node is still solved
 * exactly by the transfer path, which is also the fallback.
 *
 * sizes[0..nlayers]: layer widths (input features first, 2 outputs last); GELU between
 * layers; FP32 master parameters, BF16 weights in every product, FP32 accumulation.
 * Parameter vector: for each layer W [out x in] row-major, then b [out]. Loss: mean squared
 * error of output 0 plus the logistic loss of output 1 (targets T: [B][2]). Inputs X: [B][n0]
 * row-major float. ytf_mlp_train takes DEVICE pointers to a resident training set (n
 * samples) and runs `steps` Adam steps (β = 0.9, 0.999) on mini-batches drawn on the device
 * from a seeded hash; losses[steps] (optional) receives the mini-batch losses. */
typedef struct ytf_mlp ytf_mlp;
int ytf_mlp_create(int device, int nlayers, const int* sizes, unsigned long long seed, ytf_mlp** out);
int ytf_mlp_destroy(ytf_mlp* net);
const char* ytf_mlp_last_error(const ytf_mlp* net);
long ytf_mlp_num_params(const ytf_mlp* net);
int ytf_mlp_set_stream(ytf_mlp* net, void* stream);
int ytf_mlp_params(ytf_mlp* net, float* get, const float* set);
int ytf_mlp_forward(ytf_mlp* net, int B, const float* X, float* out, int on_device);
int ytf_mlp_gradients(ytf_mlp* net, int B, const float* X, const float* T, float* grad, float* loss, int on_device);
int ytf_mlp_train(ytf_mlp* net, long n, const float* X, const float* T, int batch, int steps, float lr,
                  unsigned long long seed, float* losses);

#ifdef __cplusplus
}
#endif

#endif /* YTF_H */

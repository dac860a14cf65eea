// ytf_capi.cu -- the C ABI of libytf (include/ytf.h): handles, argument checks with the
// reference's error messages, device workspace, and the host-side orchestration of the
// transfer and synthesis kernels.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/ytf.h"
#include "ytf_kernels.h"
#include "ytf_grid.h"

using namespace ytf;

struct ProfSpan {
  const char* name;
  cudaEvent_t a, b;
};

struct ytf_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::map<std::string, std::pair<void*, size_t>> ws;  // grow-only device workspace
  std::multimap<size_t, void*> pool;                   // released cache blocks, by size
  int refs = 0;                                        // live stacks and caches
  bool closing = false;
  // per-kernel accounting: launches always, CUDA-event time when profiling is on
  bool prof = false;
  std::vector<ProfSpan> spans;
  std::vector<cudaEvent_t> free_events;
  std::map<std::string, std::pair<double, long>> ktime;  // name -> (ms, timed launches)
  std::map<std::string, long> klaunch;                   // name -> launches
  void* pinned = nullptr;                                // page-locked staging of batched uploads
  size_t pinned_bytes = 0;
  cudaEvent_t stage_ev = nullptr;                        // last copy out of the staging block
  // plan recording: the first (eager) pass notes every workspace request's largest size by
  // name; the captured pass is served from the plan's own buffers of those sizes
  std::map<std::string, size_t>* ws_record = nullptr;
  std::map<std::string, std::pair<void*, size_t>>* ws_override = nullptr;
  // side streams of ytf_green_batch: the items of an all-1D batch run round-robin on them,
  // each slot with its own workspace (names suffixed "#<slot>" while ws_slot > 0)
  std::vector<cudaStream_t> slot_streams;
  std::vector<cudaEvent_t> slot_events;
  int ws_slot = 0;
  // polls of each bounded mbarrier wait in the int8 tensor-core pipelines before it gives up
  // (ytf_ctx_set_wait_limit)
  long wait_limit = 1L << 22;
  // workspace bound of one group of the grouped 1D int8x3 synthesis (ytf_ctx_set_group_bytes)
  size_t group_bytes = (size_t)4 << 30;
  ~ytf_ctx() {
    for (auto s : slot_streams) cudaStreamDestroy(s);
    for (auto e : slot_events) cudaEventDestroy(e);
    if (stage_ev) cudaEventDestroy(stage_ev);
    if (pinned) cudaFreeHost(pinned);
    for (auto& kv : ws) cudaFree(kv.second.first);
    for (auto& kv : pool) cudaFree(kv.second);
    for (auto& sp : spans) { cudaEventDestroy(sp.a); cudaEventDestroy(sp.b); }
    for (auto e : free_events) cudaEventDestroy(e);
  }
};

struct ytf_stack {
  ytf_ctx* ctx;
  int nL;
  std::vector<LayerDev> host;
  LayerDev* dev = nullptr;
};

struct ytf_cache {
  ytf_ctx* ctx;
  const ytf_stack* stack_ref = nullptr;
  int nL, src, nobs;
  int obs[MAXL];
  bool is2d = false, rotation = false;
  int Nk = 0, Np = 1;
  long n = 0;
  double omega = 0, d_src = 0;
  std::vector<double> kr, wr, phi, wphi, d_layer;
  std::vector<double> kri, wri;  // imaginary parts of 1D nodes/weights on a deformed contour (else empty)
  // 1D nodes handed over in device memory (ytf_transfer_desc.nodes_on_device): kr/wr stay
  // empty and the build copies them device to device from these (valid during the build call)
  const double* src_kr = nullptr;
  const double* src_wr = nullptr;
  void* block = nullptr;  // one device allocation for every array below
  size_t block_bytes = 0;
  double *d_kr = nullptr, *d_wr = nullptr, *d_phi = nullptr, *d_wphi = nullptr;
  double *d_kri = nullptr, *d_wri = nullptr;
  uint8_t *d_status = nullptr, *d_valid = nullptr, *d_tvalid = nullptr;
  double2 *d_T = nullptr, *d_Qf = nullptr, *d_Qb = nullptr, *d_sf = nullptr, *d_sb = nullptr, *d_basis = nullptr;
  int oidx(int o) const {
    for (int i = 0; i < nobs; ++i)
      if (obs[i] == o) return i;
    return -1;
  }
};

namespace {

int fail(ytf_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

#define CK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) return fail(ctx, YTF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

cudaEvent_t take_event(ytf_ctx* ctx) {
  if (!ctx->free_events.empty()) {
    cudaEvent_t e = ctx->free_events.back();
    ctx->free_events.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// launch one kernel through `f`, counting it and (when profiling) bracketing it with
// CUDA events on the context's stream
template <class F>
cudaError_t launch_named(ytf_ctx* ctx, const char* name, F&& f) {
  ctx->klaunch[name] += 1;
  if (!ctx->prof) return f();
  ProfSpan sp{name, take_event(ctx), take_event(ctx)};
  cudaEventRecord(sp.a, ctx->stream);
  cudaError_t e = f();
  cudaEventRecord(sp.b, ctx->stream);
  ctx->spans.push_back(sp);
  return e;
}
#define LAUNCH(name, expr) launch_named(ctx, name, [&]() { return (expr); })

// fold completed spans into the per-kernel totals (the stream has been synchronised)
void prof_collect(ytf_ctx* ctx) {
  for (auto& sp : ctx->spans) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, sp.a, sp.b) == cudaSuccess) {
      auto& t = ctx->ktime[sp.name];
      t.first += ms;
      t.second += 1;
    }
    ctx->free_events.push_back(sp.a);
    ctx->free_events.push_back(sp.b);
  }
  ctx->spans.clear();
}

void ctx_release(ytf_ctx* ctx) {
  if (--ctx->refs <= 0 && ctx->closing) delete ctx;
}

// cudaMalloc that, when the device is out of memory, releases the context's pool of idle cache
// blocks (every block enters the pool after its stream has finished with it) and tries once more
cudaError_t dev_malloc(ytf_ctx* ctx, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaErrorMemoryAllocation || ctx->pool.empty()) return e;
  cudaGetLastError();
  for (auto& kv : ctx->pool) cudaFree(kv.second);
  ctx->pool.clear();
  return cudaMalloc(p, bytes);
}

// `reserve`: the size a first allocation takes at least (a buffer whose size varies from call to
// call up to a known bound is allocated at the bound once, so that later calls do not pay a
// cudaFree's device-wide synchronisation to grow it)
void* ws_get(ytf_ctx* ctx, const char* name_, size_t bytes, cudaError_t* e, size_t reserve = 0) {
  *e = cudaSuccess;
  if (bytes == 0) bytes = 16;
  const std::string name = ctx->ws_slot > 0 ? std::string(name_) + "#" + std::to_string(ctx->ws_slot) : std::string(name_);
  if (ctx->ws_override) {
    auto o = ctx->ws_override->find(name);
    if (o == ctx->ws_override->end() || o->second.second < bytes) {
      *e = cudaErrorMemoryAllocation;
      return nullptr;
    }
    return o->second.first;
  }
  if (ctx->ws_record) {
    size_t& r = (*ctx->ws_record)[name];
    r = std::max(r, bytes);
  }
  auto it = ctx->ws.find(name);
  if (it != ctx->ws.end() && it->second.second >= bytes) return it->second.first;
  if (it != ctx->ws.end()) {
    // a buffer that has to grow grows by half again at least, so that calls of slowly
    // rising size do not each pay a device synchronisation and a cudaMalloc
    bytes = std::max(bytes, it->second.second + it->second.second / 2);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(it->second.first);
    ctx->ws.erase(it);
  }
  void* p = nullptr;
  if (it == ctx->ws.end() && reserve > bytes) {  // first allocation: at the bound if it fits
    if (cudaMalloc(&p, reserve) == cudaSuccess) {
      ctx->ws[name] = {p, reserve};
      return p;
    }
    cudaGetLastError();
    p = nullptr;
  }
  *e = dev_malloc(ctx, &p, bytes);
  if (*e != cudaSuccess) return nullptr;
  ctx->ws[name] = {p, bytes};
  return p;
}

// WS with a first-allocation bound (ws_get's reserve, in bytes)
#define WSR(ptr, type, name, count, reserve)                                                                 \
  type* ptr = nullptr;                                                                                       \
  {                                                                                                          \
    cudaError_t e_;                                                                                          \
    ptr = (type*)ws_get(ctx, name, sizeof(type) * (size_t)(count), &e_, (reserve));                          \
    if (!ptr) return fail(ctx, YTF_ERR_NOMEM, std::string("workspace ") + name + ": " + cudaGetErrorString(e_)); \
  }

#define WS(ptr, type, name, count)                                                                           \
  type* ptr = nullptr;                                                                                       \
  {                                                                                                          \
    cudaError_t e_;                                                                                          \
    ptr = (type*)ws_get(ctx, name, sizeof(type) * (size_t)(count), &e_);                                     \
    if (!ptr) return fail(ctx, YTF_ERR_NOMEM, std::string("workspace ") + name + ": " + cudaGetErrorString(e_)); \
  }

std::string obs_str(const int* obs, int n) {
  std::string s = "[";
  for (int i = 0; i < n; ++i) s += (i ? ", " : "") + std::to_string(obs[i]);
  return s + "]";
}

bool closed_form(const LayerDev& L) { return (L.ekind == 0 || L.ekind == 1) && L.mkind == 0; }

// a layer's Berreman matrix is finite at every node: finite ε and μ with ε33 ≠ 0 and μ33 ≠ 0
// (_berreman_core divides by both, mod_ModeSolver.jl:134-135)
bool berreman_finite(const LayerDev& L) {
  for (int i = 0; i < 18; ++i)
    if (!std::isfinite(L.eps[i]) || !std::isfinite(L.mu[i])) return false;
  return !(L.eps[16] == 0.0 && L.eps[17] == 0.0) && !(L.mu[16] == 0.0 && L.mu[17] == 0.0);
}

int upload(ytf_ctx* ctx, void* dst, const void* src, size_t bytes) {
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return YTF_OK;
}

// page-locked staging buffer of at least `bytes` (the stream is idle when it is replaced:
// every entry point that fills it synchronises before returning)
void* pinned_staging(ytf_ctx* ctx, size_t bytes) {
  if (ctx->pinned_bytes >= bytes) return ctx->pinned;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  ctx->pinned = nullptr;
  ctx->pinned_bytes = 0;
  size_t want = std::max(bytes, (size_t)1 << 20);
  if (cudaHostAlloc(&ctx->pinned, want, cudaHostAllocDefault) != cudaSuccess) {
    ctx->pinned = nullptr;
    return nullptr;
  }
  ctx->pinned_bytes = want;
  return ctx->pinned;
}

// state shared by the items of one ytf_green_batch call: pre-uploaded coordinates, one
// tensor-core error word, no per-item synchronisation
struct GreenBatch {
  const double* dzo;
  const double* dxs;
  const double* dys;
  unsigned* err;
  const double* drho = nullptr;  // 1D: the distinct radii (radii_map), pre-uploaded
  const int* drmap = nullptr;    // 1D: pixel -> radius index
};

// distinct radii hypot(x_i, y_j) in first-occurrence order over (i fastest, j), as the
// reference, and each pixel's index into them
void radii_map(int nx, const double* xs, int ny, const double* ys, std::vector<double>& ur, std::vector<int>& rmap) {
  const long npix = (long)nx * ny;
  ur.clear();
  rmap.assign(npix, 0);
  std::unordered_map<double, int> idx;
  idx.reserve(npix * 2);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      double r = std::hypot(xs[i], ys[j]);
      auto it = idx.find(r);
      if (it == idx.end()) { idx.emplace(r, (int)ur.size()); rmap[i + (long)nx * j] = (int)ur.size(); ur.push_back(r); }
      else rmap[i + (long)nx * j] = it->second;
    }
}

// allocate the cache's arrays in one block
int alloc_cache(ytf_ctx* ctx, ytf_cache* c, bool upload_nodes = true) {
  long n = c->n;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  size_t o_kr = take(8 * (size_t)c->Nk), o_wr = take(8 * (size_t)c->Nk), o_phi = take(8 * std::max<size_t>(1, c->phi.size())),
         o_wphi = take(8 * std::max<size_t>(1, c->wphi.size()));
  size_t o_kri = take(8 * std::max<size_t>(1, c->kri.size())), o_wri = take(8 * std::max<size_t>(1, c->wri.size()));
  size_t o_status = take(n), o_valid = take(n), o_tvalid = take((size_t)n * c->nobs);
  size_t o_T = take(16 * 16 * (size_t)n * c->nobs), o_Qf = take(16 * 2 * (size_t)n), o_Qb = take(16 * 2 * (size_t)n);
  size_t o_sf = take(16 * 6 * (size_t)n), o_sb = take(16 * 6 * (size_t)n), o_basis = take(16 * 16 * (size_t)n * c->nobs);
  c->block_bytes = off;
  auto it = ctx->pool.lower_bound(off);
  if (it != ctx->pool.end() && it->first <= 2 * off + (size_t(1) << 20)) {
    c->block = it->second;
    c->block_bytes = it->first;
    ctx->pool.erase(it);
  } else {
    CK(dev_malloc(ctx, &c->block, off));
  }
  char* b = (char*)c->block;
  c->d_kr = (double*)(b + o_kr); c->d_wr = (double*)(b + o_wr);
  c->d_phi = (double*)(b + o_phi); c->d_wphi = (double*)(b + o_wphi);
  c->d_kri = c->kri.empty() ? nullptr : (double*)(b + o_kri);
  c->d_wri = c->wri.empty() ? nullptr : (double*)(b + o_wri);
  c->d_status = (uint8_t*)(b + o_status); c->d_valid = (uint8_t*)(b + o_valid); c->d_tvalid = (uint8_t*)(b + o_tvalid);
  c->d_T = (double2*)(b + o_T); c->d_Qf = (double2*)(b + o_Qf); c->d_Qb = (double2*)(b + o_Qb);
  c->d_sf = (double2*)(b + o_sf); c->d_sb = (double2*)(b + o_sb); c->d_basis = (double2*)(b + o_basis);
  CK(cudaMemsetAsync(c->block, 0, off, ctx->stream));
  (void)o_status;
  int rc;
  if (!upload_nodes) return YTF_OK;
  if (c->src_kr) {
    CK(cudaMemcpyAsync(c->d_kr, c->src_kr, 8 * (size_t)c->Nk, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(c->d_wr, c->src_wr, 8 * (size_t)c->Nk, cudaMemcpyDeviceToDevice, ctx->stream));
  } else {
    if ((rc = upload(ctx, c->d_kr, c->kr.data(), 8 * c->kr.size()))) return rc;
    if ((rc = upload(ctx, c->d_wr, c->wr.data(), 8 * c->wr.size()))) return rc;
  }
  if (!c->kri.empty()) {
    if ((rc = upload(ctx, c->d_kri, c->kri.data(), 8 * c->kri.size()))) return rc;
    if ((rc = upload(ctx, c->d_wri, c->wri.data(), 8 * c->wri.size()))) return rc;
  }
  if (!c->phi.empty()) {
    if ((rc = upload(ctx, c->d_phi, c->phi.data(), 8 * c->phi.size()))) return rc;
    if ((rc = upload(ctx, c->d_wphi, c->wphi.data(), 8 * c->wphi.size()))) return rc;
  }
  return YTF_OK;
}

// which SLeft/SRight slots the walk to the observation layers reads (k_chain)
// the forward-only chain applies when every observation layer is the source layer
bool only_source_observed(const TransferParams& p) {
  for (int i = 0; i < p.nobs; ++i)
    if (p.obs[i] != p.src) return false;
  return true;
}

void need_masks(int N, int src, const int* obs, int nobs, uint32_t& needL, uint32_t& needR) {
  needL = needR = 0;
  for (int i = 0; i < nobs; ++i) {
    int o = obs[i];
    if (o < src) {
      for (int k : {o, o + 1})
        if (k >= 2 && k <= src - 1) needL |= 1u << (k - 1);
    } else if (o > src) {
      for (int k : {o, o + 1})
        if (k >= src + 1 && k <= N - 1) needR |= 1u << (k - 1);
    }
  }
}

int common_checks(ytf_ctx* ctx, const ytf_stack* st, const char* fn, int src, int nobs, const int* obs_in, std::vector<int>& obs) {
  if (!ctx) return YTF_ERR_ARG;
  if (!st) return fail(ctx, YTF_ERR_ARG, std::string(fn) + ": stack is NULL");
  if (st->ctx != ctx) return fail(ctx, YTF_ERR_STATE, std::string(fn) + ": stack belongs to another context");
  int N = st->nL;
  if (!(1 <= src && src < N))
    return fail(ctx, YTF_ERR_ARG, std::string(fn) + ": source_layer=" + std::to_string(src) + " must be in 1:" +
                                      std::to_string(N - 1) + " (the last, semi-infinite layer cannot host a source).");
  std::set<int> os;
  if (obs_in == nullptr || nobs <= 0) {
    for (int o = 1; o <= N; ++o) os.insert(o);
  } else {
    for (int i = 0; i < nobs; ++i) os.insert(obs_in[i]);
  }
  for (int o : os)
    if (o < 1 || o > N) return fail(ctx, YTF_ERR_ARG, std::string(fn) + ": obs_layers out of range 1:" + std::to_string(N));
  obs.assign(os.begin(), os.end());
  if ((int)obs.size() > MAXL) return fail(ctx, YTF_ERR_ARG, std::string(fn) + ": too many obs layers");
  return YTF_OK;
}

void fill_params(TransferParams& p, const ytf_stack* st, const ytf_cache* c) {
  std::memset(&p, 0, sizeof(p));
  p.layers = st->dev;
  p.nL = st->nL;
  p.src = c->src;
  p.nobs = c->nobs;
  for (int i = 0; i < c->nobs; ++i) p.obs[i] = c->obs[i];
  need_masks(st->nL, c->src, c->obs, c->nobs, p.needL, p.needR);
  p.omega = c->omega;
  p.Nk = c->Nk;
  p.Np = c->Np;
  p.kr = c->d_kr;
  p.phi = c->d_phi;
  p.status = c->d_status;
  p.valid = c->d_valid;
  p.tvalid = c->d_tvalid;
  p.Tout = c->d_T;
  p.Qf = c->d_Qf;
  p.Qb = c->d_Qb;
  p.sf = c->d_sf;
  p.sb = c->d_sb;
  p.basis = c->d_basis;
}

// the forward-only chain (every observation layer is the source layer)
int launch_forward_chain(ytf_ctx* ctx, const TransferParams& p) {
  CK(LAUNCH("k_iface", launch_chain_part(0, p, ctx->stream)));
  CK(LAUNCH("k_seeds", launch_chain_part(1, p, ctx->stream)));
  CK(LAUNCH("k_scan", launch_chain_part(2, p, ctx->stream)));
  return YTF_OK;
}

// per-node scratch bytes of the transfer kernels
size_t scratch_per_node(int N, uint32_t needL, uint32_t needR) {
  size_t b = (size_t)N * 20 * 16 + (size_t)std::max(N - 1, 1) * 16 * 16 + (size_t)N;
  if (needL) b += (size_t)N * 16 * 16;
  if (needR) b += (size_t)N * 16 * 16;
  return b;
}

// run k_layer_modes + k_chain over [0, total) in chunks that fit the scratch budget
int run_transfer(ytf_ctx* ctx, TransferParams p, long total) {
  const int N = p.nL;
  size_t per = scratch_per_node(N, p.needL, p.needR);
  const size_t budget = (size_t)6 << 30;  // 6 GiB of scratch per pass
  long chunk = (long)std::max<size_t>(1024, budget / per);
  chunk = std::min(chunk, total);
  WS(modes, double2, "tr_modes", (size_t)N * 20 * chunk);
  WS(lstat, uint8_t, "tr_lstat", (size_t)N * chunk);
  WS(sint, double2, "tr_sint", (size_t)std::max(N - 1, 1) * 16 * chunk);
  WS(dec, uint8_t, "tr_dec", (size_t)std::max(N - 1, 1) * chunk);
  double2* sleft = nullptr;
  double2* sright = nullptr;
  if (p.needL) { WS(sl, double2, "tr_sleft", (size_t)N * 16 * chunk); sleft = sl; }
  if (p.needR) { WS(sr, double2, "tr_sright", (size_t)N * 16 * chunk); sright = sr; }
  p.modes = modes;
  p.lstat = lstat;
  p.sint = sint;
  p.dec = dec;
  p.sleft = sleft;
  p.sright = sright;
  for (long off = 0; off < total; off += chunk) {
    p.off = off;
    p.n = std::min(chunk, total - off);
    CK(LAUNCH("k_layer_modes", launch_layer_modes(p, ctx->stream)));
    CK(LAUNCH("k_layer_modes_qr", launch_layer_modes_qr(p, ctx->stream)));
    if (only_source_observed(p)) {
      if (int rc = launch_forward_chain(ctx, p)) return rc;
    }
    else CK(LAUNCH("k_chain", launch_chain(p, ctx->stream)));
  }
  return YTF_OK;
}

}  // namespace

extern "C" {

int ytf_version(void) { return 10000; }

int ytf_ctx_create(ytf_ctx** out, int device) {
  if (!out) return YTF_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return YTF_ERR_CUDA;
  if (device < 0 || device >= ndev) return YTF_ERR_ARG;
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return YTF_ERR_CUDA;
  ytf_ctx* c = new ytf_ctx();
  c->device = device;
  c->stream = nullptr;  // legacy default stream until ytf_ctx_set_stream
  *out = c;
  return YTF_OK;
}

int ytf_ctx_destroy(ytf_ctx* ctx) {
  if (!ctx) return YTF_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->closing = true;
  if (ctx->refs <= 0) delete ctx;  // otherwise freed with its last stack or cache
  return YTF_OK;
}

int ytf_ctx_profile(ytf_ctx* ctx, int enable) {
  if (!ctx) return YTF_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  prof_collect(ctx);
  ctx->ktime.clear();
  ctx->klaunch.clear();
  ctx->prof = enable != 0;
  return YTF_OK;
}

int ytf_ctx_profile_read(ytf_ctx* ctx, int max_entries, char* names, double* total_ms, long* launches, int* n) {
  if (!ctx || !n) return YTF_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  prof_collect(ctx);
  int i = 0;
  for (auto& kv : ctx->klaunch) {
    if (i < max_entries) {
      if (names) {
        std::strncpy(names + 32 * i, kv.first.c_str(), 31);
        names[32 * i + 31] = 0;
      }
      auto it = ctx->ktime.find(kv.first);
      if (total_ms) total_ms[i] = it == ctx->ktime.end() ? 0.0 : it->second.first;
      if (launches) launches[i] = kv.second;
    }
    ++i;
  }
  *n = i;
  return YTF_OK;
}

int ytf_ctx_set_wait_limit(ytf_ctx* ctx, long polls) {
  if (!ctx) return YTF_ERR_ARG;
  if (polls < 0) return fail(ctx, YTF_ERR_ARG, "ytf_ctx_set_wait_limit: polls must be >= 0");
  ctx->wait_limit = polls == 0 ? (1L << 22) : polls;
  return YTF_OK;
}

int ytf_ctx_set_group_bytes(ytf_ctx* ctx, long bytes) {
  if (!ctx || bytes < 0) return YTF_ERR_ARG;
  ctx->group_bytes = bytes == 0 ? ((size_t)4 << 30) : (size_t)bytes;
  return YTF_OK;
}

int ytf_ctx_set_stream(ytf_ctx* ctx, void* stream) {
  if (!ctx) return YTF_ERR_ARG;
  ctx->stream = (cudaStream_t)stream;
  return YTF_OK;
}

int ytf_ctx_sync(ytf_ctx* ctx) {
  if (!ctx) return YTF_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  return YTF_OK;
}

const char* ytf_last_error(const ytf_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int ytf_stack_create(ytf_ctx* ctx, int nL, const int* eps_kind, const int* mu_kind, const double* eps, const double* mu,
                     const double* d, ytf_stack** out) {
  if (!ctx || !out) return YTF_ERR_ARG;
  *out = nullptr;
  if (nL < 2 || nL > MAXL) return fail(ctx, YTF_ERR_ARG, "ytf_stack_create: nL must be in 2:" + std::to_string(MAXL));
  if (!eps_kind || !eps || !d) return fail(ctx, YTF_ERR_ARG, "ytf_stack_create: eps_kind, eps and d are required");
  CK(cudaSetDevice(ctx->device));
  ytf_stack* s = new ytf_stack();
  s->ctx = ctx;
  ctx->refs += 1;
  s->nL = nL;
  s->host.resize(nL);
  for (int l = 0; l < nL; ++l) {
    LayerDev& L = s->host[l];
    L.ekind = eps_kind[l];
    L.mkind = mu_kind ? mu_kind[l] : 0;
    if (L.ekind < 0 || L.ekind > 3 || L.mkind < 0 || L.mkind > 3) {
      delete s;
      ctx->refs -= 1;
      return fail(ctx, YTF_ERR_ARG, "ytf_stack_create: material kind must be 0..3");
    }
    for (int i = 0; i < 18; ++i) {
      L.eps[i] = eps[18 * l + i];
      L.mu[i] = mu ? mu[18 * l + i] : ((i == 0 || i == 8 || i == 16) ? 1.0 : 0.0);
    }
    L.d = d[l];
  }
  cudaError_t e = cudaMalloc(&s->dev, sizeof(LayerDev) * nL);
  if (e != cudaSuccess) { delete s; ctx->refs -= 1; return fail(ctx, YTF_ERR_NOMEM, "ytf_stack_create: cudaMalloc failed"); }
  e = cudaMemcpy(s->dev, s->host.data(), sizeof(LayerDev) * nL, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { cudaFree(s->dev); delete s; ctx->refs -= 1; return fail(ctx, YTF_ERR_CUDA, cudaGetErrorString(e)); }
  *out = s;
  return YTF_OK;
}

int ytf_stack_destroy(ytf_stack* s) {
  if (!s) return YTF_OK;
  ytf_ctx* ctx = s->ctx;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(s->dev);
  delete s;
  ctx_release(ctx);
  return YTF_OK;
}

}  // extern "C"

namespace {

// validation and cache creation shared by the 1D/2D builds and the batch (no solve): the
// argument checks and messages of build_cavity_transfer_1d (mod_CavityTransfer.jl:196-205)
// and build_cavity_transfer_2d (:307-318)
int prepare_cache(ytf_ctx* ctx, const ytf_stack* st, bool is2d, double omega, int source_layer, int nk,
                  const double* k_nodes, const double* k_weights, int nphi, const double* phi_nodes,
                  const double* phi_weights, int nobs, const int* obs_layers, int check_symmetry, int rotation,
                  bool upload_nodes, ytf_cache** out, bool* use_rot, bool nodes_dev = false) {
  *out = nullptr;
  *use_rot = false;
  const char* fn = is2d ? "build_cavity_transfer_2d" : "build_cavity_transfer_1d";
  std::vector<int> obs;
  int rc = common_checks(ctx, st, fn, source_layer, nobs, obs_layers, obs);
  if (rc) return rc;
  if (!is2d) {
    if (nk < 0 || (nk > 0 && (!k_nodes || !k_weights)))
      return fail(ctx, YTF_ERR_ARG, "build_cavity_transfer_1d: kx_nodes/wt_nodes length mismatch");
    if (check_symmetry)
      for (auto& L : st->host)
        if (!closed_form(L))
          return fail(ctx, YTF_ERR_ARG,
                      "build_cavity_transfer_1d: the 1D path requires an isotropic/uniaxial stack "
                      "(`_is_azimuthally_symmetric_stack`); use the 2D (kρ,φ) cache for biaxial/gyrotropic.");
  } else {
    if (nk < 0 || (nk > 0 && (!k_nodes || !k_weights)))
      return fail(ctx, YTF_ERR_ARG, "build_cavity_transfer_2d: kρ nodes/weights length mismatch");
    if (nphi < 0 || (nphi > 0 && (!phi_nodes || !phi_weights)))
      return fail(ctx, YTF_ERR_ARG, "build_cavity_transfer_2d: φ nodes/weights length mismatch");
    bool sym = true;
    for (auto& L : st->host) sym = sym && closed_form(L);
    *use_rot = rotation == YTF_ROT_AUTO ? sym : rotation != 0;
    if (*use_rot && !sym)
      return fail(ctx, YTF_ERR_ARG, "build_cavity_transfer_2d: rotation=true requires an azimuthally symmetric stack");
  }
  // A layer on the general path goes through Julia's eigen, which refuses a non-finite
  // matrix with an ArgumentError that the reference's per-node try/catch does not catch
  // (mod_CavityTransfer.jl:249-251): the whole build fails at its first node. Closed-form
  // layers (isotropic/uniaxial ε, isotropic μ) never call eigen; their non-finite nodes
  // become invalid data, as in the reference.
  if ((is2d ? (long)nk * nphi : (long)nk) > 0)
    for (auto& L : st->host)
      if (!closed_form(L) && !berreman_finite(L)) return fail(ctx, YTF_ERR_ARG, "matrix contains Infs or NaNs");
  CK(cudaSetDevice(ctx->device));
  ytf_cache* c = new ytf_cache();
  c->ctx = ctx;
  ctx->refs += 1;
  c->stack_ref = st;
  c->nL = st->nL;
  c->src = source_layer;
  c->nobs = (int)obs.size();
  for (int i = 0; i < c->nobs; ++i) c->obs[i] = obs[i];
  c->omega = omega;
  c->is2d = is2d;
  c->rotation = *use_rot;
  c->Nk = nk;
  c->Np = is2d ? nphi : 1;
  c->n = is2d ? (long)nk * nphi : nk;
  if (nodes_dev) {
    c->src_kr = k_nodes;
    c->src_wr = k_weights;
  } else {
    c->kr.assign(k_nodes, k_nodes + nk);
    c->wr.assign(k_weights, k_weights + nk);
  }
  if (is2d) {
    c->phi.assign(phi_nodes, phi_nodes + nphi);
    c->wphi.assign(phi_weights, phi_weights + nphi);
  }
  for (auto& L : st->host) c->d_layer.push_back(L.d);
  c->d_src = st->host[source_layer - 1].d;
  if ((rc = alloc_cache(ctx, c, upload_nodes))) { ytf_cache_destroy(c); return rc; }
  *out = c;
  return YTF_OK;
}

// φ = 0 base solve per kρ, then the exact rotation to every φ (azimuthally symmetric stack)
int solve_rotation(ytf_ctx* ctx, const ytf_stack* st, ytf_cache* c, const TransferParams& p) {
  long nb = c->Nk;
  int N = st->nL;
  WS(modes, double2, "tr_modes", (size_t)N * 20 * nb);
  WS(lstat, uint8_t, "tr_lstat", (size_t)N * nb);
  WS(sint, double2, "tr_sint", (size_t)std::max(N - 1, 1) * 16 * nb);
  WS(bstat, uint8_t, "tr_bstatus", (size_t)nb);
  WS(btv, uint8_t, "tr_btvalid", (size_t)nb * c->nobs);
  WS(bT, double2, "tr_bT", (size_t)16 * nb * c->nobs);
  TransferParams b = p;
  b.mode = 2;
  b.n = nb;
  b.off = 0;
  b.nout = nb;
  b.modes = modes;
  b.lstat = lstat;
  b.sint = sint;
  WS(bdec, uint8_t, "tr_dec", (size_t)std::max(N - 1, 1) * nb);
  b.dec = bdec;
  if (b.needL) { WS(sl, double2, "tr_sleft", (size_t)N * 16 * nb); b.sleft = sl; }
  if (b.needR) { WS(sr, double2, "tr_sright", (size_t)N * 16 * nb); b.sright = sr; }
  b.status = bstat;
  b.tvalid = btv;
  b.Tout = bT;
  CK(LAUNCH("k_layer_modes", launch_layer_modes(b, ctx->stream)));
  CK(LAUNCH("k_layer_modes_qr", launch_layer_modes_qr(b, ctx->stream)));
  if (only_source_observed(b)) {
    if (int rc = launch_forward_chain(ctx, b)) return rc;
  }
  else CK(LAUNCH("k_chain", launch_chain(b, ctx->stream)));
  TransferParams f = p;
  f.mode = 1;
  f.n = nb;
  f.off = 0;
  f.nout = c->n;
  f.modes = modes;
  CK(LAUNCH("k_rotate_fill", launch_rotate_fill(f, bstat, btv, bT, ctx->stream)));
  return YTF_OK;
}

int finish_build(ytf_ctx* ctx, ytf_cache* c, ytf_cache** out) {
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) { ytf_cache_destroy(c); return fail(ctx, YTF_ERR_CUDA, cudaGetErrorString(e)); }
  prof_collect(ctx);
  *out = c;
  return YTF_OK;
}

}  // namespace

extern "C" {

int ytf_transfer_1d(ytf_ctx* ctx, const ytf_stack* st, double omega, int source_layer, int nk, const double* kx_nodes,
                    const double* wt_nodes, int nobs, const int* obs_layers, int check_symmetry, ytf_cache** out) {
  if (!ctx || !out) return YTF_ERR_ARG;
  *out = nullptr;
  ytf_cache* c;
  bool rot;
  int rc = prepare_cache(ctx, st, false, omega, source_layer, nk, kx_nodes, wt_nodes, 0, nullptr, nullptr, nobs,
                         obs_layers, check_symmetry, YTF_ROT_OFF, true, &c, &rot);
  if (rc) return rc;
  TransferParams p;
  fill_params(p, st, c);
  p.mode = 0;
  p.nout = c->n;
  if (c->n > 0 && (rc = run_transfer(ctx, p, c->n))) { ytf_cache_destroy(c); return rc; }
  return finish_build(ctx, c, out);
}

int ytf_transfer_2d(ytf_ctx* ctx, const ytf_stack* st, double omega, int source_layer, int nkr, const double* kr_nodes,
                    const double* kr_weights, int nphi, const double* phi_nodes, const double* phi_weights, int nobs,
                    const int* obs_layers, int rotation, ytf_cache** out) {
  if (!ctx || !out) return YTF_ERR_ARG;
  *out = nullptr;
  ytf_cache* c;
  bool use_rot;
  int rc = prepare_cache(ctx, st, true, omega, source_layer, nkr, kr_nodes, kr_weights, nphi, phi_nodes, phi_weights,
                         nobs, obs_layers, 1, rotation, true, &c, &use_rot);
  if (rc) return rc;
  TransferParams p;
  fill_params(p, st, c);
  if (c->n > 0) {
    if (!use_rot) {
      p.mode = 1;
      p.nout = c->n;
      rc = run_transfer(ctx, p, c->n);
    } else {
      rc = solve_rotation(ctx, st, c, p);
    }
    if (rc) { ytf_cache_destroy(c); return rc; }
  }
  return finish_build(ctx, c, out);
}

int ytf_cavity_response(ytf_ctx* ctx, const ytf_stack* st, double omega, int source_layer, long n, const double* kr,
                        double phi, double* out) {
  if (!ctx || (n > 0 && (!kr || !out)) || n < 0) return YTF_ERR_ARG;
  if (!st) return fail(ctx, YTF_ERR_ARG, "_cavity_response: stack is NULL");
  if (st->ctx != ctx) return fail(ctx, YTF_ERR_STATE, "_cavity_response: stack belongs to another context");
  const int N = st->nL;
  if (!(1 <= source_layer && source_layer < N))
    return fail(ctx, YTF_ERR_ARG, "_cavity_response: source layer " + std::to_string(source_layer) + " outside 1:" +
                                      std::to_string(N - 1));
  if (n == 0) return YTF_OK;
  CK(cudaSetDevice(ctx->device));
  // a (kρ, φ) grid of n x 1 nodes solved by the forward-only chain in response mode
  WS(dk, double, "cr_k", n);
  WS(dphi, double, "cr_phi", 1);
  WS(dresp, double, "cr_out", n);
  WS(dstat, uint8_t, "cr_status", n);
  int rc;
  if ((rc = upload(ctx, dk, kr, 8 * (size_t)n))) return rc;
  if ((rc = upload(ctx, dphi, &phi, 8))) return rc;
  TransferParams p;
  std::memset(&p, 0, sizeof(p));
  p.layers = st->dev;
  p.nL = N;
  p.src = source_layer;
  p.nobs = 1;
  p.obs[0] = source_layer;
  p.omega = omega;
  p.mode = 1;
  p.Nk = (int)n;
  p.Np = 1;
  p.kr = dk;
  p.phi = dphi;
  p.nout = n;
  p.status = dstat;
  p.resp = dresp;
  if ((rc = run_transfer(ctx, p, n))) return rc;
  CK(cudaMemcpyAsync(out, dresp, 8 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  prof_collect(ctx);
  return YTF_OK;
}

int ytf_cavity_response_batch(ytf_ctx* ctx, int nitems, const ytf_stack* const* stacks, const double* omega,
                              const int* source_layer, const long* counts, const double* kr, double phi, double* out) {
  if (!ctx || nitems < 0 || (nitems > 0 && (!stacks || !omega || !source_layer || !counts))) return YTF_ERR_ARG;
  long total = 0;
  for (int i = 0; i < nitems; ++i) {
    const ytf_stack* st = stacks[i];
    const std::string at = "_cavity_response (item " + std::to_string(i) + "): ";
    if (counts[i] < 0) return fail(ctx, YTF_ERR_ARG, at + "negative node count");
    if (!st) return fail(ctx, YTF_ERR_ARG, at + "stack is NULL");
    if (st->ctx != ctx) return fail(ctx, YTF_ERR_STATE, at + "stack belongs to another context");
    if (!(1 <= source_layer[i] && source_layer[i] < st->nL))
      return fail(ctx, YTF_ERR_ARG, at + "source layer " + std::to_string(source_layer[i]) + " outside 1:" +
                                        std::to_string(st->nL - 1));
    total += counts[i];
  }
  if (total == 0) return YTF_OK;
  if (!kr || !out) return YTF_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  WS(dk, double, "crb_k", total);
  WS(dphi, double, "crb_phi", 1);
  WS(dresp, double, "crb_out", total);
  WS(dstat, uint8_t, "crb_status", total);
  int rc;
  if ((rc = upload(ctx, dk, kr, 8 * (size_t)total))) return rc;
  if ((rc = upload(ctx, dphi, &phi, 8))) return rc;
  // each item is its own (kρ, φ) grid of counts[i] x 1 nodes, solved by the forward-only
  // chain in response mode; all items of a pass share the same five batched launches (the
  // batched kernels map a flat index to (item, node) and run the single-item per-node code),
  // passes bounded by the 6 GiB scratch budget
  const size_t budget = (size_t)6 << 30;
  std::vector<TransferParams> ps;
  std::vector<size_t> scr;
  long off = 0;
  for (int i = 0; i < nitems; ++i) {
    const long n = counts[i];
    if (n == 0) continue;
    TransferParams p;
    std::memset(&p, 0, sizeof(p));
    p.layers = stacks[i]->dev;
    p.nL = stacks[i]->nL;
    p.src = source_layer[i];
    p.nobs = 1;
    p.obs[0] = source_layer[i];
    p.omega = omega[i];
    p.mode = 1;
    p.Nk = (int)n;
    p.Np = 1;
    p.kr = dk + off;
    p.phi = dphi;
    p.n = n;
    p.off = 0;
    p.nout = n;
    p.status = dstat + off;
    p.resp = dresp + off;
    ps.push_back(p);
    scr.push_back(scratch_per_node(p.nL, 0, 0) * (size_t)n + 4 * 256);
    off += n;
  }
  size_t first = 0;
  while (first < ps.size()) {
    size_t last = first, used = 0;
    while (last < ps.size() && (last == first || used + scr[last] <= budget)) used += scr[last++];
    const int m = (int)(last - first);
    if (used > budget) {  // one item larger than a pass: its own chunked solve
      if ((rc = run_transfer(ctx, ps[first], ps[first].n))) return rc;
      first = last;
      continue;
    }
    WS(arena, char, "crb_scratch", used);
    size_t o = 0;
    auto carve = [&](size_t bytes) {
      char* q = arena + o;
      o += (bytes + 255) & ~size_t(255);
      return q;
    };
    std::vector<long> offm(m + 1, 0), offs(m + 1, 0), offi(m + 1, 0);
    std::vector<TransferParams> part(ps.begin() + first, ps.begin() + last);
    for (int j = 0; j < m; ++j) {
      TransferParams& q = part[j];
      const int N = q.nL;
      const long n = q.n;
      q.modes = (double2*)carve((size_t)N * 20 * 16 * n);
      q.lstat = (uint8_t*)carve((size_t)N * n);
      q.sint = (double2*)carve((size_t)std::max(N - 1, 1) * 16 * 16 * n);
      q.dec = (uint8_t*)carve((size_t)std::max(N - 1, 1) * n);
      offm[j + 1] = offm[j] + (long)N * n;
      offs[j + 1] = offs[j] + n;
      offi[j + 1] = offi[j] + (long)(N - 1) * n;
    }
    const size_t pbytes = sizeof(TransferParams) * m, lbytes = sizeof(long) * (m + 1);
    WS(dpar, char, "crb_params", pbytes + 3 * lbytes);
    std::vector<char> hbuf(pbytes + 3 * lbytes);
    std::memcpy(hbuf.data(), part.data(), pbytes);
    std::memcpy(hbuf.data() + pbytes, offm.data(), lbytes);
    std::memcpy(hbuf.data() + pbytes + lbytes, offs.data(), lbytes);
    std::memcpy(hbuf.data() + pbytes + 2 * lbytes, offi.data(), lbytes);
    CK(cudaMemcpyAsync(dpar, hbuf.data(), hbuf.size(), cudaMemcpyHostToDevice, ctx->stream));
    const TransferParams* dp = (const TransferParams*)dpar;
    const long* doffm = (const long*)(dpar + pbytes);
    const long* doffs = doffm + (m + 1);
    const long* doffi = doffs + (m + 1);
    CK(LAUNCH("k_layer_modes", launch_transfer_batch(0, dp, doffm, m, offm[m], ctx->stream)));
    CK(LAUNCH("k_layer_modes_qr", launch_transfer_batch(1, dp, doffm, m, offm[m], ctx->stream)));
    if (offi[m]) CK(LAUNCH("k_iface", launch_transfer_batch(6, dp, doffi, m, offi[m], ctx->stream)));
    CK(LAUNCH("k_seeds", launch_transfer_batch(5, dp, doffs, m, offs[m], ctx->stream)));
    CK(LAUNCH("k_scan", launch_transfer_batch(7, dp, doffs, m, offs[m], ctx->stream)));
    // the host block is read by the copy above before the next pass reuses it
    CK(cudaStreamSynchronize(ctx->stream));
    first = last;
  }
  CK(cudaMemcpyAsync(out, dresp, 8 * (size_t)total, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  prof_collect(ctx);
  return YTF_OK;
}

int ytf_layer_light_lines(const double* eps, const double* mu, double omega, double phi, double* out, int* n) {
  if (!eps || !n) return YTF_ERR_ARG;
  static const double mu_one[18] = {1, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1, 0};
  auto L = grid::layer_light_lines(eps, mu ? mu : mu_one, omega, phi);
  if (out)
    for (size_t i = 0; i < L.size() && i < 3; ++i) out[i] = L[i];
  *n = (int)L.size();
  return YTF_OK;
}

static int rule_from_features(ytf_ctx* ctx, const grid::Features& F, const ytf_grid_params* prm, long cap, double* k,
                              double* w, long* n, ytf_grid_info* info, const char* fn);

static int nodes_1d_impl(ytf_ctx* ctx, const ytf_stack* st, double omega, int source_layer, const ytf_grid_params* prm,
                         int npoles, const double* pq, const double* pG, long cap, double* k, double* w, long* n,
                         ytf_grid_info* info) {
  if (!ctx || !prm || !n) return YTF_ERR_ARG;
  if (!st) return fail(ctx, YTF_ERR_ARG, "point_kx_grid: stack is NULL");
  if (st->ctx != ctx) return fail(ctx, YTF_ERR_STATE, "point_kx_grid: stack belongs to another context");
  const int N = st->nL;
  if (!(1 <= source_layer && source_layer < N))
    return fail(ctx, YTF_ERR_ARG, "point_kx_grid: source_layer=" + std::to_string(source_layer) + " must be in 1:" +
                                      std::to_string(N - 1));
  if (!(prm->h_min > 0)) return fail(ctx, YTF_ERR_ARG, "point_kx_grid: h_min must be positive");
  if (prm->order < 1) return fail(ctx, YTF_ERR_ARG, "point_kx_grid: order must be ≥ 1");
  if (!(prm->rtol > 0 && prm->rtol < 1)) return fail(ctx, YTF_ERR_ARG, "point_kx_grid: rtol must be in (0, 1)");
  std::vector<const double*> eps(N), mu(N);
  for (int j = 0; j < N; ++j) { eps[j] = st->host[j].eps; mu[j] = st->host[j].mu; }
  // the pole scan's evaluator: the cavity response of the source layer at φ = 0, on the device
  grid::Eval f = [&](const std::vector<double>& ks, std::vector<double>& out) -> int {
    out.assign(ks.size(), 0.0);
    if (ks.empty()) return 0;
    return ytf_cavity_response(ctx, st, omega, source_layer, (long)ks.size(), ks.data(), 0.0, out.data());
  };
  grid::Features F;
  int rc = grid::features_1d(eps, mu, omega, prm->h_min, prm->rho_max, prm->target_decay, prm->kr_cap, 1e5,
                             npoles < 0 && prm->scan != 0, 1e-3, 1.05, f, F);
  if (rc) return rc;
  if (npoles >= 0) {  // poles proposed by the caller instead of the scan
    F.poles.clear();
    for (int i = 0; i < npoles; ++i)
      if (pq[i] > 0 && pG[i] > 0 && pq[i] < F.Kcut) F.poles.push_back({pq[i], pG[i], 0.0, 0.0});
    F.cl = grid::clusters(F.poles, 0.0);
  }
  return rule_from_features(ctx, F, prm, cap, k, w, n, info, "point_kx_grid");
}

// fixed_kρ_rule on the features: panels, the info block, the Gauss-Legendre nodes
static int rule_from_features(ytf_ctx* ctx, const grid::Features& F, const ytf_grid_params* prm, long cap, double* k,
                              double* w, long* n, ytf_grid_info* info, const char* fn) {
  std::vector<std::pair<double, double>> panels;
  try {
    panels = grid::fixed_kr_panels(F, prm->order, prm->rtol, 0.5, 12, 0.05, 4.0, 4.0, 0.5);
  } catch (std::exception& e) {
    return fail(ctx, YTF_ERR_ARG, e.what());
  }
  const long tot = (long)panels.size() * prm->order;
  *n = tot;
  if (info) {
    double* pan = info->panels;
    const long pcap = info->panels_cap;
    std::memset(info, 0, sizeof(*info));
    info->panels = pan;
    info->panels_cap = pcap;
    if (pan && pcap >= (long)panels.size())
      for (size_t i = 0; i < panels.size(); ++i) { pan[2 * i] = panels[i].first; pan[2 * i + 1] = panels[i].second; }
    info->Kcut = F.Kcut;
    info->kmax = F.kmax;
    info->n_panels = (long)panels.size();
    info->n_poles = (int)F.poles.size();
    for (int i = 0; i < (int)F.poles.size() && i < YTF_GRID_MAX_POLES; ++i) {
      info->poles[i][0] = F.poles[i].q;
      info->poles[i][1] = F.poles[i].G;
    }
    info->n_light_lines = (int)F.light_lines.size();
    for (int i = 0; i < (int)F.light_lines.size() && i < YTF_GRID_MAX_LINES; ++i) info->light_lines[i] = F.light_lines[i];
  }
  if (!k || !w) return YTF_OK;  // size query
  if (cap < tot)
    return fail(ctx, YTF_ERR_ARG, std::string(fn) + ": output capacity " + std::to_string(cap) + " < " +
                                      std::to_string(tot) + " nodes");
  std::vector<double> pa(panels.size()), pb(panels.size());
  for (size_t i = 0; i < panels.size(); ++i) { pa[i] = panels[i].first; pb[i] = panels[i].second; }
  return ytf_gl_rule(ctx, (int)panels.size(), pa.data(), pb.data(), prm->order, (int)F.singular_lines.size(),
                     F.singular_lines.data(), k, w);
}

int ytf_nodes_1d(ytf_ctx* ctx, const ytf_stack* st, double omega, int source_layer, const ytf_grid_params* prm, long cap,
                 double* k, double* w, long* n, ytf_grid_info* info) {
  return nodes_1d_impl(ctx, st, omega, source_layer, prm, -1, nullptr, nullptr, cap, k, w, n, info);
}

int ytf_nodes_from_poles(ytf_ctx* ctx, const ytf_stack* st, double omega, int source_layer, const ytf_grid_params* prm,
                         int npoles, const double* q, const double* G, long cap, double* k, double* w, long* n,
                         ytf_grid_info* info) {
  if (npoles < 0 || (npoles > 0 && (!q || !G))) return YTF_ERR_ARG;
  return nodes_1d_impl(ctx, st, omega, source_layer, prm, npoles, q, G, cap, k, w, n, info);
}

int ytf_rule_panels_batch(ytf_ctx* ctx, int nprob, const ytf_stack* const* stacks, const double* omega,
                          const int* source_layer, const ytf_grid_params* prm, const int* npoles, const double* q,
                          const double* G, long cap, double* panels, long* counts, long* total) {
  if (!ctx || nprob < 0 || (nprob > 0 && (!stacks || !omega || !source_layer || !prm || !npoles || !counts)) || !total)
    return YTF_ERR_ARG;
  // the checks of nodes_1d_impl, in problem order (the first failing problem is reported)
  std::vector<long> qoff(nprob + 1, 0);
  for (int j = 0; j < nprob; ++j) {
    const std::string tag = " (problem " + std::to_string(j) + ")";
    const ytf_stack* st = stacks[j];
    if (!st) return fail(ctx, YTF_ERR_ARG, "point_kx_grid: stack is NULL" + tag);
    if (st->ctx != ctx) return fail(ctx, YTF_ERR_STATE, "point_kx_grid: stack belongs to another context" + tag);
    if (!(1 <= source_layer[j] && source_layer[j] < st->nL))
      return fail(ctx, YTF_ERR_ARG, "point_kx_grid: source_layer=" + std::to_string(source_layer[j]) + " must be in 1:" +
                                        std::to_string(st->nL - 1) + tag);
    const ytf_grid_params& P = prm[j];
    if (!(P.h_min > 0)) return fail(ctx, YTF_ERR_ARG, "point_kx_grid: h_min must be positive" + tag);
    if (P.order < 1) return fail(ctx, YTF_ERR_ARG, "point_kx_grid: order must be ≥ 1" + tag);
    if (!(P.rtol > 0 && P.rtol < 1)) return fail(ctx, YTF_ERR_ARG, "point_kx_grid: rtol must be in (0, 1)" + tag);
    if (npoles[j] < 0 && P.scan) return fail(ctx, YTF_ERR_ARG, "ytf_rule_panels_batch: the pole scan runs per problem" + tag);
    qoff[j + 1] = qoff[j] + std::max(npoles[j], 0);
  }
  if (qoff[nprob] > 0 && (!q || !G)) return YTF_ERR_ARG;
  // features and panels per problem on the host threads (host arithmetic only: no scan)
  std::vector<std::vector<std::pair<double, double>>> out(nprob);
  std::vector<std::string> errs(nprob);
  auto one = [&](int j) {
    const ytf_stack* st = stacks[j];
    const int N = st->nL;
    std::vector<const double*> eps(N), mu(N);
    for (int l = 0; l < N; ++l) { eps[l] = st->host[l].eps; mu[l] = st->host[l].mu; }
    const ytf_grid_params& P = prm[j];
    grid::Eval none = [](const std::vector<double>&, std::vector<double>& o) -> int { o.clear(); return 0; };
    grid::Features F;
    try {
      if (grid::features_1d(eps, mu, omega[j], P.h_min, P.rho_max, P.target_decay, P.kr_cap, 1e5, false, 1e-3, 1.05,
                            none, F)) {
        errs[j] = "point_kx_grid: feature extraction failed";
        return;
      }
      if (npoles[j] >= 0) {
        F.poles.clear();
        for (long i = qoff[j]; i < qoff[j + 1]; ++i)
          if (q[i] > 0 && G[i] > 0 && q[i] < F.Kcut) F.poles.push_back({q[i], G[i], 0.0, 0.0});
        F.cl = grid::clusters(F.poles, 0.0);
      }
      out[j] = grid::fixed_kr_panels(F, P.order, P.rtol, 0.5, 12, 0.05, 4.0, 4.0, 0.5);
    } catch (std::exception& e) {
      errs[j] = e.what();
    }
  };
  const int nthr = (int)std::max(1u, std::min<unsigned>(std::min(std::thread::hardware_concurrency(), 32u),
                                                        (unsigned)std::max(nprob, 1)));
  if (nthr <= 1 || nprob < 8) {
    for (int j = 0; j < nprob; ++j) one(j);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < nthr; ++t)
      pool.emplace_back([&, t]() {
        for (int j = t; j < nprob; j += nthr) one(j);
      });
    for (auto& th : pool) th.join();
  }
  long tot = 0;
  for (int j = 0; j < nprob; ++j) {
    if (!errs[j].empty()) return fail(ctx, YTF_ERR_ARG, errs[j] + " (problem " + std::to_string(j) + ")");
    counts[j] = (long)out[j].size();
    tot += counts[j];
  }
  *total = tot;
  if (tot > cap || (tot > 0 && !panels))
    return fail(ctx, YTF_ERR_ARG, "ytf_rule_panels_batch: " + std::to_string(tot) + " panels exceed the capacity " +
                                      std::to_string(cap));
  long o = 0;
  for (int j = 0; j < nprob; ++j)
    for (auto& pr : out[j]) {
      panels[2 * o] = pr.first;
      panels[2 * o + 1] = pr.second;
      ++o;
    }
  return YTF_OK;
}

int ytf_peaks_batch(int nwin, int npts, const double* ks, const double* logR, double prominence, double floor_rel,
                    long cap, int* counts, double* q, double* G, long* total) {
  if (nwin < 0 || npts < 0 || (nwin > 0 && npts > 0 && (!ks || !logR)) || !counts || !total) return YTF_ERR_ARG;
  long t = 0;
  std::vector<std::pair<double, double>> pk;
  for (int w = 0; w < nwin; ++w) {
    pk.clear();
    grid::sampled_peaks(ks + (size_t)w * npts, logR + (size_t)w * npts, npts, prominence, floor_rel, pk);
    counts[w] = (int)pk.size();
    for (auto& e : pk) {
      if (q && G && t < cap) { q[t] = e.first; G[t] = e.second; }
      ++t;
    }
  }
  *total = t;
  return (q && G && t > cap) ? YTF_ERR_ARG : YTF_OK;
}

int ytf_adaptive_seeds(ytf_ctx* ctx, const ytf_stack* st, double omega, int source_layer, const ytf_grid_params* prm,
                       long cap, double* seeds, long* n) {
  if (!ctx || !prm || !n) return YTF_ERR_ARG;
  if (!st) return fail(ctx, YTF_ERR_ARG, "adaptive_seeds: stack is NULL");
  if (st->ctx != ctx) return fail(ctx, YTF_ERR_STATE, "adaptive_seeds: stack belongs to another context");
  const int N = st->nL;
  if (!(1 <= source_layer && source_layer < N))
    return fail(ctx, YTF_ERR_ARG, "point_kx_grid: source_layer=" + std::to_string(source_layer) + " must be in 1:" +
                                      std::to_string(N - 1));
  if (!(prm->h_min > 0)) return fail(ctx, YTF_ERR_ARG, "adaptive_seeds: h_min must be positive");
  if (!(prm->rtol > 0 && prm->rtol < 1)) return fail(ctx, YTF_ERR_ARG, "adaptive_seeds: rtol must be in (0, 1)");
  std::vector<const double*> eps(N), mu(N);
  for (int j = 0; j < N; ++j) { eps[j] = st->host[j].eps; mu[j] = st->host[j].mu; }
  grid::Eval f = [&](const std::vector<double>& ks, std::vector<double>& out) -> int {
    out.assign(ks.size(), 0.0);
    if (ks.empty()) return 0;
    return ytf_cavity_response(ctx, st, omega, source_layer, (long)ks.size(), ks.data(), 0.0, out.data());
  };
  grid::Features F;
  int rc = grid::features_1d(eps, mu, omega, prm->h_min, prm->rho_max, prm->target_decay, prm->kr_cap, 1e5,
                             prm->scan != 0, 1e-3, 1.05, f, F);
  if (rc) return rc;
  auto S = grid::adaptive_seeds(F, prm->rtol);
  *n = (long)S.size();
  if (!seeds) return YTF_OK;
  if (cap < *n) return fail(ctx, YTF_ERR_ARG, "adaptive_seeds: output capacity too small");
  std::copy(S.begin(), S.end(), seeds);
  return YTF_OK;
}

int ytf_nodes_2d(ytf_ctx* ctx, const ytf_stack* st, double omega, int source_layer, const ytf_grid_params* prm,
                 int n_phi_scan, long cap, double* k, double* w, long* n, long* n_phi, ytf_grid_info* info) {
  if (!ctx || !prm || !n || !n_phi) return YTF_ERR_ARG;
  if (!st) return fail(ctx, YTF_ERR_ARG, "point_kρ_grid_2d: stack is NULL");
  if (st->ctx != ctx) return fail(ctx, YTF_ERR_STATE, "point_kρ_grid_2d: stack belongs to another context");
  const int N = st->nL;
  if (!(1 <= source_layer && source_layer < N))
    return fail(ctx, YTF_ERR_ARG, "point_kρ_grid_2d: source_layer=" + std::to_string(source_layer) +
                                      " must be in 1:" + std::to_string(N - 1));
  if (!(prm->h_min > 0)) return fail(ctx, YTF_ERR_ARG, "point_kρ_grid_2d: h_min must be positive");
  if (prm->order < 1) return fail(ctx, YTF_ERR_ARG, "point_kρ_grid_2d: order must be ≥ 1");
  if (!(prm->rtol > 0 && prm->rtol < 1)) return fail(ctx, YTF_ERR_ARG, "point_kρ_grid_2d: rtol must be in (0, 1)");
  if (n_phi_scan < 1) return fail(ctx, YTF_ERR_ARG, "point_kρ_grid_2d: N_φ_scan must be ≥ 1");
  std::vector<const double*> eps(N), mu(N);
  bool sym = true, diag = true;
  for (int j = 0; j < N; ++j) {
    const LayerDev& L = st->host[j];
    eps[j] = L.eps;
    mu[j] = L.mu;
    sym = sym && closed_form(L);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        if (a != b) {
          const int e = 2 * (a + 3 * b);
          if (L.eps[e] != 0.0 || L.eps[e + 1] != 0.0 || L.mu[e] != 0.0 || L.mu[e + 1] != 0.0) diag = false;
        }
  }
  // the pole scan's evaluator along each direction: the source layer's cavity response on the device
  grid::EvalAt f = [&](double phi) -> grid::Eval {
    return [&, phi](const std::vector<double>& ks, std::vector<double>& out) -> int {
      out.assign(ks.size(), 0.0);
      if (ks.empty()) return 0;
      return ytf_cavity_response(ctx, st, omega, source_layer, (long)ks.size(), ks.data(), phi, out.data());
    };
  };
  grid::Features F;
  int rc = grid::features_2d(eps, mu, sym, diag, omega, prm->h_min, prm->rho_max, prm->target_decay, prm->kr_cap, 1e5,
                             prm->scan != 0, 1e-3, 1.05, n_phi_scan, 2.5, 64, prm->rtol, 1.5, f, F);
  if (rc) return rc;
  *n_phi = F.N_phi;
  return rule_from_features(ctx, F, prm, cap, k, w, n, info, "point_kρ_grid_2d");
}

int ytf_transfer_1d_contour(ytf_ctx* ctx, const ytf_stack* st, double omega, int source_layer, int nk,
                            const double* k_re, const double* k_im, const double* w_re, const double* w_im, int nobs,
                            const int* obs_layers, ytf_cache** out) {
  if (!ctx || !out) return YTF_ERR_ARG;
  *out = nullptr;
  if (nk > 0 && (!k_im || !w_im))
    return fail(ctx, YTF_ERR_ARG, "build_cavity_transfer_1d: contour nodes need imaginary parts");
  ytf_cache* c;
  bool rot;
  int rc = prepare_cache(ctx, st, false, omega, source_layer, nk, k_re, w_re, 0, nullptr, nullptr, nobs, obs_layers, 1,
                         YTF_ROT_OFF, false, &c, &rot);
  if (rc) return rc;
  // the cache block was laid out before the imaginary parts were known: lay it out again
  c->kri.assign(k_im, k_im + nk);
  c->wri.assign(w_im, w_im + nk);
  if (c->block) {
    cudaStreamSynchronize(ctx->stream);
    ctx->pool.emplace(c->block_bytes, c->block);
    c->block = nullptr;
  }
  if ((rc = alloc_cache(ctx, c, true))) { ytf_cache_destroy(c); return rc; }
  TransferParams p;
  fill_params(p, st, c);
  p.mode = 0;
  p.nout = c->n;
  p.kr_im = c->d_kri;
  if (c->n > 0 && (rc = run_transfer(ctx, p, c->n))) { ytf_cache_destroy(c); return rc; }
  return finish_build(ctx, c, out);
}

int ytf_bessel_j(ytf_ctx* ctx, int order, long n, const double* z_re, const double* z_im, double* out_re,
                 double* out_im) {
  if (!ctx || order < 0 || order > 2 || n < 0 || (n > 0 && (!z_re || !z_im || !out_re || !out_im))) return YTF_ERR_ARG;
  if (n == 0) return YTF_OK;
  CK(cudaSetDevice(ctx->device));
  WS(buf, double, "bj_buf", 4 * (size_t)n);
  int rc;
  if ((rc = upload(ctx, buf, z_re, 8 * (size_t)n)) || (rc = upload(ctx, buf + n, z_im, 8 * (size_t)n))) return rc;
  CK(LAUNCH("k_bessel_eval", launch_bessel_eval(n, order, buf, buf + n, buf + 2 * n, buf + 3 * n, ctx->stream)));
  CK(cudaMemcpyAsync(out_re, buf + 2 * n, 8 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(out_im, buf + 3 * n, 8 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return YTF_OK;
}

int ytf_bessel_j01(ytf_ctx* ctx, long n, const double* x, double* j0, double* j1) {
  if (!ctx || n < 0 || (n > 0 && (!x || !j0 || !j1))) return YTF_ERR_ARG;
  if (n == 0) return YTF_OK;
  CK(cudaSetDevice(ctx->device));
  WS(buf, double, "bj01", 3 * (size_t)n);
  int rc;
  if ((rc = upload(ctx, buf, x, 8 * (size_t)n))) return rc;
  CK(launch_bessel_j01(buf, n, buf + n, buf + 2 * n, ctx->stream));
  CK(cudaMemcpyAsync(j0, buf + n, 8 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(j1, buf + 2 * n, 8 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return YTF_OK;
}

int ytf_transfer_batch(ytf_ctx* ctx, int nb, const ytf_transfer_desc* d, ytf_cache** out) {
  if (!ctx || nb < 0 || (nb > 0 && (!d || !out))) return YTF_ERR_ARG;
  for (int i = 0; i < nb; ++i) out[i] = nullptr;
  if (nb == 0) return YTF_OK;
  CK(cudaSetDevice(ctx->device));
  std::vector<ytf_cache*> cs(nb, nullptr);
  std::vector<char> rot(nb, 0);
  auto abort_all = [&](int rc) {
    cudaStreamSynchronize(ctx->stream);
    for (auto c : cs)
      if (c) ytf_cache_destroy(c);
    return rc;
  };
  // 1. validate and create every cache; node arrays go up from one page-locked block
  size_t stage = 0;
  for (int i = 0; i < nb; ++i) {
    bool r = false;
    const bool is2d = d[i].nphi > 0 || d[i].is2d;
    int rc = YTF_OK;
    if (is2d && d[i].nodes_on_device)
      rc = fail(ctx, YTF_ERR_ARG, "build_cavity_transfer_2d: nodes_on_device applies to 1D items only");
    if (!rc)
      rc = prepare_cache(ctx, d[i].stack, is2d, d[i].omega, d[i].source_layer, d[i].nk, d[i].k_nodes, d[i].k_weights,
                         d[i].nphi, d[i].phi_nodes, d[i].phi_weights, d[i].nobs, d[i].obs_layers,
                         d[i].check_symmetry, d[i].rotation, false, &cs[i], &r, d[i].nodes_on_device != 0);
    if (rc) {
      std::string m = ctx->err;
      abort_all(rc);
      return fail(ctx, rc, m + " (batch item " + std::to_string(i) + ")");
    }
    rot[i] = r;
    stage += 2 * cs[i]->kr.size() + 2 * cs[i]->phi.size();
  }
  // 2. the fused passes: items grouped so that their node scratch fits the budget
  const size_t budget = (size_t)6 << 30;
  std::vector<TransferParams> ps(nb);
  std::vector<size_t> scratch(nb, 0);
  for (int i = 0; i < nb; ++i) {
    fill_params(ps[i], d[i].stack, cs[i]);
    ps[i].mode = cs[i]->is2d ? 1 : 0;
    ps[i].n = cs[i]->n;
    ps[i].off = 0;
    ps[i].nout = cs[i]->n;
    const int N = ps[i].nL;
    const bool fast = only_source_observed(ps[i]);
    size_t per = (size_t)N * 20 * 16 + (size_t)N;
    if (fast) per += (size_t)std::max(N - 1, 1) * (16 * 16 + 1);
    if (!fast) per = scratch_per_node(N, ps[i].needL, ps[i].needR);
    scratch[i] = per * (size_t)cs[i]->n + 5 * 256;
  }
  // per pass: every item's block, then the forward-only and general subsets, 3 offset arrays
  size_t pbytes = 2 * (size_t)nb * sizeof(TransferParams) + 4 * (size_t)(nb + 1) * sizeof(long);
  char* h = (char*)pinned_staging(ctx, 8 * std::max<size_t>(stage, 1) + pbytes + 64);
  if (!h) return abort_all(fail(ctx, YTF_ERR_NOMEM, "build_cavity_transfer: page-locked staging allocation failed"));
  {
    double* hd = (double*)h;
    size_t k = 0;
    for (int i = 0; i < nb; ++i) {
      ytf_cache* c = cs[i];
      auto put = [&](double* dst, const std::vector<double>& v) -> int {
        if (v.empty()) return YTF_OK;
        std::memcpy(hd + k, v.data(), 8 * v.size());
        cudaError_t e = cudaMemcpyAsync(dst, hd + k, 8 * v.size(), cudaMemcpyHostToDevice, ctx->stream);
        k += v.size();
        return e == cudaSuccess ? YTF_OK : fail(ctx, YTF_ERR_CUDA, cudaGetErrorString(e));
      };
      int rc;
      if ((rc = put(c->d_kr, c->kr)) || (rc = put(c->d_wr, c->wr)) || (rc = put(c->d_phi, c->phi)) ||
          (rc = put(c->d_wphi, c->wphi)))
        return abort_all(rc);
      if (c->src_kr && c->Nk > 0) {  // device-resident nodes: device to device, on the same stream
        cudaError_t e = cudaMemcpyAsync(c->d_kr, c->src_kr, 8 * (size_t)c->Nk, cudaMemcpyDeviceToDevice, ctx->stream);
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(c->d_wr, c->src_wr, 8 * (size_t)c->Nk, cudaMemcpyDeviceToDevice, ctx->stream);
        if (e != cudaSuccess) return abort_all(fail(ctx, YTF_ERR_CUDA, cudaGetErrorString(e)));
      }
    }
    h += ((8 * k + 63) / 64) * 64;
  }
  // rotation items and items too large for one pass take the single-problem paths
  for (int i = 0; i < nb; ++i) {
    if (cs[i]->n == 0 || !(rot[i] || scratch[i] > budget)) continue;
    int rc = rot[i] ? solve_rotation(ctx, d[i].stack, cs[i], ps[i]) : run_transfer(ctx, ps[i], cs[i]->n);
    if (rc) return abort_all(rc);
  }
  int first = 0;
  bool staged = false;
  while (first < nb) {
    std::vector<int> items;
    size_t used = 0;
    int i = first;
    for (; i < nb; ++i) {
      if (cs[i]->n == 0 || rot[i] || scratch[i] > budget) continue;
      if (used + scratch[i] > budget) break;
      items.push_back(i);
      used += scratch[i];
    }
    first = i;
    if (items.empty()) continue;
    WSR(arena, char, "tb_scratch", used, budget);
    size_t o = 0;
    auto carve = [&](size_t bytes) {
      char* q = arena + o;
      o += (bytes + 255) & ~size_t(255);
      return q;
    };
    const int m = (int)items.size();
    // the previous pass's parameter upload reads the same staging bytes: wait for that copy
    // only (its kernels keep running)
    if (staged) CK(cudaEventSynchronize(ctx->stage_ev));
    TransferParams* hp = (TransferParams*)h;
    long* offm = (long*)(hp + m);
    long* offs = offm + (m + 1);
    long* offg = offs + (m + 1);
    long* offi = offg + (m + 1);
    std::vector<int> fast_ids, gen_ids;
    offm[0] = 0;
    for (int j = 0; j < m; ++j) {
      TransferParams& q = ps[items[j]];
      const int N = q.nL;
      const long n = q.n;
      q.modes = (double2*)carve((size_t)N * 20 * 16 * n);
      q.lstat = (uint8_t*)carve((size_t)N * n);
      if (only_source_observed(q)) {
        q.sint = (double2*)carve((size_t)std::max(N - 1, 1) * 16 * 16 * n);
        q.dec = (uint8_t*)carve((size_t)std::max(N - 1, 1) * n);
        fast_ids.push_back(j);
      } else {
        q.sint = (double2*)carve((size_t)std::max(N - 1, 1) * 16 * 16 * n);
        q.sleft = q.needL ? (double2*)carve((size_t)N * 16 * 16 * n) : nullptr;
        q.sright = q.needR ? (double2*)carve((size_t)N * 16 * 16 * n) : nullptr;
        gen_ids.push_back(j);
      }
      offm[j + 1] = offm[j] + (long)N * n;
    }
    // parameter blocks: all items (mode kernels), then the forward-only and general subsets
    const int nf = (int)fast_ids.size(), ng = (int)gen_ids.size();
    std::vector<TransferParams> all(m);
    for (int j = 0; j < m; ++j) all[j] = ps[items[j]];
    std::memcpy(hp, all.data(), sizeof(TransferParams) * m);
    offs[0] = 0;
    offg[0] = 0;
    offi[0] = 0;
    std::vector<TransferParams> pf, pg;
    for (int j = 0; j < nf; ++j) {
      const TransferParams& q = all[fast_ids[j]];
      pf.push_back(q);
      offs[j + 1] = offs[j] + q.n;
      offi[j + 1] = offi[j] + (long)(q.nL - 1) * q.n;
    }
    for (int j = 0; j < ng; ++j) { pg.push_back(all[gen_ids[j]]); offg[j + 1] = offg[j] + all[gen_ids[j]].n; }
    const size_t blk = sizeof(TransferParams) * m + 4 * sizeof(long) * (m + 1);
    TransferParams* hpf = (TransferParams*)(h + blk);
    TransferParams* hpg = hpf + nf;
    if (nf) std::memcpy(hpf, pf.data(), sizeof(TransferParams) * nf);
    if (ng) std::memcpy(hpg, pg.data(), sizeof(TransferParams) * ng);
    const size_t tot = blk + sizeof(TransferParams) * (nf + ng);
    WS(dpar, char, "tb_params", tot);
    CK(cudaMemcpyAsync(dpar, h, tot, cudaMemcpyHostToDevice, ctx->stream));
    if (!ctx->stage_ev) CK(cudaEventCreateWithFlags(&ctx->stage_ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ctx->stage_ev, ctx->stream));
    staged = true;
    const TransferParams* dp = (const TransferParams*)dpar;
    const long* doffm = (const long*)(dp + m);
    const long* doffs = doffm + (m + 1);
    const long* doffg = doffs + (m + 1);
    const long* doffi = doffg + (m + 1);
    const TransferParams* dpf = (const TransferParams*)(dpar + blk);
    const TransferParams* dpg = dpf + nf;
    CK(LAUNCH("k_layer_modes", launch_transfer_batch(0, dp, doffm, m, offm[m], ctx->stream)));
    CK(LAUNCH("k_layer_modes_qr", launch_transfer_batch(1, dp, doffm, m, offm[m], ctx->stream)));
    if (nf) {
      if (offi[nf]) CK(LAUNCH("k_iface", launch_transfer_batch(6, dpf, doffi, nf, offi[nf], ctx->stream)));
      CK(LAUNCH("k_seeds", launch_transfer_batch(5, dpf, doffs, nf, offs[nf], ctx->stream)));
      CK(LAUNCH("k_scan", launch_transfer_batch(7, dpf, doffs, nf, offs[nf], ctx->stream)));
    }
    if (ng) CK(LAUNCH("k_chain", launch_transfer_batch(3, dpg, doffg, ng, offg[ng], ctx->stream)));
  }
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return abort_all(fail(ctx, YTF_ERR_CUDA, cudaGetErrorString(e)));
  prof_collect(ctx);
  for (int i = 0; i < nb; ++i) out[i] = cs[i];
  return YTF_OK;
}

int ytf_cache_destroy(ytf_cache* c) {
  if (!c) return YTF_OK;
  ytf_ctx* ctx = c->ctx;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (c->block) {
    if (ctx->closing) cudaFree(c->block);
    else ctx->pool.emplace(c->block_bytes, c->block);
  }
  delete c;
  ctx_release(ctx);
  return YTF_OK;
}

int ytf_cache_info(const ytf_cache* c, long* n_nodes, int* n_obs, int* obs_layers, int* is2d, int* rotation) {
  if (!c) return YTF_ERR_ARG;
  if (n_nodes) *n_nodes = c->n;
  if (n_obs) *n_obs = c->nobs;
  if (obs_layers)
    for (int i = 0; i < c->nobs; ++i) obs_layers[i] = c->obs[i];
  if (is2d) *is2d = c->is2d;
  if (rotation) *rotation = c->rotation;
  return YTF_OK;
}

int ytf_cache_status(ytf_ctx* ctx, const ytf_cache* c, unsigned char* valid, unsigned char* tvalid, unsigned char* status) {
  if (!ctx || !c) return YTF_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  if (valid) CK(cudaMemcpyAsync(valid, c->d_valid, c->n, cudaMemcpyDeviceToHost, ctx->stream));
  if (tvalid) CK(cudaMemcpyAsync(tvalid, c->d_tvalid, (size_t)c->n * c->nobs, cudaMemcpyDeviceToHost, ctx->stream));
  if (status) CK(cudaMemcpyAsync(status, c->d_status, c->n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return YTF_OK;
}

int ytf_cache_export(ytf_ctx* ctx, const ytf_cache* c, double* T, double* Qf, double* Qb, double* sf, double* sb,
                     double* basis) {
  if (!ctx || !c) return YTF_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  long n = c->n;
  auto fetch = [&](const double2* dsrc, long elems, long nn, double* dst, bool per_obs, int no) -> int {
    // device SoA [o][e][n] -> host AoS [o][n][e]
    std::vector<double2> h((size_t)elems * nn * no);
    cudaError_t e = cudaMemcpy(h.data(), dsrc, sizeof(double2) * h.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(ctx, YTF_ERR_CUDA, cudaGetErrorString(e));
    for (int o = 0; o < no; ++o)
      for (long k = 0; k < nn; ++k)
        for (long el = 0; el < elems; ++el) {
          double2 v = h[((size_t)o * elems + el) * nn + k];
          size_t di = (((size_t)o * nn + k) * elems + el) * 2;
          dst[di] = v.x;
          dst[di + 1] = v.y;
        }
    (void)per_obs;
    return YTF_OK;
  };
  CK(cudaStreamSynchronize(ctx->stream));
  int rc;
  if (T && (rc = fetch(c->d_T, 16, n, T, true, c->nobs))) return rc;
  if (Qf && (rc = fetch(c->d_Qf, 2, n, Qf, false, 1))) return rc;
  if (Qb && (rc = fetch(c->d_Qb, 2, n, Qb, false, 1))) return rc;
  if (sf && (rc = fetch(c->d_sf, 6, n, sf, false, 1))) return rc;
  if (sb && (rc = fetch(c->d_sb, 6, n, sb, false, 1))) return rc;
  if (basis && (rc = fetch(c->d_basis, 16, n, basis, true, c->nobs))) return rc;
  return YTF_OK;
}

// the synthesis parameters of closed_form_G(cache, obs_layer, zsrc_local, ...; terms) with
// its argument checks (z rows left unset)
static int synth_setup(ytf_ctx* ctx, const ytf_cache* c, int obs_layer, double zsrc_local, int terms, int nz,
                       SynthParams& sp) {
  int oi = c->oidx(obs_layer);
  if (oi < 0)
    return fail(ctx, YTF_ERR_ARG, "amplitude_at: obs_layer=" + std::to_string(obs_layer) +
                                      " not in this cache's obs_layers " + obs_str(c->obs, c->nobs));
  if (terms < 0 || terms > 4)
    return fail(ctx, YTF_ERR_ARG, "closed_form_G: terms must be :all, :direct, :scattered, :toeplitz or :hankel");
  bool same = obs_layer == c->src;
  if ((terms == YTF_TERMS_TOEPLITZ || terms == YTF_TERMS_HANKEL || terms == YTF_TERMS_DIRECT) && !same)
    return fail(ctx, YTF_ERR_ARG, "closed_form_G: terms needs obs_layer == source_layer (" + std::to_string(c->src) +
                                      "), got " + std::to_string(obs_layer));
  double zpos = c->src == 1 ? c->d_src - zsrc_local : zsrc_local;
  const double se = 1.4901161193847656e-08;
  if (!(-se <= zpos && zpos <= c->d_src + se))
    return fail(ctx, YTF_ERR_ARG, "amplitude_at: zsrc_local=" + std::to_string(zsrc_local) + " outside [0," +
                                      std::to_string(c->d_src) + "]");
  std::memset(&sp, 0, sizeof(sp));
  CacheView& v = sp.c;
  v.n = c->n; v.Nk = c->Nk; v.Np = c->Np; v.src = c->src; v.d_src = c->d_src;
  v.kr = c->d_kr; v.wr = c->d_wr; v.phi = c->d_phi; v.wphi = c->d_wphi;
  v.kri = c->d_kri; v.wri = c->d_wri;
  v.valid = c->d_valid;
  v.tvalid = c->d_tvalid + (size_t)oi * c->n;
  v.T = c->d_T + (size_t)oi * 16 * c->n;
  v.Qf = c->d_Qf; v.Qb = c->d_Qb; v.sf = c->d_sf; v.sb = c->d_sb;
  v.basis = c->d_basis + (size_t)oi * 16 * c->n;
  sp.same = same;
  switch (terms) {
    case YTF_TERMS_ALL: sp.uf_F = sp.ub_F = sp.uf_B = sp.ub_B = 1.0; sp.with_direct = same; break;
    case YTF_TERMS_SCATTERED: sp.uf_F = sp.ub_F = sp.uf_B = sp.ub_B = 1.0; sp.with_direct = 0; break;
    case YTF_TERMS_DIRECT: sp.with_direct = 1; break;
    case YTF_TERMS_TOEPLITZ: sp.uf_F = 1.0; sp.ub_B = 1.0; sp.with_direct = 1; break;
    case YTF_TERMS_HANKEL: sp.ub_F = 1.0; sp.uf_B = 1.0; sp.with_direct = 0; break;
  }
  sp.zpos = zpos;
  sp.d_obs = c->d_layer[obs_layer - 1];
  sp.nz = nz;
  return YTF_OK;
}

// P_n (n = 0, 1, 2; 26 nz real columns x nr radii) of the 1D synthesis over the nodes of sp.c:
// the per-node coefficient columns (k_coef1d) and the three order contractions -- complex J_n
// with FP64 GEMMs on a deformed contour, the int8x3 tensor-core pipeline, or FP64 GEMMs
static int synth1d_P(ytf_ctx* ctx, const SynthParams& sp, int nz, int nr, const double* drho, int precision, int nsm,
                     const GreenBatch* gb, double* P0, double* P1, double* P2) {
  const long nk = sp.c.n;
  WS(amp1, double2, "g_amp", (size_t)12 * nk);
  const bool i8 = precision == YTF_PREC_INT8X3;
  // FP64 coefficient columns for the FP64 contractions, FP32 ones for the int8x3 digits
  double *C0 = nullptr, *C1 = nullptr, *C2 = nullptr;
  float *F0 = nullptr, *F1 = nullptr, *F2 = nullptr;
  if (i8) {
    WS(Cf, float, "g_Cf", (size_t)C1D_RT * nz * nk);
    F0 = Cf; F1 = Cf + (size_t)C1D_OFF1 * nz * nk; F2 = Cf + (size_t)C1D_OFF2 * nz * nk;
    CK(LAUNCH("k_coef1d", launch_coef1d_amp(sp, amp1, F0, F1, F2, ctx->stream)));
  } else {
    WS(C, double, "g_C", (size_t)C1D_RT * nz * nk);
    C0 = C; C1 = C + (size_t)C1D_OFF1 * nz * nk; C2 = C + (size_t)C1D_OFF2 * nz * nk;
    CK(LAUNCH("k_coef1d", launch_coef1d_amp(sp, amp1, C0, C1, C2, ctx->stream)));
  }
    if (sp.c.kri && i8) {
      // nodes on a deformed contour, int8 tensor cores: the complex J_n(kρ ρ) tables (FP64),
      // their real and imaginary parts as digit images fixed point per (order, slice, radius)
      // relative to the slice's largest part, two int8x3 contractions per order against the
      // FP32 coefficient columns (Re J and Im J), then the complex combine as the FP64 path
      const float* Cn8[3] = {F0, F1, F2};
      double* Pn8[3] = {P0, P1, P2};
      const int Nn8[3] = {C1D_R0 * nz, C1D_R1 * nz, C1D_R2 * nz};
      unsigned* err = gb ? gb->err : nullptr;
      if (!err) {
        WS(e1, unsigned, "g_tc_err", 1);
        err = e1;
        CK(cudaMemsetAsync(err, 0, sizeof(unsigned), ctx->stream));
      }
      WS(Jc, double, "g_Jc", 6 * (size_t)nr * nk);
      CK(LAUNCH("k_bessel_c", launch_bessel_c(sp.c.kr, sp.c.kri, nk, drho, nr, Jc, ctx->stream)));
      long kchunk;
      {
        const int ct0 = bessel_i8_ctile(Nn8[0]);
        const long tiles = (long)((nr + 127) / 128) * ((Nn8[0] + ct0 - 1) / ct0);
        const long want = std::max(1L, (long)nsm / tiles);
        kchunk = (nk + want - 1) / want;
        kchunk = std::min(16384L, std::max(64L, ((kchunk + 63) / 64) * 64));
      }
      const int nchunk = (int)((nk + kchunk - 1) / kchunk);
      const size_t nst = (size_t)(kchunk / 64);
      const size_t abytes = (size_t)((nr + 127) / 128) * nchunk * nst * bessel_i8_stage_bytes_a();
      WS(Ai, uint8_t, "g_bic_a", 6 * abytes);
      WS(rs, double, "g_bic_rs", 3 * (size_t)nchunk * nr);
      uint8_t* imgs[6];
      for (int i = 0; i < 6; ++i) imgs[i] = Ai + i * abytes;
      BesselI8 lay;
      std::memset(&lay, 0, sizeof(lay));
      lay.M = nr; lay.K = nk; lay.ntile_m = (nr + 127) / 128; lay.kchunk = kchunk; lay.nchunk = nchunk;
      CK(LAUNCH("k_bessel_i8", launch_jtable_images(lay, Jc, rs, imgs, ctx->stream)));
      const size_t pab = (size_t)nr * C1D_RMAX * nz;
      WS(Pab, double, "g_Pab", 2 * pab);
      for (int o = 0; o < 3; ++o) {
        BesselI8 bp;
        std::memset(&bp, 0, sizeof(bp));
        bp.M = nr; bp.N = Nn8[o]; bp.K = nk; bp.order = o;
        bp.ctile = bessel_i8_ctile(bp.N);
        bp.Np = ((bp.ctile + 15) / 16) * 16;
        bp.ntile_n = (bp.N + bp.ctile - 1) / bp.ctile;
        bp.ntile_m = (nr + 127) / 128;
        bp.kchunk = kchunk;
        bp.nchunk = nchunk;
        WS(Bi, uint8_t, "g_bi_b", (size_t)bp.ntile_n * bp.nchunk * nst * bessel_i8_stage_bytes_b(bp.Np));
        WS(cm, unsigned long long, "g_bi_cmax", (size_t)bp.nchunk * bp.N);
        WS(pt, double, "g_bi_part", (size_t)bp.nchunk * bp.N * nr);
        bp.kr = sp.c.kr; bp.rho = drho; bp.C = Cn8[o]; bp.ldc = nk;
        bp.Bimg = Bi; bp.colmax = cm; bp.partial = pt; bp.err = err;
        bp.wait_limit = ctx->wait_limit;
        bp.aimg_ready = 1;
        bp.rowscale = rs + (size_t)o * nchunk * nr;
        for (int part = 0; part < 2; ++part) {
          bp.Aimg = imgs[2 * o + part];
          CK(LAUNCH("k_bessel_i8", launch_bessel_i8(bp, Pab + (size_t)part * pab, ctx->stream)));
        }
        CK(LAUNCH("k_combine_complex", launch_combine_complex(nr, Nn8[o], Pab, Pab + pab, Pn8[o], ctx->stream)));
      }
      if (!gb) {
        unsigned herr = 0;
        CK(cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (herr) return fail(ctx, YTF_ERR_CUDA, "closed_form_G: a tensor-core pipeline wait timed out");
      }
      return YTF_OK;
    }
    if (sp.c.kri) {
      // nodes on a deformed contour: complex J_n(kρ ρ) tables, two FP64 GEMMs per order
      // (Re J and Im J against the real/imaginary coefficient columns), then the complex combine
      WS(Jc, double, "g_Jc", 6 * (size_t)nr * nk);
      CK(LAUNCH("k_bessel_c", launch_bessel_c(sp.c.kr, sp.c.kri, nk, drho, nr, Jc, ctx->stream)));
      const double* Cn[3] = {C0, C1, C2};
      double* Pn[3] = {P0, P1, P2};
      const int Nn[3] = {C1D_R0 * nz, C1D_R1 * nz, C1D_R2 * nz};
      const size_t pab = (size_t)nr * C1D_RMAX * nz;
      WS(Pab, double, "g_Pab", 2 * pab);
      for (int o = 0; o < 3; ++o) {
        long tiles = (long)((nr + 127) / 128) * ((Nn[o] + 127) / 128);
        long want = (2L * nsm + tiles - 1) / tiles;
        int sp0 = dgemm_splits((int)nk, (int)std::max(1L, std::min(want, std::max(1L, nk / 256))));
        WS(Pp, double, "g_partial", (size_t)sp0 * nr * Nn[o]);
        for (int part = 0; part < 2; ++part) {
          const double* Jp = Jc + (size_t)(2 * o + part) * nr * nk;
          CK(LAUNCH("k_dgemm_nt", launch_dgemm_nt(nr, Nn[o], (int)nk, Jp, Cn[o], Pp, sp0, ctx->stream)));
          CK(LAUNCH("k_reduce_splits", launch_reduce_splits((long)nr * Nn[o], sp0, Pp,
                                                            Pab + (size_t)part * pab, ctx->stream)));
        }
        CK(LAUNCH("k_combine_complex", launch_combine_complex(nr, Nn[o], Pab, Pab + pab, Pn[o], ctx->stream)));
      }
      return YTF_OK;
    }
    if (i8) {
      // int8 tensor cores: J_n(kρ) and the coefficient columns as fixed-point digit images,
      // exact INT32 accumulation, FP64 sum of the node slices into P_n
      const float* Cn8[3] = {F0, F1, F2};
      double* Pn8[3] = {P0, P1, P2};
      const int Nn8[3] = {C1D_R0 * nz, C1D_R1 * nz, C1D_R2 * nz};
      unsigned* err = gb ? gb->err : nullptr;
      if (!err) {
        WS(e1, unsigned, "g_tc_err", 1);
        err = e1;
        CK(cudaMemsetAsync(err, 0, sizeof(unsigned), ctx->stream));
      }
      // one node slicing for the three orders (that of order 0, the widest), so the J_n
      // digit images of all three come from one Bessel evaluation per (ρ, k)
      long kchunk;
      {
        const int ct0 = bessel_i8_ctile(Nn8[0]);
        const long tiles = (long)((nr + 127) / 128) * ((Nn8[0] + ct0 - 1) / ct0);
        const long want = std::max(1L, (long)nsm / tiles);
        kchunk = (nk + want - 1) / want;
        kchunk = std::min(16384L, std::max(64L, ((kchunk + 63) / 64) * 64));
      }
      const int nchunk = (int)((nk + kchunk - 1) / kchunk);
      const size_t nst = (size_t)(kchunk / 64);
      const size_t abytes = (size_t)((nr + 127) / 128) * nchunk * nst * bessel_i8_stage_bytes_a();
      WS(A0i, uint8_t, "g_bi_a0", abytes);
      WS(A1i, uint8_t, "g_bi_a1", abytes);
      WS(A2i, uint8_t, "g_bi_a2", abytes);
      uint8_t* Aord[3] = {A0i, A1i, A2i};
      WS(kminb, double, "g_bi_kmin", nchunk);
      CK(LAUNCH("k_bessel_i8", launch_slice_kmin(sp.c.kr, nk, kchunk, nchunk, kminb, ctx->stream)));
      for (int o = 0; o < 3; ++o) {
        BesselI8 bp;
        std::memset(&bp, 0, sizeof(bp));
        bp.M = nr; bp.N = Nn8[o]; bp.K = nk; bp.order = o;
        bp.ctile = bessel_i8_ctile(bp.N);
        bp.Np = ((bp.ctile + 15) / 16) * 16;
        bp.ntile_n = (bp.N + bp.ctile - 1) / bp.ctile;
        bp.ntile_m = (nr + 127) / 128;
        bp.kchunk = kchunk;
        bp.nchunk = nchunk;
        WS(Bi, uint8_t, "g_bi_b", (size_t)bp.ntile_n * bp.nchunk * nst * bessel_i8_stage_bytes_b(bp.Np));
        WS(cm, unsigned long long, "g_bi_cmax", (size_t)bp.nchunk * bp.N);
        WS(pt, double, "g_bi_part", (size_t)bp.nchunk * bp.N * nr);
        bp.kr = sp.c.kr; bp.rho = drho; bp.C = Cn8[o]; bp.ldc = nk;
        bp.Aimg = Aord[o]; bp.Bimg = Bi; bp.colmax = cm; bp.partial = pt; bp.err = err;
        bp.wait_limit = ctx->wait_limit;
        bp.kmin = kminb;
        if (o == 0) CK(LAUNCH("k_bessel_i8", launch_bessel_i8_aimg3(bp, A0i, A1i, A2i, ctx->stream)));
        bp.aimg_ready = 1;
        CK(LAUNCH("k_bessel_i8", launch_bessel_i8(bp, Pn8[o], ctx->stream)));
      }
      if (!gb) {
        unsigned herr = 0;
        CK(cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (herr) return fail(ctx, YTF_ERR_CUDA, "closed_form_G: a tensor-core pipeline wait timed out");
      }
      return YTF_OK;
    }
    WS(J, double, "g_J", 3 * (size_t)nr * nk);
    double *J0 = J, *J1 = J + (size_t)nr * nk, *J2 = J + 2 * (size_t)nr * nk;
    CK(LAUNCH("k_bessel", launch_bessel(sp.c.kr, nk, drho, nr, J0, J1, J2, ctx->stream)));
    auto splits_for = [&](int M, int N) {
      long tiles = (long)((M + 127) / 128) * ((N + 127) / 128);
      long want = (2L * nsm + tiles - 1) / tiles;
      long maxs = std::max(1L, nk / 256);
      return (int)std::max(1L, std::min(want, maxs));
    };
    const int Nn[3] = {C1D_R0 * nz, C1D_R1 * nz, C1D_R2 * nz};
    const int sps[3] = {splits_for(nr, Nn[0]), splits_for(nr, Nn[1]), splits_for(nr, Nn[2])};
    size_t part = 0;
    for (int o = 0; o < 3; ++o) part = std::max(part, (size_t)sps[o] * nr * Nn[o]);
    WS(Pp, double, "g_partial", part);
    const double* Jn[3] = {J0, J1, J2};
    const double* Cn[3] = {C0, C1, C2};
    double* Pn[3] = {P0, P1, P2};
    for (int o = 0; o < 3; ++o) {
      int sp_ = dgemm_splits((int)nk, sps[o]);
      CK(LAUNCH("k_dgemm_nt", launch_dgemm_nt(nr, Nn[o], (int)nk, Jn[o], Cn[o], Pp, sp_, ctx->stream)));
      CK(LAUNCH("k_reduce_splits", launch_reduce_splits((long)nr * Nn[o], sp_, Pp, Pn[o], ctx->stream)));
    }
  return YTF_OK;
}

// the node range [b0, b0 + nb) of a 1D cache as a cache view of its own: per-node scalars by
// pointer offset, the multi-row arrays (T, Qf, Qb, sf, sb, basis: rows of n entries) copied
// into a compact [row][nb] block with one strided copy each
static int node_chunk_view(ytf_ctx* ctx, const CacheView& v, long b0, long nb, double2* buf, CacheView& out) {
  out = v;
  out.n = nb;
  out.Nk = nb;
  out.kr = v.kr + b0;
  out.wr = v.wr + b0;
  if (v.kri) { out.kri = v.kri + b0; out.wri = v.wri + b0; }
  out.valid = v.valid + b0;
  out.tvalid = v.tvalid + b0;
  struct Rows { const double2* src; int rows; const double2** dst; } rows[6] = {
      {v.T, 16, &out.T}, {v.Qf, 2, &out.Qf}, {v.Qb, 2, &out.Qb}, {v.sf, 6, &out.sf}, {v.sb, 6, &out.sb},
      {v.basis, 16, &out.basis}};
  double2* d = buf;
  for (auto& r : rows) {
    CK(cudaMemcpy2DAsync(d, sizeof(double2) * nb, r.src + b0, sizeof(double2) * v.n, sizeof(double2) * nb, r.rows,
                         cudaMemcpyDeviceToDevice, ctx->stream));
    *r.dst = d;
    d += (size_t)r.rows * nb;
  }
  return YTF_OK;
}

// nodes per pass of the 1D synthesis: the coefficient columns and digit images of a pass take
// about 18 KB per node at 64 heights, so a pass stays within a few GB whatever the rule's size
constexpr long SYNTH1D_NODE_CHUNK = 1L << 18;

static int green_impl(ytf_ctx* ctx, const ytf_cache* c, int obs_layer, double zsrc_local, int nz, const double* z_obs,
                      int nx, const double* xs, int ny, const double* ys, int terms, int precision, double* out,
                      int out_is_device, const GreenBatch* gb) {
  if (!ctx || !c || !out) return YTF_ERR_ARG;
  if (c->ctx != ctx) return fail(ctx, YTF_ERR_STATE, "closed_form_G: cache belongs to another context");
  SynthParams sp;
  {
    int rc0 = synth_setup(ctx, c, obs_layer, zsrc_local, terms, nz, sp);
    if (rc0) return rc0;
  }
  if (precision != YTF_PREC_FP64 && precision != YTF_PREC_SPLIT_BF16 && precision != YTF_PREC_INT8X3)
    return fail(ctx, YTF_ERR_ARG, "closed_form_G: unknown precision mode");
  if (nz < 0 || nx < 0 || ny < 0) return fail(ctx, YTF_ERR_ARG, "closed_form_G: negative grid size");
  CK(cudaSetDevice(ctx->device));
  long npix = (long)nx * ny;
  long nout = npix * nz * 9;
  if (nout == 0) return YTF_OK;
  CacheView& v = sp.c;
  const double *dzo, *dxs, *dys;
  int rc;
  if (gb) {
    dzo = gb->dzo; dxs = gb->dxs; dys = gb->dys;
  } else {
    WS(uzo, double, "g_zo", nz);
    WS(uxs, double, "g_xs", nx);
    WS(uys, double, "g_ys", ny);
    if ((rc = upload(ctx, uzo, z_obs, 8 * (size_t)nz))) return rc;
    if ((rc = upload(ctx, uxs, xs, 8 * (size_t)nx))) return rc;
    if ((rc = upload(ctx, uys, ys, 8 * (size_t)ny))) return rc;
    dzo = uzo; dxs = uxs; dys = uys;
  }
  sp.zo = dzo;
  double2* G;
  if (out_is_device) {
    G = (double2*)out;
  } else {
    WS(g, double2, "g_out", nout);
    G = g;
  }
  int nsm = 148;
  {
    int dev = ctx->device;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  if (c->n == 0) {  // an empty rule integrates to zero
    CK(cudaMemsetAsync(G, 0, sizeof(double2) * nout, ctx->stream));
  } else if (!c->is2d) {
    std::vector<double> ur;
    std::vector<int> rmap;
    radii_map(nx, xs, ny, ys, ur, rmap);
    int nr = (int)ur.size();
    long nk = c->n;
    const double* drho;
    const int* drmap;
    if (gb && gb->drho) {
      drho = gb->drho;
      drmap = gb->drmap;
    } else {
      WS(urho, double, "g_rho", nr);
      WS(urmap, int, "g_rmap", npix);
      if ((rc = upload(ctx, urho, ur.data(), 8 * (size_t)nr))) return rc;
      if ((rc = upload(ctx, urmap, rmap.data(), 4 * (size_t)npix))) return rc;
      drho = urho;
      drmap = urmap;
    }
    WS(P, double, "g_P", (size_t)C1D_RT * nz * nr);
    double *P0 = P, *P1 = P + (size_t)C1D_OFF1 * nz * nr, *P2 = P + (size_t)C1D_OFF2 * nz * nr;
    if (nk <= SYNTH1D_NODE_CHUNK) {
      if ((rc = synth1d_P(ctx, sp, nz, nr, drho, precision, nsm, gb, P0, P1, P2))) return rc;
    } else {
      // G is linear in the node sum: the rule in passes of at most SYNTH1D_NODE_CHUNK nodes,
      // their P_n summed (the reference sums closed_form_G over node chunks the same way,
      // chunked_2d, mod_ClosedFormGrid.jl:449-467)
      const size_t np = (size_t)C1D_RT * nz * nr;
      WS(Pacc, double, "g_Pacc", np);
      WS(Pc, double, "g_Pchunk", np);
      WS(cbuf, double2, "g_chunk_cache", (size_t)48 * SYNTH1D_NODE_CHUNK);
      CK(cudaMemsetAsync(Pacc, 0, sizeof(double) * np, ctx->stream));
      for (long b0 = 0; b0 < nk; b0 += SYNTH1D_NODE_CHUNK) {
        const long nb = std::min(SYNTH1D_NODE_CHUNK, nk - b0);
        SynthParams spc = sp;
        if ((rc = node_chunk_view(ctx, sp.c, b0, nb, cbuf, spc.c))) return rc;
        if ((rc = synth1d_P(ctx, spc, nz, nr, drho, precision, nsm, gb, Pc, Pc + (size_t)C1D_OFF1 * nz * nr,
                            Pc + (size_t)C1D_OFF2 * nz * nr)))
          return rc;
        CK(LAUNCH("k_add", launch_add(np, Pc, Pacc, ctx->stream)));
      }
      CK(cudaMemcpyAsync(P, Pacc, sizeof(double) * np, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    CK(LAUNCH("k_assemble1d", launch_assemble1d(nx, ny, nz, dxs, dys, drmap, nr, P0, P1, P2, G, ctx->stream)));
  } else {
    int ncol = 9 * nz;
    WS(S, double2, "g_S", (size_t)ncol * c->n);
    WS(amp, double2, "g_amp", (size_t)12 * c->n);
    if (precision == YTF_PREC_INT8X3) {
      // int8 tensor cores: FP32 phase tables, fixed-point digits, exact INT32 accumulation,
      // FP64 reduction of the node slices
      LateralI8 lp;
      std::memset(&lp, 0, sizeof(lp));
      lp.npix = npix; lp.n = c->n; lp.nx = nx; lp.ny = ny; lp.ncol = ncol;
      lp.ctile = lateral_i8_ctile(ncol);
      lp.Np = ((2 * lp.ctile + 15) / 16) * 16;
      lp.ntile = (ncol + lp.ctile - 1) / lp.ctile;
      lp.S = S;
      // one CTA per SM: (pixel tiles x column tiles) x node slices fill one wave; a slice
      // holds at most 16384 nodes so the INT32 accumulators cannot overflow
      long tiles = ((npix + 127) / 128) * lp.ntile;
      long want = std::max(1L, (long)nsm / tiles);
      long kchunk = (c->n + want - 1) / want;
      kchunk = std::min(16384L, std::max(32L, ((kchunk + 31) / 32) * 32));
      lp.kchunk = kchunk;
      lp.nchunk = (int)((c->n + kchunk - 1) / kchunk);
      lp.n_pad = (long)lp.nchunk * kchunk;
      WS(Px, float2, "g_px", (size_t)lp.n_pad * nx);
      WS(Py, float2, "g_py", (size_t)lp.n_pad * ny);
      // evenly spaced x and y (to 4 ulp of the progression): the tables by recurrence
      double ev[4];
      bool even = xs && ys && nx >= 1 && ny >= 1;
      auto spaced = [&](const double* v, int m, double& a0, double& d) {
        a0 = v[0];
        d = m > 1 ? (v[m - 1] - v[0]) / (m - 1) : 0.0;
        const double tol = 4 * 2.220446049250313e-16 * std::max(std::fabs(v[0]), std::fabs(v[m - 1]));
        bool ok = std::isfinite(d);
        for (int r = 0; r < m && ok; ++r) ok = std::fabs(v[r] - (v[0] + r * d)) <= tol;
        return ok;
      };
      if (even) even = spaced(xs, nx, ev[0], ev[1]) && spaced(ys, ny, ev[2], ev[3]);
      CK(LAUNCH("k_phase_tables", launch_phase_tables_pad(v, nx, ny, dxs, dys, lp.n_pad, Px, Py, ctx->stream,
                                                          even ? ev : nullptr)));
      lp.Px = Px; lp.Py = Py;
      WS(Bq, uint8_t, "g_i8_b", (size_t)lp.ntile * lp.nchunk * (kchunk / 32) * lateral_i8_stage_bytes(lp.Np));
      WS(cmax, unsigned long long, "g_i8_cmax", (size_t)lp.nchunk * ncol);
      CK(cudaMemsetAsync(cmax, 0, sizeof(unsigned long long) * lp.nchunk * ncol, ctx->stream));
      CK(LAUNCH("k_strengths2d", launch_strengths2d(sp, S, ctx->stream, cmax, kchunk, amp)));
      WS(Gp, double2, "g_partial2", (size_t)lp.nchunk * npix * ncol);
      unsigned* err = gb ? gb->err : nullptr;
      if (!err) {
        WS(e1, unsigned, "g_tc_err", 1);
        err = e1;
        CK(cudaMemsetAsync(err, 0, sizeof(unsigned), ctx->stream));
      }
      lp.Bq = Bq; lp.colmax = cmax; lp.partial = Gp; lp.err = err;
      lp.wait_limit = ctx->wait_limit;
      CK(LAUNCH("k_lateral_i8", launch_lateral_i8(lp, ctx->stream)));
      CK(LAUNCH("k_reduce_splits2", launch_reduce_splits2(npix * ncol, lp.nchunk, Gp, G, ctx->stream)));
      if (!gb) {
        unsigned herr = 0;
        CK(cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (herr) return fail(ctx, YTF_ERR_CUDA, "closed_form_G: a tensor-core pipeline wait timed out");
      }
    } else {
      CK(LAUNCH("k_strengths2d", launch_strengths2d(sp, S, ctx->stream, nullptr, 0, amp)));
      if (precision == YTF_PREC_SPLIT_BF16) {
        // tensor cores: FP32 phase tables, split-BF16 contraction, FP64 reduction of the slices
        WS(Px, float2, "g_px", (size_t)c->n * nx);
        WS(Py, float2, "g_py", (size_t)c->n * ny);
        CK(LAUNCH("k_phase_tables", launch_phase_tables(v, nx, ny, dxs, dys, Px, Py, ctx->stream)));
        LateralTC lp;
        std::memset(&lp, 0, sizeof(lp));
        lp.npix = npix; lp.n = c->n; lp.nx = nx; lp.ny = ny; lp.ncol = ncol;
        lp.ctile = lateral_tc_ctile(ncol);
        lp.Np = ((2 * lp.ctile + 15) / 16) * 16;
        lp.Px = Px; lp.Py = Py; lp.S = S;
        // one CTA per SM (tensor memory, registers): tiles x node slices fill one wave
        long tiles = ((npix + 127) / 128) * ((ncol + lp.ctile - 1) / lp.ctile);
        long want = std::max(1L, (long)nsm / tiles);
        long kchunk = (c->n + want - 1) / want;
        kchunk = std::max(16L, ((kchunk + 15) / 16) * 16);
        int splits = (int)((c->n + kchunk - 1) / kchunk);
        lp.kchunk = kchunk;
        WS(Gp, double2, "g_partial2", (size_t)splits * npix * ncol);
        unsigned* err = gb ? gb->err : nullptr;
        if (!err) {
          WS(e1, unsigned, "g_tc_err", 1);
          err = e1;
          CK(cudaMemsetAsync(err, 0, sizeof(unsigned), ctx->stream));
        }
        lp.partial = Gp;
        lp.err = err;
        CK(LAUNCH("k_lateral_tc", launch_lateral_tc(lp, splits, ctx->stream)));
        CK(LAUNCH("k_reduce_splits2", launch_reduce_splits2(npix * ncol, splits, Gp, G, ctx->stream)));
        if (!gb) {
          unsigned herr = 0;
          CK(cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
          CK(cudaStreamSynchronize(ctx->stream));
          if (herr) return fail(ctx, YTF_ERR_CUDA, "closed_form_G: a tensor-core pipeline wait timed out");
        }
      } else {
        long tiles = ((npix + 63) / 64) * ((ncol + 31) / 32);
        long want = (4L * nsm + tiles - 1) / tiles;
        int splits = (int)std::max(1L, std::min(want, std::max(1L, c->n / 512)));
        splits = lateral_splits(c->n, splits);
        WS(Gp, double2, "g_partial2", (size_t)splits * npix * ncol);
        CK(LAUNCH("k_lateral", launch_lateral(v, nx, ny, dxs, dys, ncol, S, Gp, splits, ctx->stream)));
        CK(LAUNCH("k_reduce_splits2", launch_reduce_splits2(npix * ncol, splits, Gp, G, ctx->stream)));
      }
    }
  }
synthesis_done:
  if (!out_is_device) CK(cudaMemcpyAsync(out, G, sizeof(double2) * nout, cudaMemcpyDeviceToHost, ctx->stream));
  if (!gb) {
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
  }
  return YTF_OK;
}

int ytf_green(ytf_ctx* ctx, const ytf_cache* c, int obs_layer, double zsrc_local, int nz, const double* z_obs, int nx,
              const double* xs, int ny, const double* ys, int terms, int precision, double* out, int out_is_device) {
  return green_impl(ctx, c, obs_layer, zsrc_local, nz, z_obs, nx, xs, ny, ys, terms, precision, out, out_is_device,
                    nullptr);
}

// ------------------------------------------------------------------------------------
// Grouped 1D int8x3 synthesis inside ytf_green_batch: the batch's 1D items of real nodes
// (at most SYNTH1D_GROUP_MAX_NODES nodes) in groups whose workspace stays within the context's
// group bound (ytf_ctx_set_group_bytes, default 4 GiB); each group is seven launches whatever
// its item count (amplitudes, coefficient columns, slice minima, J_n images, coefficient
// images with their slice maxima, contraction, slice sum + assembly), with every item's blocks side by side in each
// grid; items with host outputs get a device G in the group's workspace, copied out after it. Per item the
// arithmetic is the per-item path's; only the node slicing of the contraction differs
// (slices of about SYNTH1D_GROUP_SLICE nodes, whose fixed-point scales are per slice).
// ------------------------------------------------------------------------------------
constexpr long SYNTH1D_GROUP_SLICE = 4096;
// largest item of the grouped path (about 14 KB of workspace per node at 64 heights, so an item
// of this size is a group of its own of ~15 GB); larger rules take the per-item node passes
constexpr long SYNTH1D_GROUP_MAX_NODES = 1L << 20;

struct Group1DLayout {
  int item;
  long nk;
  int nz, nr, ntm;
  long kchunk, ldc;
  int nchunk;
  int N[3], ctile[3], Np[3], ntn[3];
  size_t off_amp, off_C, off_A[3], off_B[3], off_pt[3];
  size_t cm_off[3], cm_bytes;  // slice maxima, in the group's separate maxima block
  size_t off_G;  // device G of an item whose output is host memory (copied out after its group)
  size_t off_kmin;  // [nchunk] smallest node of each slice
  size_t bytes;
};

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

static Group1DLayout group1d_layout(int item, long nk, int nz, int nr, long npix, bool host_out, long slice) {
  Group1DLayout L;
  std::memset(&L, 0, sizeof(L));
  L.item = item; L.nk = nk; L.nz = nz; L.nr = nr;
  L.ntm = (nr + 127) / 128;
  int nchunk = (int)std::max(1L, (nk + slice - 1) / slice);
  long kchunk = (nk + nchunk - 1) / nchunk;
  kchunk = std::min(16384L, std::max(64L, ((kchunk + 63) / 64) * 64));
  L.kchunk = kchunk;
  L.nchunk = (int)((nk + kchunk - 1) / kchunk);
  const size_t nst = (size_t)(kchunk / 64);
  size_t off = 0;
  auto take = [&](size_t b) { size_t o = off; off += align256(b); return o; };
  L.off_amp = take(sizeof(double2) * 12 * (size_t)nk);
  L.ldc = (nk + 3) / 4 * 4;
  L.off_C = take(sizeof(float) * C1D_RT * (size_t)nz * L.ldc);
  for (int o = 0; o < 3; ++o) {
    L.N[o] = (o == 0 ? C1D_R0 : o == 1 ? C1D_R1 : C1D_R2) * nz;
    L.ctile[o] = bessel_i8_ctile(L.N[o]);
    L.Np[o] = ((L.ctile[o] + 15) / 16) * 16;
    L.ntn[o] = (L.N[o] + L.ctile[o] - 1) / L.ctile[o];
    L.off_A[o] = take((size_t)L.ntm * L.nchunk * nst * bessel_i8_stage_bytes_a());
    L.off_B[o] = take((size_t)L.ntn[o] * L.nchunk * nst * bessel_i8_stage_bytes_b(L.Np[o]));
    L.off_pt[o] = take(sizeof(double) * (size_t)L.nchunk * L.N[o] * nr);
  }
  L.off_G = host_out ? take(sizeof(double2) * 9 * (size_t)npix * nz) : 0;
  L.off_kmin = take(sizeof(double) * (size_t)L.nchunk);
  L.bytes = off;
  size_t cm = 0;
  for (int o = 0; o < 3; ++o) {
    L.cm_off[o] = cm;
    cm += sizeof(unsigned long long) * (size_t)L.nchunk * L.N[o];
  }
  L.cm_bytes = cm;
  return L;
}

// device descriptor block of one group: items, entries and the seven block tables
struct Group1DDesc {
  size_t off_it, off_bp, off_first, bytes;
  int ni;
  long grid[7];

};

static bool group1d_eligible(const ytf_ctx* ctx, const ytf_green_desc& g) {
  const ytf_cache* c = g.cache;
  return c && c->ctx == ctx && !c->is2d && !c->d_kri && c->n > 0 && c->n <= SYNTH1D_GROUP_MAX_NODES &&
         g.precision == YTF_PREC_INT8X3 && g.out && g.nz > 0 && g.nx > 0 && g.ny > 0 && g.xs && g.ys && g.z_obs;
}

int ytf_green_batch(ytf_ctx* ctx, int nb, const ytf_green_desc* d) {
  if (!ctx || nb < 0 || (nb > 0 && !d)) return YTF_ERR_ARG;
  if (nb == 0) return YTF_OK;
  CK(cudaSetDevice(ctx->device));
  // every item's coordinates (and, for 1D items, its distinct radii and pixel -> radius map)
  // in one page-locked block, one upload
  size_t tot = 0;
  bool all1d = nb >= 2;
  for (int i = 0; i < nb; ++i) {
    if (d[i].nz < 0 || d[i].nx < 0 || d[i].ny < 0)
      return fail(ctx, YTF_ERR_ARG, "closed_form_G: negative grid size (batch item " + std::to_string(i) + ")");
    tot += (size_t)d[i].nz + d[i].nx + d[i].ny;
    if (!d[i].cache || d[i].cache->is2d || d[i].cache->ctx != ctx) all1d = false;
  }
  std::vector<std::vector<double>> ur(nb);
  std::vector<std::vector<int>> rmap(nb);
  std::vector<size_t> orho(nb, 0), omap(nb, 0);
  size_t tot_r = 0, tot_m = 0;
  for (int i = 0; i < nb; ++i) {
    if (!d[i].cache || d[i].cache->is2d || !d[i].xs || !d[i].ys) continue;
    radii_map(d[i].nx, d[i].xs, d[i].ny, d[i].ys, ur[i], rmap[i]);
    orho[i] = tot_r;
    omap[i] = tot_m;
    tot_r += ur[i].size();
    tot_m += rmap[i].size();
  }
  const size_t nd = std::max<size_t>(tot + tot_r, 1);  // doubles, then the int maps
  const size_t bytes = 8 * nd + 4 * tot_m;
  // the grouped 1D int8x3 items: layouts, groups within the workspace budget (largest items
  // first, so each grid starts with its longest blocks), descriptor sizes
  std::vector<SynthParams> gsp(nb);
  std::vector<char> grouped(nb, 0);
  std::vector<Group1DLayout> lay;
  {
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
    double ctas = 0.0;  // contraction CTAs of all candidates at one-node slices
    std::vector<int> cand;
    for (int i = 0; i < nb; ++i) {
      if (!group1d_eligible(ctx, d[i]) || ur[i].empty()) continue;
      SynthParams sp;
      if (synth_setup(ctx, d[i].cache, d[i].obs_layer, d[i].zsrc_local, d[i].terms, d[i].nz, sp) != YTF_OK) {
        ctx->err.clear();  // the item takes the per-item path, which reports its error
        continue;
      }
      gsp[i] = sp;
      cand.push_back(i);
      const double ntm = (double)((ur[i].size() + 127) / 128);
      for (int od = 0; od < 3; ++od) {
        const int N = (od == 0 ? C1D_R0 : od == 1 ? C1D_R1 : C1D_R2) * d[i].nz, ct = bessel_i8_ctile(N);
        ctas += ntm * (double)((N + ct - 1) / ct) * (double)d[i].cache->n;
      }
    }
    // slices of SYNTH1D_GROUP_SLICE nodes, finer when that leaves under two CTAs per SM
    long slice = SYNTH1D_GROUP_SLICE;
    if (!cand.empty() && ctas / (double)slice < 2.0 * nsm)
      slice = std::max(64L, std::min(slice, (long)(ctas / (2.0 * nsm)) / 64 * 64));
    for (int i : cand)
      lay.push_back(group1d_layout(i, d[i].cache->n, d[i].nz, (int)ur[i].size(), (long)d[i].nx * d[i].ny,
                                   !d[i].out_is_device, slice));
    std::stable_sort(lay.begin(), lay.end(), [](const Group1DLayout& a, const Group1DLayout& b) { return a.nk > b.nk; });
  }
  std::vector<std::pair<size_t, size_t>> groups;  // [begin, end) into lay
  std::vector<size_t> item_base(lay.size(), 0), item_cm(lay.size(), 0);
  size_t group_ws = 0, group_cm_max = 0;
  for (size_t j = 0, cur = 0, cur_cm = 0; j < lay.size(); ++j) {
    if (groups.empty() || (cur > 0 && cur + lay[j].bytes > ctx->group_bytes)) {
      groups.push_back({j, j});
      cur = cur_cm = 0;
    }
    item_base[j] = cur;
    item_cm[j] = cur_cm;
    cur += lay[j].bytes;
    cur_cm += lay[j].cm_bytes;
    groups.back().second = j + 1;
    group_ws = std::max(group_ws, cur);
    group_cm_max = std::max(group_cm_max, cur_cm);
    grouped[lay[j].item] = 1;
  }
  std::vector<Group1DDesc> gdesc(groups.size());
  const size_t desc_off = align256(bytes);
  size_t desc_bytes = 0;
  for (size_t g = 0; g < groups.size(); ++g) {
    const int ni = (int)(groups[g].second - groups[g].first);
    Group1DDesc& D = gdesc[g];
    D.ni = ni;
    D.off_it = desc_off + desc_bytes;
    D.off_bp = D.off_it + align256(sizeof(Synth1DItem) * ni);
    D.off_first = D.off_bp + align256(sizeof(BesselI8) * 3 * ni);
    D.bytes = align256(sizeof(Synth1DItem) * ni) + align256(sizeof(BesselI8) * 3 * ni) +
              align256(sizeof(long) * (5 * (size_t)(ni + 1) + 2 * (size_t)(3 * ni + 1)));

    desc_bytes += D.bytes;
  }
  const size_t total_bytes = desc_off + desc_bytes;
  double* h = (double*)pinned_staging(ctx, total_bytes);
  if (!h) return fail(ctx, YTF_ERR_NOMEM, "closed_form_G: page-locked staging allocation failed");
  std::vector<size_t> o(nb);
  size_t k = 0;
  for (int i = 0; i < nb; ++i) {
    o[i] = k;
    if (d[i].nz) std::memcpy(h + k, d[i].z_obs, 8 * (size_t)d[i].nz);
    k += d[i].nz;
    if (d[i].nx) std::memcpy(h + k, d[i].xs, 8 * (size_t)d[i].nx);
    k += d[i].nx;
    if (d[i].ny) std::memcpy(h + k, d[i].ys, 8 * (size_t)d[i].ny);
    k += d[i].ny;
  }
  int* hm = (int*)(h + nd);
  for (int i = 0; i < nb; ++i) {
    if (!ur[i].empty()) std::memcpy(h + tot + orho[i], ur[i].data(), 8 * ur[i].size());
    if (!rmap[i].empty()) std::memcpy(hm + omap[i], rmap[i].data(), 4 * rmap[i].size());
  }
  WS(dc, double, "gb_coords", (total_bytes + 7) / 8);
  WS(err, unsigned, "gb_tc_err", 1);
  const int* dm = (const int*)(dc + nd);
  uint8_t* gws = nullptr;
  uint8_t* gcm = nullptr;
  if (group_ws) {
    WSR(w, uint8_t, "gb1_ws", group_ws, ctx->group_bytes);
    WS(wc, uint8_t, "gb1_cmax", group_cm_max);
    gws = w;
    gcm = wc;
  }
  // the groups' descriptors, behind the coordinates in the same staging block and copy
  for (size_t g = 0; g < groups.size(); ++g) {
    Group1DDesc& D = gdesc[g];
    const int ni = D.ni;
    Synth1DItem* hit = (Synth1DItem*)((char*)h + D.off_it);
    BesselI8* hbp = (BesselI8*)((char*)h + D.off_bp);
    long* hf = (long*)((char*)h + D.off_first);
    long* f_ref = hf;
    long* f_coef = f_ref + (ni + 1);
    long* f_aimg = f_coef + (ni + 1);
    long* f_asm = f_aimg + (ni + 1);
    long* f_kmin = f_asm + (ni + 1);
    long* f_bimg = f_kmin + (ni + 1);
    long* f_gemm = f_bimg + (3 * ni + 1);
    long nref = 0, ncoef = 0, naimg = 0, nasm = 0, nbimg = 0, ngemm = 0, nkmin = 0;
    for (int q = 0; q < ni; ++q) {
      const size_t j = groups[g].first + q;
      const Group1DLayout& L = lay[j];
      const int i = L.item;
      uint8_t* base = gws + item_base[j];
      Synth1DItem& it = hit[q];
      std::memset(&it, 0, sizeof(it));
      it.sp = gsp[i];
      it.sp.zo = dc + o[i];
      it.amp = (double2*)(base + L.off_amp);
      it.C = (float*)(base + L.off_C);
      it.ldc = L.ldc;
      it.nx = d[i].nx; it.ny = d[i].ny; it.nr = L.nr;
      it.xs = dc + o[i] + d[i].nz;
      it.ys = dc + o[i] + d[i].nz + d[i].nx;
      it.rmap = dm + omap[i];
      it.G = d[i].out_is_device ? (double2*)d[i].out : (double2*)(base + L.off_G);
      it.nchunk = L.nchunk;
      it.kchunk = L.kchunk;
      {  // evenly spaced heights (to 4 ulp of the progression): rows by recurrence
        const double* zv = d[i].z_obs;
        const int m = d[i].nz;
        const double dz = m > 1 ? (zv[m - 1] - zv[0]) / (m - 1) : 0.0;
        const double tol = 4 * 2.220446049250313e-16 * std::max(std::fabs(zv[0]), std::fabs(zv[m - 1]));
        bool even = m > 1 && std::isfinite(dz) && dz != 0.0;
        for (int r = 0; r < m && even; ++r) even = std::fabs(zv[r] - (zv[0] + r * dz)) <= tol;
        it.dz = even ? dz : 0.0;
      }
      for (int od = 0; od < 3; ++od) it.part[od] = (const double*)(base + L.off_pt[od]);
      const long nkb = (L.nk + 127) / 128;
      f_ref[q] = nref; nref += nkb;
      f_coef[q] = ncoef; ncoef += nkb * ((L.nz + COEF1D_ZB_GROUP - 1) / COEF1D_ZB_GROUP);
      f_aimg[q] = naimg; naimg += ((long)L.ntm * 128 * L.nchunk * (L.kchunk / 4) + 255) / 256;
      f_asm[q] = nasm; nasm += ((long)d[i].nx * d[i].ny * L.nz + 127) / 128;
      f_kmin[q] = nkmin; nkmin += L.nchunk;
      const size_t coff[3] = {0, (size_t)C1D_OFF1 * L.nz * L.ldc, (size_t)C1D_OFF2 * L.nz * L.ldc};
      for (int od = 0; od < 3; ++od) {
        BesselI8& bp = hbp[3 * q + od];
        std::memset(&bp, 0, sizeof(bp));
        bp.M = L.nr; bp.N = L.N[od]; bp.K = L.nk; bp.order = od;
        bp.ctile = L.ctile[od]; bp.Np = L.Np[od];
        bp.ntile_m = L.ntm; bp.ntile_n = L.ntn[od];
        bp.kchunk = L.kchunk; bp.nchunk = L.nchunk;
        bp.kr = gsp[i].c.kr;
        bp.rho = dc + tot + orho[i];
        bp.C = it.C + coff[od];
        bp.ldc = L.ldc;
        bp.Aimg = base + L.off_A[od];
        bp.Bimg = base + L.off_B[od];
        bp.colmax = (unsigned long long*)(gcm + item_cm[j] + L.cm_off[od]);
        bp.partial = (double*)(base + L.off_pt[od]);
        bp.err = err;
        bp.wait_limit = ctx->wait_limit;
        bp.aimg_ready = 1;
        bp.kmin = (double*)(base + L.off_kmin);
        const int e = 3 * q + od;
        f_bimg[e] = nbimg;
        nbimg += (long)bp.ntile_n * (bp.Np / 8) * bp.nchunk;
        f_gemm[e] = ngemm; ngemm += (long)bp.ntile_m * bp.ntile_n * bp.nchunk;
      }
    }
    f_ref[ni] = nref; f_coef[ni] = ncoef; f_aimg[ni] = naimg; f_asm[ni] = nasm; f_kmin[ni] = nkmin;
    f_bimg[3 * ni] = nbimg; f_gemm[3 * ni] = ngemm;
    const long grid[7] = {nref, ncoef, naimg, nbimg, ngemm, nasm, nkmin};
    for (int k = 0; k < 7; ++k) D.grid[k] = grid[k];
  }
  CK(cudaMemcpyAsync(dc, h, total_bytes, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemsetAsync(err, 0, sizeof(unsigned), ctx->stream));
  for (size_t g = 0; g < groups.size(); ++g) {
    const Group1DDesc& D = gdesc[g];
    const int ni = D.ni;
    const char* dbase = (const char*)dc;
    Synth1DGroup G;
    G.ni = ni;
    G.it = (const Synth1DItem*)(dbase + D.off_it);
    G.bp = (const BesselI8*)(dbase + D.off_bp);
    const long* df = (const long*)(dbase + D.off_first);
    G.first_reflect = df;
    G.first_coef = df + (ni + 1);
    G.first_aimg = df + 2 * (ni + 1);
    G.first_asm = df + 3 * (ni + 1);
    G.first_kmin = df + 4 * (ni + 1);
    G.first_bimg = df + 5 * (ni + 1);
    G.first_gemm = G.first_bimg + (3 * ni + 1);
    for (int k = 0; k < 7; ++k) G.grid[k] = D.grid[k];
    CK(LAUNCH("k_reflect2d", launch_reflect_coef_group(G, 0, ctx->stream)));
    CK(LAUNCH("k_coef1d", launch_reflect_coef_group(G, 1, ctx->stream)));
    CK(LAUNCH("k_aimg_bessel3", launch_bessel_i8_group(G, 0, ctx->stream)));
    CK(LAUNCH("k_bimg_real", launch_bessel_i8_group(G, 1, ctx->stream)));
    CK(LAUNCH("k_gemm_i8_img", launch_bessel_i8_group(G, 2, ctx->stream)));
    CK(LAUNCH("k_assemble1d", launch_assemble1d_group(G, ctx->stream)));
    for (size_t j = groups[g].first; j < groups[g].second; ++j) {
      const int i = lay[j].item;
      if (d[i].out_is_device) continue;
      CK(cudaMemcpyAsync(d[i].out, gws + item_base[j] + lay[j].off_G,
                         sizeof(double2) * 9 * (size_t)d[i].nx * d[i].ny * d[i].nz, cudaMemcpyDeviceToHost,
                         ctx->stream));
    }
  }
  // an all-1D batch runs its items round-robin on kSlots side streams (each item is a chain
  // of small dependent launches; independent items overlap), forked from and joined to the
  // context's stream
  constexpr int kSlots = 4;
  const int nslot = all1d ? std::min(kSlots, nb) : 0;
  if (nslot) {
    while ((int)ctx->slot_streams.size() < kSlots) {
      cudaStream_t s;
      cudaEvent_t e;
      CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ctx->slot_streams.push_back(s);
      ctx->slot_events.push_back(e);
    }
    CK(cudaEventRecord(ctx->slot_events[0], ctx->stream));
    for (int s = 0; s < nslot; ++s) CK(cudaStreamWaitEvent(ctx->slot_streams[s], ctx->slot_events[0], 0));
  }
  cudaStream_t main = ctx->stream;
  int rc = YTF_OK;
  for (int i = 0; i < nb && !rc; ++i) {
    if (grouped[i]) continue;
    GreenBatch gb{dc + o[i], dc + o[i] + d[i].nz, dc + o[i] + d[i].nz + d[i].nx, err};
    if (!ur[i].empty()) {
      gb.drho = dc + tot + orho[i];
      gb.drmap = dm + omap[i];
    }
    if (nslot) {
      ctx->stream = ctx->slot_streams[i % nslot];
      ctx->ws_slot = 1 + i % nslot;
    }
    rc = green_impl(ctx, d[i].cache, d[i].obs_layer, d[i].zsrc_local, d[i].nz, d[i].z_obs, d[i].nx, d[i].xs,
                    d[i].ny, d[i].ys, d[i].terms, d[i].precision, d[i].out, d[i].out_is_device, &gb);
  }
  ctx->stream = main;
  ctx->ws_slot = 0;
  for (int s = 0; s < nslot; ++s) {
    cudaEventRecord(ctx->slot_events[s], ctx->slot_streams[s]);
    cudaStreamWaitEvent(main, ctx->slot_events[s], 0);
  }
  if (rc) {
    cudaStreamSynchronize(main);
    return rc;
  }
  unsigned herr = 0;
  CK(cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  prof_collect(ctx);
  if (herr) return fail(ctx, YTF_ERR_CUDA, "closed_form_G: a tensor-core pipeline wait timed out");
  return YTF_OK;
}

// Gauss-Legendre rule: Newton on the three-term recurrence in long double, rounded once
int ytf_gauss_legendre(int n, double* x, double* w) {
  if (n < 1 || !x || !w) return YTF_ERR_ARG;
  for (int i = 0; i < n; ++i) {
    long double z = cosl(3.14159265358979323846264338327950288L * (i + 0.75L) / (n + 0.5L));
    long double p0 = 1, p1 = z, dp = 0;
    for (int it = 0; it < 100; ++it) {
      p0 = 1; p1 = z;
      for (int k = 2; k <= n; ++k) { long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
      dp = n * (z * p1 - p0) / (z * z - 1);
      long double dz = p1 / dp;
      z -= dz;
      if (fabsl(dz) < 1e-30L) break;
    }
    p0 = 1; p1 = z;
    for (int k = 2; k <= n; ++k) { long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
    dp = n * (z * p1 - p0) / (z * z - 1);
    x[n - 1 - i] = (double)z;
    w[n - 1 - i] = (double)(2.0L / ((1 - z * z) * dp * dp));
  }
  if (n % 2 == 1) x[n / 2] = 0.0;
  return YTF_OK;
}

int ytf_gl_rule(ytf_ctx* ctx, int npanels, const double* pa, const double* pb, int order, int nsing, const double* singular,
                double* nodes, double* weights) {
  if (!ctx || npanels < 0 || order < 1 || (npanels > 0 && (!pa || !pb || !nodes || !weights))) return YTF_ERR_ARG;
  if (npanels == 0) return YTF_OK;
  CK(cudaSetDevice(ctx->device));
  std::vector<double> xi(order), wx(order);
  ytf_gauss_legendre(order, xi.data(), wx.data());
  std::set<double> S;
  for (int i = 0; i < nsing; ++i) S.insert(singular[i]);
  std::vector<int> side(npanels);
  for (int i = 0; i < npanels; ++i) side[i] = S.count(pa[i]) ? 1 : (S.count(pb[i]) ? -1 : 0);
  size_t np = npanels, tot = (size_t)npanels * order;
  WS(buf, double, "gl_buf", 2 * np + 2 * (size_t)order + 2 * tot);
  WS(dside, int, "gl_side", np);
  double *da = buf, *db = buf + np, *dxi = buf + 2 * np, *dwx = dxi + order, *dn = dwx + order, *dw = dn + tot;
  int rc;
  if ((rc = upload(ctx, da, pa, 8 * np)) || (rc = upload(ctx, db, pb, 8 * np)) || (rc = upload(ctx, dxi, xi.data(), 8 * (size_t)order)) ||
      (rc = upload(ctx, dwx, wx.data(), 8 * (size_t)order)) || (rc = upload(ctx, dside, side.data(), 4 * np)))
    return rc;
  CK(LAUNCH("k_gl_nodes", launch_gl_nodes(npanels, da, db, dside, dxi, dwx, order, dn, dw, ctx->stream)));
  CK(cudaMemcpyAsync(nodes, dn, 8 * tot, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(weights, dw, 8 * tot, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return YTF_OK;
}

static int gl_rule_batch_impl(ytf_ctx* ctx, int nsets, const int* npanels, const double* pa, const double* pb,
                              int order, const int* nsing, const double* singular, double* nodes, double* weights,
                              bool out_dev);

int ytf_gl_rule_batch(ytf_ctx* ctx, int nsets, const int* npanels, const double* pa, const double* pb, int order,
                      const int* nsing, const double* singular, double* nodes, double* weights) {
  return gl_rule_batch_impl(ctx, nsets, npanels, pa, pb, order, nsing, singular, nodes, weights, false);
}

int ytf_gl_rule_batch_device(ytf_ctx* ctx, int nsets, const int* npanels, const double* pa, const double* pb, int order,
                             const int* nsing, const double* singular, double* d_nodes, double* d_weights) {
  return gl_rule_batch_impl(ctx, nsets, npanels, pa, pb, order, nsing, singular, d_nodes, d_weights, true);
}

}  // extern "C"

static int gl_rule_batch_impl(ytf_ctx* ctx, int nsets, const int* npanels, const double* pa, const double* pb,
                              int order, const int* nsing, const double* singular, double* nodes, double* weights,
                              bool out_dev) {
  if (!ctx || nsets < 0 || order < 1 || (nsets > 0 && (!npanels || !nsing))) return YTF_ERR_ARG;
  size_t np = 0, ns = 0;
  for (int j = 0; j < nsets; ++j) {
    if (npanels[j] < 0 || nsing[j] < 0) return fail(ctx, YTF_ERR_ARG, "gl_rule: negative count (set " + std::to_string(j) + ")");
    np += npanels[j];
    ns += nsing[j];
  }
  if (np == 0) return YTF_OK;
  if (!pa || !pb || !nodes || !weights || (ns > 0 && !singular)) return YTF_ERR_ARG;
  CK(cudaSetDevice(ctx->device));
  std::vector<double> xi(order), wx(order);
  ytf_gauss_legendre(order, xi.data(), wx.data());
  // each panel's substitution side from its own set's singular points, as ytf_gl_rule
  std::vector<int> side(np);
  size_t p0 = 0, s0 = 0;
  for (int j = 0; j < nsets; ++j) {
    // a set's few singular points (exact matches, as the set lookup of ytf_gl_rule)
    const double* S0 = singular + s0;
    const double* S1 = S0 + nsing[j];
    auto has = [&](double v) { return std::find(S0, S1, v) != S1; };
    for (int i = 0; i < npanels[j]; ++i) {
      const size_t q = p0 + i;
      side[q] = has(pa[q]) ? 1 : (has(pb[q]) ? -1 : 0);
    }
    p0 += npanels[j];
    s0 += nsing[j];
  }
  const size_t tot = np * order;
  WS(buf, double, "glb_buf", 2 * np + 2 * (size_t)order + (out_dev ? 0 : 2 * tot));
  WS(dside, int, "glb_side", np);
  double *da = buf, *db = buf + np, *dxi = buf + 2 * np, *dwx = dxi + order;
  double *dn = out_dev ? nodes : dwx + order, *dw = out_dev ? weights : dn + tot;
  int rc;
  if ((rc = upload(ctx, da, pa, 8 * np)) || (rc = upload(ctx, db, pb, 8 * np)) || (rc = upload(ctx, dxi, xi.data(), 8 * (size_t)order)) ||
      (rc = upload(ctx, dwx, wx.data(), 8 * (size_t)order)) || (rc = upload(ctx, dside, side.data(), 4 * np)))
    return rc;
  CK(LAUNCH("k_gl_nodes", launch_gl_nodes((int)np, da, db, dside, dxi, dwx, order, dn, dw, ctx->stream)));
  if (out_dev) return YTF_OK;  // stream-ordered: later work on the context's stream sees the rule
  CK(cudaMemcpyAsync(nodes, dn, 8 * tot, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(weights, dw, 8 * tot, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return YTF_OK;
}

// =====================================================================================
// Uneven-batch plans (no counterpart in the reference; the contract is in ytf.h). Creation
// validates every item, creates the caches, lays out one staging block of inputs (nodes,
// weights, coordinates, 1D radii) and one of host outputs, and groups the node solves into
// passes that share one scratch arena; ytf_plan_retune builds the tile tables and records
// the graph: H2D of the inputs, counter reset, per pass the persistent stage kernels
// (modes, QR pass, forward-only match/seeds/iface/scan or the general chain), the batched
// synthesis and its chunk sums, D2H of the host outputs.
// =====================================================================================
struct ytf_plan {
  ytf_ctx* ctx = nullptr;
  int nb = 0;
  std::vector<ytf_transfer_desc> tr;
  std::vector<ytf_green_desc> gr;
  std::vector<ytf_cache*> cs;
  std::vector<TransferParams> ps;      // per item, scratch pointers into the arena
  std::vector<std::vector<int>> passes;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  std::vector<size_t> in_node, in_coord;  // per item offsets into the input staging (doubles)
  size_t in_count = 0;
  double* h_in = nullptr;
  double* d_in = nullptr;
  std::vector<std::vector<int>> rmap;  // 1D items: pixel -> distinct radius (first occurrence)
  std::vector<int> nr;
  std::vector<size_t> rmap_off;
  int* d_rmap = nullptr;
  std::vector<long> g_off;             // host-output items: offset into h_G / d_G (complex); else -1
  std::vector<char> direct;            // host output page-locked: the graph copies G straight into it
  size_t g_count = 0;
  double2* h_G = nullptr;
  double2* d_G = nullptr;
  std::vector<SynthParams> sps;
  std::vector<long> nout_syn;          // per item: partial outputs per chunk (0: no synthesis)
  std::vector<char> large;             // 2D items beyond the small-set limits (or not FP64): their
                                       // synthesis is closed_form_G's own kernels in the graph
  std::map<std::string, std::pair<void*, size_t>> wsbufs;  // those kernels' workspaces
  unsigned* d_err = nullptr;           // tensor-core wait-timeout word of those kernels
  unsigned* h_err = nullptr;
  ytf_tune tune{};
  char* tb = nullptr;
  size_t tb_bytes = 0;
  cudaStream_t cap = nullptr;
  cudaStream_t copy = nullptr;          // captured side branch: the large items' output copies
  std::vector<cudaEvent_t> fork_ev;     // one per large item with a page-locked host output, + join
  std::vector<char> copied;             // output copied on the side branch in the current graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  bool pending = false;
  std::map<std::string, long> kcount;  // kernels per run, by name
  long nodes = 0;
  int nsm = 148;
};

namespace {

void plan_release_graph(ytf_plan* P) {
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->graph) cudaGraphDestroy(P->graph);
  if (P->tb) cudaFree(P->tb);
  P->exec = nullptr;
  P->graph = nullptr;
  P->tb = nullptr;
  P->tb_bytes = 0;
  P->kcount.clear();
  for (auto e : P->fork_ev) cudaEventDestroy(e);
  P->fork_ev.clear();
}

void plan_free(ytf_plan* P) {
  if (!P) return;
  cudaSetDevice(P->ctx->device);
  cudaStreamSynchronize(P->ctx->stream);
  if (P->cap) cudaStreamSynchronize(P->cap);
  plan_release_graph(P);
  if (P->cap) cudaStreamDestroy(P->cap);
  if (P->copy) cudaStreamDestroy(P->copy);
  if (P->e0) cudaEventDestroy(P->e0);
  if (P->e1) cudaEventDestroy(P->e1);
  if (P->arena) cudaFree(P->arena);
  if (P->d_in) cudaFree(P->d_in);
  if (P->d_rmap) cudaFree(P->d_rmap);
  if (P->d_G) cudaFree(P->d_G);
  if (P->h_in) cudaFreeHost(P->h_in);
  if (P->h_G) cudaFreeHost(P->h_G);
  if (P->d_err) cudaFree(P->d_err);
  if (P->h_err) cudaFreeHost(P->h_err);
  for (auto& kv : P->wsbufs) cudaFree(kv.second.first);
  for (auto c : P->cs)
    if (c) ytf_cache_destroy(c);
  delete P;
}

// distinct radii of a pixel set in first-occurrence order over (i fastest, j), as the 1D
// synthesis of closed_form_G
void radius_map(int nx, int ny, const double* xs, const double* ys, std::vector<double>& ur, std::vector<int>& rm) {
  ur.clear();
  rm.assign((size_t)nx * ny, 0);
  std::unordered_map<double, int> idx;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const double r = std::hypot(xs[i], ys[j]);
      auto it = idx.find(r);
      if (it == idx.end()) {
        idx.emplace(r, (int)ur.size());
        rm[i + (size_t)nx * j] = (int)ur.size();
        ur.push_back(r);
      } else {
        rm[i + (size_t)nx * j] = it->second;
      }
    }
}

int plan_fail(ytf_ctx* ctx, int rc, int item) {
  ctx->err += " (plan item " + std::to_string(item) + ")";
  return rc;
}

// the synthesis of the large 2D items through closed_form_G's own path, on the plan's stream
// with the coordinates of the device staging, outputs into the plan's buffers: recording the
// workspace sizes (rec) or from the plan's workspaces (ovr, inside the capture). Profiling is
// off meanwhile; the launch counts it adds go to the plan's per-run counts (captured pass).
int plan_large_synthesis(ytf_plan* P, std::map<std::string, size_t>* rec,
                         std::map<std::string, std::pair<void*, size_t>>* ovr) {
  ytf_ctx* ctx = P->ctx;
  const cudaStream_t saved = ctx->stream;
  const bool prof = ctx->prof;
  const auto klaunch = ctx->klaunch;
  ctx->stream = P->cap;
  ctx->prof = false;
  ctx->ws_record = rec;
  ctx->ws_override = ovr;
  int rc = YTF_OK;
  size_t nfork = 0;
  for (int i = 0; i < P->nb && !rc; ++i) {
    if (!P->large[i]) continue;
    const ytf_green_desc& g = P->gr[i];
    const double* co = P->d_in + P->in_coord[i];
    GreenBatch gb{co, co + g.nz, co + g.nz + g.nx, P->d_err};
    double* out = P->g_off[i] >= 0 ? (double*)(P->d_G + P->g_off[i]) : g.out;
    rc = green_impl(ctx, P->cs[i], g.obs_layer, g.zsrc_local, g.nz, g.z_obs, g.nx, g.xs, g.ny, g.ys, g.terms,
                    g.precision, out, 1, &gb);
    if (rc) rc = plan_fail(ctx, rc, i);
    // captured pass: a page-locked host output is copied on the side branch as soon as its
    // item is done, overlapping the next items' kernels
    if (!rc && ovr && P->direct[i] && P->g_off[i] >= 0 && nfork < P->fork_ev.size()) {
      cudaEvent_t ev = P->fork_ev[nfork++];
      cudaError_t e = cudaEventRecord(ev, P->cap);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(P->copy, ev, 0);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(g.out, P->d_G + P->g_off[i], 16 * (size_t)g.nx * g.ny * g.nz * 9, cudaMemcpyDeviceToHost,
                            P->copy);
      if (e != cudaSuccess) rc = fail(ctx, YTF_ERR_CUDA, std::string("ytf_plan: output copy: ") + cudaGetErrorString(e));
      else P->copied[i] = 1;
    }
  }
  // join the side branch back into the captured stream
  if (!rc && ovr && nfork > 0) {
    cudaEvent_t join = P->fork_ev.back();
    cudaError_t e = cudaEventRecord(join, P->copy);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(P->cap, join, 0);
    if (e != cudaSuccess) rc = fail(ctx, YTF_ERR_CUDA, std::string("ytf_plan: output copy join: ") + cudaGetErrorString(e));
  }
  if (ovr)
    for (auto& kv : ctx->klaunch) {
      auto it = klaunch.find(kv.first);
      const long d = kv.second - (it == klaunch.end() ? 0 : it->second);
      if (d > 0) P->kcount[kv.first] += d;
    }
  ctx->klaunch = klaunch;
  ctx->ws_record = nullptr;
  ctx->ws_override = nullptr;
  ctx->stream = saved;
  ctx->prof = prof;
  return rc;
}

// validation, caches, staging, outputs and passes (everything the tiles do not change)
int plan_build(ytf_plan* P) {
  ytf_ctx* ctx = P->ctx;
  const int nb = P->nb;
  P->cs.assign(nb, nullptr);
  P->ps.resize(nb);
  P->sps.resize(nb);
  P->rmap.resize(nb);
  P->nr.assign(nb, 0);
  P->rmap_off.assign(nb, 0);
  P->g_off.assign(nb, -1);
  P->nout_syn.assign(nb, 0);
  P->large.assign(nb, 0);
  P->direct.assign(nb, 0);
  P->in_node.assign(nb, 0);
  P->in_coord.assign(nb, 0);
  size_t rmap_count = 0;
  for (int i = 0; i < nb; ++i) {
    const ytf_transfer_desc& d = P->tr[i];
    const ytf_green_desc& g = P->gr[i];
    const bool is2d = d.nphi > 0 || d.is2d;
    bool rot = false;
    if (d.nodes_on_device)
      return plan_fail(ctx, fail(ctx, YTF_ERR_ARG, "ytf_plan_create: plans take host node arrays (nodes_on_device = 0)"), i);
    int rc = prepare_cache(ctx, d.stack, is2d, d.omega, d.source_layer, d.nk, d.k_nodes, d.k_weights, d.nphi,
                           d.phi_nodes, d.phi_weights, d.nobs, d.obs_layers, d.check_symmetry, YTF_ROT_OFF, false,
                           &P->cs[i], &rot);
    if (rc) return plan_fail(ctx, rc, i);
    ytf_cache* c = P->cs[i];
    P->nodes += c->n;
    if (g.nz < 0 || g.nx < 0 || g.ny < 0) return plan_fail(ctx, fail(ctx, YTF_ERR_ARG, "closed_form_G: negative grid size"), i);
    const long npix0 = (long)g.nx * g.ny;
    P->large[i] = is2d && (g.precision != YTF_PREC_FP64 || g.nz > SYN_MAXZ || npix0 > SYN_MAXPIX ||
                           npix0 * 9 * g.nz > SYN_MAXOUT);
    if (!is2d && g.precision != YTF_PREC_FP64)
      return plan_fail(ctx, fail(ctx, YTF_ERR_ARG, "ytf_plan_create: a plan's 1D synthesis is FP64 (precision must be YTF_PREC_FP64)"), i);
    if (!is2d && g.nz > SYN_MAXZ)
      return plan_fail(ctx, fail(ctx, YTF_ERR_ARG, "ytf_plan_create: at most " + std::to_string(SYN_MAXZ) + " z rows per 1D item"), i);
    if ((g.nz && !g.z_obs) || (g.nx && !g.xs) || (g.ny && !g.ys) || !g.out)
      return plan_fail(ctx, fail(ctx, YTF_ERR_ARG, "ytf_plan_create: NULL coordinate or output array"), i);
    if ((rc = synth_setup(ctx, c, g.obs_layer, g.zsrc_local, g.terms, g.nz, P->sps[i]))) return plan_fail(ctx, rc, i);
    const long npix = (long)g.nx * g.ny;
    if (is2d) {
      P->nout_syn[i] = P->large[i] ? 0 : npix * 9 * g.nz;
    } else {
      std::vector<double> ur;
      radius_map(g.nx, g.ny, g.xs, g.ys, ur, P->rmap[i]);
      P->nr[i] = (int)ur.size();
      if (P->nr[i] > SYN_MAXR || (long)P->nr[i] * 13 * g.nz > SYN_MAXOUT)
        return plan_fail(ctx, fail(ctx, YTF_ERR_ARG, "ytf_plan_create: 1D items need at most " + std::to_string(SYN_MAXR) +
                                                         " distinct radii and 13*nz*radii <= " + std::to_string(SYN_MAXOUT)), i);
      P->nout_syn[i] = (long)P->nr[i] * 13 * g.nz;
      P->rmap_off[i] = rmap_count;
      rmap_count += (size_t)npix;
    }
    if (npix * g.nz == 0) P->nout_syn[i] = 0;
    // input staging: nodes, weights, φ nodes and weights, then z rows, x, y, 1D radii
    P->in_node[i] = P->in_count;
    P->in_count += 2 * c->kr.size() + 2 * c->phi.size();
    P->in_coord[i] = P->in_count;
    P->in_count += (size_t)g.nz + g.nx + g.ny + P->nr[i];
    if (!g.out_is_device && npix * g.nz > 0) {
      P->g_off[i] = (long)P->g_count;
      P->g_count += (size_t)npix * g.nz * 9;
      cudaPointerAttributes at;
      if (cudaPointerGetAttributes(&at, g.out) == cudaSuccess && at.type == cudaMemoryTypeHost) P->direct[i] = 1;
      cudaGetLastError();
    }
  }
  CK(cudaHostAlloc(&P->h_in, 8 * std::max<size_t>(P->in_count, 1), cudaHostAllocDefault));
  CK(cudaMalloc(&P->d_in, 8 * std::max<size_t>(P->in_count, 1)));
  CK(cudaMemset(P->d_in, 0, 8 * std::max<size_t>(P->in_count, 1)));
  CK(cudaMalloc(&P->d_err, sizeof(unsigned)));
  CK(cudaMemset(P->d_err, 0, sizeof(unsigned)));
  CK(cudaHostAlloc(&P->h_err, sizeof(unsigned), cudaHostAllocDefault));
  *P->h_err = 0;
  if (P->g_count) {
    CK(cudaHostAlloc(&P->h_G, 16 * P->g_count, cudaHostAllocDefault));
    CK(cudaMalloc(&P->d_G, 16 * P->g_count));
  }
  if (rmap_count) {
    std::vector<int> all(rmap_count);
    for (int i = 0; i < nb; ++i)
      if (!P->rmap[i].empty()) std::copy(P->rmap[i].begin(), P->rmap[i].end(), all.begin() + P->rmap_off[i]);
    CK(cudaMalloc(&P->d_rmap, 4 * rmap_count));
    CK(cudaMemcpy(P->d_rmap, all.data(), 4 * rmap_count, cudaMemcpyHostToDevice));
  }
  // the caches read their nodes from the device copy of the staging; the synthesis its rows
  for (int i = 0; i < nb; ++i) {
    ytf_cache* c = P->cs[i];
    double* b = P->d_in + P->in_node[i];
    const size_t nk = c->kr.size(), np = c->phi.size();
    c->d_kr = b;
    c->d_wr = b + nk;
    if (np) {
      c->d_phi = b + 2 * nk;
      c->d_wphi = b + 2 * nk + np;
    }
    SynthParams& sp = P->sps[i];
    sp.c.kr = c->d_kr; sp.c.wr = c->d_wr; sp.c.phi = c->d_phi; sp.c.wphi = c->d_wphi;
    sp.zo = P->d_in + P->in_coord[i];
  }
  // node-solve passes under the scratch budget, items in order
  const size_t budget = (size_t)6 << 30;
  std::vector<size_t> need(nb, 0);
  for (int i = 0; i < nb; ++i) {
    ytf_cache* c = P->cs[i];
    TransferParams& q = P->ps[i];
    fill_params(q, P->tr[i].stack, c);
    q.mode = c->is2d ? 1 : 0;
    q.n = c->n;
    q.off = 0;
    q.nout = c->n;
    if (c->n == 0) continue;
    const int N = q.nL;
    const long n = q.n;
    auto r256 = [](size_t b) { return (b + 255) & ~size_t(255); };
    size_t b = r256((size_t)N * 20 * 16 * n) + r256((size_t)N * n) + r256((size_t)std::max(N - 1, 1) * 16 * 16 * n);
    if (only_source_observed(q)) b += r256((size_t)std::max(N - 1, 1) * n);
    else b += (q.needL ? r256((size_t)N * 16 * 16 * n) : 0) + (q.needR ? r256((size_t)N * 16 * 16 * n) : 0);
    need[i] = b;
  }
  {
    std::vector<int> cur;
    size_t used = 0;
    for (int i = 0; i < nb; ++i) {
      if (!need[i]) continue;
      if (!cur.empty() && used + need[i] > budget) {
        P->passes.push_back(cur);
        P->arena_bytes = std::max(P->arena_bytes, used);
        cur.clear();
        used = 0;
      }
      cur.push_back(i);
      used += need[i];
    }
    if (!cur.empty()) {
      P->passes.push_back(cur);
      P->arena_bytes = std::max(P->arena_bytes, used);
    }
  }
  if (P->arena_bytes) CK(cudaMalloc(&P->arena, P->arena_bytes));
  for (auto& pass : P->passes) {
    size_t o = 0;
    auto carve = [&](size_t bytes) {
      char* q = P->arena + o;
      o += (bytes + 255) & ~size_t(255);
      return q;
    };
    for (int i : pass) {
      TransferParams& q = P->ps[i];
      const int N = q.nL;
      const long n = q.n;
      q.modes = (double2*)carve((size_t)N * 20 * 16 * n);
      q.lstat = (uint8_t*)carve((size_t)N * n);
      q.sint = (double2*)carve((size_t)std::max(N - 1, 1) * 16 * 16 * n);
      if (only_source_observed(q)) {
        q.dec = (uint8_t*)carve((size_t)std::max(N - 1, 1) * n);
      } else {
        q.sleft = q.needL ? (double2*)carve((size_t)N * 16 * 16 * n) : nullptr;
        q.sright = q.needR ? (double2*)carve((size_t)N * 16 * 16 * n) : nullptr;
      }
    }
  }
  CK(cudaStreamCreateWithFlags(&P->cap, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&P->copy, cudaStreamNonBlocking));
  CK(cudaEventCreate(&P->e0));
  CK(cudaEventCreate(&P->e1));
  CK(synth_small_init());
  CK(cudaStreamSynchronize(ctx->stream));  // cache blocks cleared before the first run
  // one eager pass of the large items' synthesis (on the zeroed inputs) records the largest
  // size of each workspace it asks for; the plan then owns buffers of those sizes
  std::map<std::string, size_t> rec;
  int rc = plan_large_synthesis(P, &rec, nullptr);
  if (rc) return rc;
  CK(cudaStreamSynchronize(P->cap));
  for (auto& kv : rec) {
    void* b = nullptr;
    CK(cudaMalloc(&b, kv.second));
    P->wsbufs[kv.first] = {b, kv.second};
  }
  return YTF_OK;
}

}  // namespace

extern "C" int ytf_plan_retune(ytf_plan* P, const ytf_tune* tune_in) {
  if (!P) return YTF_ERR_ARG;
  ytf_ctx* ctx = P->ctx;
  ytf_tune t{128, 4, 1024, 2048, 2};
  if (tune_in) t = *tune_in;
  if (!(t.block == 128 || t.block == 256) || t.ctas_per_sm < 1 || t.ctas_per_sm > 32 || t.tile < 1 || t.chunk < 16 ||
      t.chunk % 16 != 0 || t.synth_ctas_per_sm < 1 || t.synth_ctas_per_sm > 8)
    return fail(ctx, YTF_ERR_ARG, "ytf_plan_retune: block 128|256, ctas_per_sm 1..32, tile >= 1, chunk a positive "
                                  "multiple of 16, synth_ctas_per_sm 1..8");
  CK(cudaSetDevice(ctx->device));
  if (P->pending) {
    CK(cudaEventSynchronize(P->e1));
    P->pending = false;
  }
  plan_release_graph(P);
  P->tune = t;
  const int nb = P->nb;
  // host image of the tile-dependent block: per pass the parameter array and its tile
  // tables per stage, the synthesis items with their offsets, then the counters and partials
  struct Launch {
    int stage;
    size_t params;  // byte offset of the pass's TransferParams array
    size_t prob, start, end;
    int ntiles;
    int counter;
  };
  std::vector<char> hb;
  auto put = [&](const void* src, size_t bytes) {  // src NULL: zero bytes
    size_t o = (hb.size() + 255) & ~size_t(255);
    hb.resize(o + bytes, 0);
    if (bytes && src) std::memcpy(hb.data() + o, src, bytes);
    return o;
  };
  std::vector<Launch> launches;
  int ncounter = 0;
  for (auto& pass : P->passes) {
    std::vector<TransferParams> pp;
    for (int i : pass) pp.push_back(P->ps[i]);
    const size_t po = put(pp.data(), sizeof(TransferParams) * pp.size());
    const int stages[] = {0, 1, 6, 5, 7, 3};
    for (int st : stages) {
      std::vector<int> prob;
      std::vector<long> a, b;
      for (int j = 0; j < (int)pass.size(); ++j) {
        const TransferParams& q = pp[j];
        const bool fast = only_source_observed(q);
        long units;
        if (st == 0 || st == 1) units = (long)q.nL * q.n;
        else if (st == 3) units = fast ? 0 : q.n;
        else if (st == 6) units = fast ? (long)(q.nL - 1) * q.n : 0;
        else units = fast ? q.n : 0;
        for (long u = 0; u < units; u += t.tile) {
          prob.push_back(j);
          a.push_back(u);
          b.push_back(std::min(units, u + (long)t.tile));
        }
      }
      if (prob.empty()) continue;
      Launch L;
      L.stage = st;
      L.params = po;
      L.prob = put(prob.data(), 4 * prob.size());
      L.start = put(a.data(), 8 * a.size());
      L.end = put(b.data(), 8 * b.size());
      L.ntiles = (int)prob.size();
      L.counter = ncounter++;
      launches.push_back(L);
    }
  }
  // synthesis items (those with outputs), chunk and finish offsets
  std::vector<SynthItem> items;
  std::vector<long> woff{0}, foff{0};
  std::vector<int> item_of;
  size_t npart = 0, syn_smem = 0;
  for (int i = 0; i < nb; ++i) {
    const ytf_green_desc& g = P->gr[i];
    const long npix = (long)g.nx * g.ny;
    if (npix * g.nz == 0 || P->large[i]) continue;
    SynthItem it;
    std::memset(&it, 0, sizeof(it));
    it.sp = P->sps[i];
    const double* co = P->d_in + P->in_coord[i];
    it.xs = co + g.nz;
    it.ys = co + g.nz + g.nx;
    it.nx = g.nx;
    it.ny = g.ny;
    it.is2d = P->cs[i]->is2d ? 1 : 0;
    it.rho = co + g.nz + g.nx + g.ny;
    it.rmap = it.is2d ? nullptr : P->d_rmap + P->rmap_off[i];
    it.nr = P->nr[i];
    const long n = P->cs[i]->n;
    it.nw = (int)((n + t.chunk - 1) / t.chunk);
    it.G = P->g_off[i] >= 0 ? P->d_G + P->g_off[i] : (double2*)g.out;
    items.push_back(it);
    item_of.push_back(i);
    syn_smem = std::max(syn_smem, synth_small_smem(it.is2d, (int)npix, it.nr, g.nz));
    npart += (size_t)it.nw * P->nout_syn[i];
    woff.push_back(woff.back() + it.nw);
    foff.push_back(foff.back() + (it.is2d ? npix * 9 * g.nz : npix * g.nz));
  }
  const int synth_counter = ncounter++;
  size_t o_items = 0, o_woff = 0, o_foff = 0;
  if (!items.empty()) {
    o_items = put(items.data(), sizeof(SynthItem) * items.size());
    o_woff = put(woff.data(), 8 * woff.size());
    o_foff = put(foff.data(), 8 * foff.size());
  }
  const size_t o_ctr = put(nullptr, 4 * (size_t)ncounter);
  const size_t o_part = (hb.size() + 255) & ~size_t(255);  // partial sums: device only
  P->tb_bytes = o_part + 16 * std::max<size_t>(npart, 1);
  CK(cudaMalloc(&P->tb, P->tb_bytes));
  // partial-sum pointers of the synthesis items, now that the block's address is known
  {
    size_t po = 0;
    for (size_t k = 0; k < items.size(); ++k) {
      SynthItem* it = reinterpret_cast<SynthItem*>(hb.data() + o_items) + k;
      it->partial = reinterpret_cast<double2*>(P->tb + o_part) + po;
      po += (size_t)it->nw * P->nout_syn[item_of[k]];
    }
  }
  CK(cudaMemcpy(P->tb, hb.data(), hb.size(), cudaMemcpyHostToDevice));
  // side-branch events of the large items' page-locked outputs (+ one to join), made before
  // the capture
  P->copied.assign(nb, 0);
  {
    int nd = 0;
    for (int i = 0; i < nb; ++i) nd += P->large[i] && P->direct[i] && P->g_off[i] >= 0;
    for (int k = 0; k < nd + (nd > 0); ++k) {
      cudaEvent_t ev;
      CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      P->fork_ev.push_back(ev);
    }
  }
  // record the graph
  unsigned* ctr = reinterpret_cast<unsigned*>(P->tb + o_ctr);
  const int nsm = P->nsm;
  cudaStream_t s = P->cap;
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  auto step = [&](cudaError_t r) {
    if (e == cudaSuccess && r != cudaSuccess) e = r;
  };
  if (P->in_count) step(cudaMemcpyAsync(P->d_in, P->h_in, 8 * P->in_count, cudaMemcpyHostToDevice, s));
  step(cudaMemsetAsync(ctr, 0, 4 * (size_t)ncounter, s));
  step(cudaMemsetAsync(P->d_err, 0, sizeof(unsigned), s));
  static const char* names[] = {"k_persist_modes", "k_persist_qr", "", "k_persist_chain", "",
                                "k_persist_seeds", "k_persist_iface", "k_persist_scan"};
  for (auto& L : launches) {
    TileQueue q;
    q.prob = reinterpret_cast<const int*>(P->tb + L.prob);
    q.start = reinterpret_cast<const long*>(P->tb + L.start);
    q.end = reinterpret_cast<const long*>(P->tb + L.end);
    q.ntiles = L.ntiles;
    q.counter = ctr + L.counter;
    const int grid = std::min(L.ntiles, t.ctas_per_sm * nsm);
    step(launch_persist(L.stage, t.block, grid, reinterpret_cast<const TransferParams*>(P->tb + L.params), q, s));
    P->kcount[names[L.stage]] += 1;
  }
  if (!items.empty()) {
    const SynthItem* di = reinterpret_cast<const SynthItem*>(P->tb + o_items);
    const long* dw = reinterpret_cast<const long*>(P->tb + o_woff);
    const long* df = reinterpret_cast<const long*>(P->tb + o_foff);
    if (woff.back() > 0) {
      const int grid = (int)std::min<long>(woff.back(), (long)t.synth_ctas_per_sm * nsm);
      step(launch_synth_small(di, (int)items.size(), dw, woff.back(), ctr + synth_counter, t.chunk, grid, syn_smem, s));
      P->kcount["k_synth_small"] += 1;
    }
    step(launch_synth_finish(di, (int)items.size(), df, foff.back(), s));
    P->kcount["k_synth_finish"] += 1;
  }
  int lrc = YTF_OK;
  if (e == cudaSuccess) lrc = plan_large_synthesis(P, nullptr, &P->wsbufs);
  // host outputs: page-locked ones straight from the device buffer, the rest in one copy to
  // the plan's staging (delivered by ytf_plan_wait)
  {
    size_t lo = 0, hi = 0;
    bool any = false;
    for (int i = 0; i < nb; ++i) {
      if (P->g_off[i] < 0) continue;
      const ytf_green_desc& g = P->gr[i];
      const size_t cnt = (size_t)g.nx * g.ny * g.nz * 9;
      if (P->direct[i]) {
        if (!P->copied[i]) step(cudaMemcpyAsync(g.out, P->d_G + P->g_off[i], 16 * cnt, cudaMemcpyDeviceToHost, s));
      } else {
        if (!any) lo = P->g_off[i];
        any = true;
        hi = P->g_off[i] + cnt;
      }
    }
    if (any) step(cudaMemcpyAsync(P->h_G + lo, P->d_G + lo, 16 * (hi - lo), cudaMemcpyDeviceToHost, s));
  }
  step(cudaMemcpyAsync(P->h_err, P->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  cudaError_t ee = cudaStreamEndCapture(s, &P->graph);
  if (lrc) {
    if (P->graph) cudaGraphDestroy(P->graph);
    P->graph = nullptr;
    plan_release_graph(P);
    return lrc;
  }
  if (e == cudaSuccess) e = ee;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&P->exec, P->graph, 0);
  if (e != cudaSuccess) {
    plan_release_graph(P);
    return fail(ctx, YTF_ERR_CUDA, std::string("ytf_plan_retune: graph capture: ") + cudaGetErrorString(e));
  }
  return YTF_OK;
}

extern "C" int ytf_plan_create(ytf_ctx* ctx, int nb, const ytf_transfer_desc* tr, const ytf_green_desc* gr,
                               const ytf_tune* tune, ytf_plan** out) {
  if (!ctx || !out || nb < 0 || (nb > 0 && (!tr || !gr))) return YTF_ERR_ARG;
  *out = nullptr;
  CK(cudaSetDevice(ctx->device));
  ytf_plan* P = new ytf_plan();
  P->ctx = ctx;
  P->nb = nb;
  P->tr.assign(tr, tr + nb);
  P->gr.assign(gr, gr + nb);
  cudaDeviceGetAttribute(&P->nsm, cudaDevAttrMultiProcessorCount, ctx->device);
  int rc = plan_build(P);
  if (!rc) rc = ytf_plan_retune(P, tune);
  if (rc) {
    std::string m = ctx->err;
    plan_free(P);
    ctx->err = m;
    return rc;
  }
  *out = P;
  return YTF_OK;
}

extern "C" int ytf_plan_run(ytf_plan* P) {
  if (!P || !P->exec) return YTF_ERR_ARG;
  ytf_ctx* ctx = P->ctx;
  CK(cudaSetDevice(ctx->device));
  if (P->pending) {  // the staging is read by the previous run's copy
    CK(cudaEventSynchronize(P->e1));
    P->pending = false;
  }
  for (int i = 0; i < P->nb; ++i) {
    const ytf_transfer_desc& d = P->tr[i];
    const ytf_green_desc& g = P->gr[i];
    const ytf_cache* c = P->cs[i];
    double* h = P->h_in + P->in_node[i];
    const size_t nk = c->kr.size(), np = c->phi.size();
    if (nk) {
      std::memcpy(h, d.k_nodes, 8 * nk);
      std::memcpy(h + nk, d.k_weights, 8 * nk);
    }
    if (np) {
      std::memcpy(h + 2 * nk, d.phi_nodes, 8 * np);
      std::memcpy(h + 2 * nk + np, d.phi_weights, 8 * np);
    }
    double* hc = P->h_in + P->in_coord[i];
    if (g.nz) std::memcpy(hc, g.z_obs, 8 * (size_t)g.nz);
    if (g.nx) std::memcpy(hc + g.nz, g.xs, 8 * (size_t)g.nx);
    if (g.ny) std::memcpy(hc + g.nz + g.nx, g.ys, 8 * (size_t)g.ny);
    if (!c->is2d && P->nr[i]) {
      std::vector<double> ur;
      std::vector<int> rm;
      radius_map(g.nx, g.ny, g.xs, g.ys, ur, rm);
      if (rm != P->rmap[i]) return plan_fail(ctx, fail(ctx, YTF_ERR_ARG, "ytf_plan_run: the pattern of equal radii changed"), i);
      std::memcpy(hc + g.nz + g.nx + g.ny, ur.data(), 8 * ur.size());
    }
  }
  CK(cudaEventRecord(P->e0, ctx->stream));
  if (ctx->prof) {
    ProfSpan sp{"ytf_plan_graph", take_event(ctx), take_event(ctx)};
    CK(cudaEventRecord(sp.a, ctx->stream));
    CK(cudaGraphLaunch(P->exec, ctx->stream));
    CK(cudaEventRecord(sp.b, ctx->stream));
    ctx->spans.push_back(sp);
  } else {
    CK(cudaGraphLaunch(P->exec, ctx->stream));
  }
  CK(cudaEventRecord(P->e1, ctx->stream));
  for (auto& kv : P->kcount) ctx->klaunch[kv.first] += kv.second;
  P->pending = true;
  return YTF_OK;
}

extern "C" int ytf_plan_wait(ytf_plan* P, float* device_ms) {
  if (!P) return YTF_ERR_ARG;
  ytf_ctx* ctx = P->ctx;
  CK(cudaSetDevice(ctx->device));
  if (!P->pending) {
    if (device_ms) *device_ms = 0.f;
    return YTF_OK;
  }
  CK(cudaEventSynchronize(P->e1));
  P->pending = false;
  if (*P->h_err) return fail(ctx, YTF_ERR_CUDA, "ytf_plan_wait: a tensor-core pipeline wait timed out");
  for (int i = 0; i < P->nb; ++i)
    if (P->g_off[i] >= 0 && !P->direct[i]) {
      const ytf_green_desc& g = P->gr[i];
      std::memcpy(g.out, P->h_G + P->g_off[i], 16 * (size_t)g.nx * g.ny * g.nz * 9);
    }
  if (device_ms) CK(cudaEventElapsedTime(device_ms, P->e0, P->e1));
  if (ctx->prof) {
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
  }
  return YTF_OK;
}

extern "C" int ytf_plan_cache(const ytf_plan* P, int item, const ytf_cache** out) {
  if (!P || !out || item < 0 || item >= P->nb) return YTF_ERR_ARG;
  *out = P->cs[item];
  return YTF_OK;
}

extern "C" int ytf_plan_info(const ytf_plan* P, long* nodes, int* passes, int* kernels, long* h2d_bytes,
                             long* d2h_bytes) {
  if (!P) return YTF_ERR_ARG;
  if (nodes) *nodes = P->nodes;
  if (passes) *passes = (int)P->passes.size();
  if (kernels) {
    long k = 0;
    for (auto& kv : P->kcount) k += kv.second;
    *kernels = (int)k;
  }
  if (h2d_bytes) *h2d_bytes = 8 * (long)P->in_count;
  if (d2h_bytes) *d2h_bytes = 16 * (long)P->g_count;
  return YTF_OK;
}

extern "C" int ytf_plan_destroy(ytf_plan* P) {
  if (!P) return YTF_OK;
  plan_free(P);
  return YTF_OK;
}

// =====================================================================================
// Allocation-free 2D synthesis (ytf_green_noalloc)
//
// Some callers cannot let a library call cudaMalloc: a host that owns every device byte
// through its own pool (a Julia CUDA.jl session, a caching allocator), or a caller on a
// latency-critical path where cudaMalloc's implicit device-wide synchronisation is not
// allowed. For them the 2D synthesis runs with its scratch (the per-node strengths and
// the split-k partial sums) in this fixed array instead of the context's workspace. The
// array is part of the loaded library: every GPU that loads libytf holds its 64 MiB
// until the process exits. Its device address is looked up once per device, on that
// device's first call (so make that first call before any stream capture) and cached for
// the life of the process: after a cudaDeviceReset the cached address is stale, so a host
// that resets a device must not call this entry point on it again.
// =====================================================================================
#include <mutex>

#define YTF_NOALLOC_SCRATCH_COMPLEX (1L << 22)  // 4,194,304 complex doubles = 64 MiB

static __device__ __align__(256) double2 ytf_noalloc_scratch[YTF_NOALLOC_SCRATCH_COMPLEX];

namespace {
std::mutex g_noalloc_mu;
double2* g_noalloc_ptr[256] = {};

// device address of the scratch array on the current device (set up on first use)
cudaError_t noalloc_scratch(int device, double2** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (device < 0 || device >= 256) return cudaErrorInvalidDevice;
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, ytf_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[device] = (double2*)p;
  }
  *out = g_noalloc_ptr[device];
  return cudaSuccess;
}
}  // namespace

extern "C" int ytf_green_noalloc(ytf_ctx* ctx, const ytf_cache* c, int obs_layer, double zsrc_local, int nz,
                                 const double* z_obs_dev, int nx, const double* xs_dev, int ny, const double* ys_dev,
                                 int terms, double* out_dev) {
  if (!ctx) return YTF_ERR_ARG;
  if (!c || !out_dev || !z_obs_dev || !xs_dev || !ys_dev)
    return fail(ctx, YTF_ERR_ARG, "ytf_green_noalloc: null cache, coordinate or output pointer");
  if (c->ctx != ctx) return fail(ctx, YTF_ERR_STATE, "ytf_green_noalloc: cache belongs to another context");
  if (!c->is2d) return fail(ctx, YTF_ERR_ARG, "ytf_green_noalloc: needs a 2D (kρ, φ) cache");
  SynthParams sp;
  {
    int rc0 = synth_setup(ctx, c, obs_layer, zsrc_local, terms, nz, sp);
    if (rc0) return rc0;
  }
  if (nz < 0 || nx < 0 || ny < 0) return fail(ctx, YTF_ERR_ARG, "closed_form_G: negative grid size");
  // as ytf_green: an empty grid writes nothing, an empty rule integrates to zero
  if ((long)nx * ny * nz == 0) return YTF_OK;
  CK(cudaSetDevice(ctx->device));
  if (c->n == 0) {
    CK(cudaMemsetAsync(out_dev, 0, sizeof(double2) * 9 * (size_t)nx * ny * nz, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return YTF_OK;
  }
  const long npix = (long)nx * ny, ncol = 9L * nz, n = c->n;
  // scratch: strengths [ncol][n] then splits x [npix][ncol] partial sums
  const long need1 = ncol * n + npix * ncol;
  if (need1 > YTF_NOALLOC_SCRATCH_COMPLEX)
    return fail(ctx, YTF_ERR_ARG, "ytf_green_noalloc: 9*nz*(n_nodes + Nx*Ny) = " + std::to_string(need1) +
                                      " complex values exceed the fixed scratch of " +
                                      std::to_string((long)YTF_NOALLOC_SCRATCH_COMPLEX) + " (64 MiB)");
  double2* scratch = nullptr;
  CK(noalloc_scratch(ctx->device, &scratch));
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device);
  long tiles = ((npix + 63) / 64) * ((ncol + 31) / 32);
  long want = (4L * nsm + tiles - 1) / tiles;
  long fit = (YTF_NOALLOC_SCRATCH_COMPLEX - ncol * n) / (npix * ncol);
  int splits = (int)std::max(1L, std::min(std::min(want, fit), std::max(1L, n / 512)));
  splits = lateral_splits(n, splits);
  double2* S = scratch;
  double2* Gp = scratch + ncol * n;
  const CacheView& v = sp.c;
  sp.zo = z_obs_dev;
  // every element of S and of the used partial sums is written before it is read in this
  // call, so nothing left by an earlier call needs clearing
  CK(launch_strengths2d(sp, S, ctx->stream));
  CK(launch_lateral(v, nx, ny, xs_dev, ys_dev, (int)ncol, S, Gp, splits, ctx->stream));
  CK(launch_reduce_splits2(npix * ncol, splits, Gp, (double2*)out_dev, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return YTF_OK;
}

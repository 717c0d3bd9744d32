// C ABI and host engine: context, device buffers, the per-chunk LM driver.
//
// One LM iteration is a fixed sequence of seven kernels over every island of
// the chunk, captured once into a CUDA graph and replayed; islands carry
// their state and flags on the device (converged islands retire by flag, a
// rejected step re-uses the cached Gauss-Newton blocks), so the host only
// synchronises every UPH_CHECK_EVERY iterations to stop early.  The
// reference syncs the host on every step (island_solver.py:2971-2977).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/uniphot_b200.h"
#include "uph_internal.cuh"

int uph_render_setup();
int uph_solve_setup();
int uph_gram_tc_setup();
void launch_set_probe(const ClassDev& c, cudaStream_t s);
void launch_fill_float(float* p, float v, int n, cudaStream_t s);

#define UPH_CHECK_EVERY 4
#define UPH_MAX_STREAMS 32
#define UPH_HIGH_PRIORITY_STREAMS 4
#define UPH_QUEUE_LANES 8

namespace {

// Device buffer from the device's stream-ordered memory pool: allocated on
// the owning context's stream, released without synchronising the device;
// freed memory stays in the pool (its release threshold is raised at context
// creation) for the next job to reuse.  Every release follows a
// synchronisation of all streams that used the buffer (job and context
// teardown synchronise first), so the free is issued on the legacy stream,
// whose handle stays valid whatever the owner's stream has become.
struct DevBuf {
  void* ptr = nullptr;
  size_t cap = 0;
  void release() {
    if (ptr) cudaFreeAsync(ptr, 0);
    ptr = nullptr;
    cap = 0;
  }
};

// A context buffer that the chunks of a live job may bind (field stacks,
// PSF models, the Sersic table).  The chunk keeps a reference; an upload
// overwrites the buffer in place only when no chunk holds it, and otherwise
// swaps in a fresh allocation, so a job's chunks keep reading the inputs
// they were added with while the context takes the next field (one job may
// hold the chunks of several fields).
using SBuf = std::shared_ptr<DevBuf>;

SBuf sbuf_new() {
  return SBuf(new DevBuf(), [](DevBuf* b) {
    b->release();
    delete b;
  });
}

inline void* sptr(const SBuf& b) { return b ? b->ptr : nullptr; }

struct PolyPsf {
  SBuf coefs, os;
  int nt = 0, nb = 0;
};

}  // namespace

struct uph_ctx {
  int device = 0;
  DevBuf sp[32];   // sparse grid solve: inputs, per-source work, the system
  DevBuf isl[13];  // island decomposition
  int isl_tries = UPH_ISLAND_TRIES_DEFAULT;  // unite attempts per coupled pair
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  // field
  SBuf dstack, wstack;
  int nb = 0, Hp = 0, Wp = 0, pad = 0;
  // psf
  std::map<int, PolyPsf> poly;
  SBuf mog, mog_os;
  int mog_k = 0, mog_nt = 0, mog_nb = 0;
  // table
  SBuf tb_knots, tb_amps, tb_lv, tb_core;
  // the "direct" backend's exponential mixture
  SBuf exp_amp, exp_var;
  int exp_k = 0;
  int tb_n = 0, tb_k = 0;
  double tb_nmin = 0, tb_nmax = 0;
  int* h_active = nullptr;  // pinned
  DevBuf bgc;               // per-tile background coefficients (stack build)
  // events that free the two pinned staging slots of the field upload
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  float timing[4] = {0, 0, 0, 0};
  int64_t launches = 0;
  int sm_count = 148;
};

namespace {

int set_err(uph_ctx* c, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

int cuda_err(uph_ctx* c, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return UPH_OK;
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return set_err(c, UPH_ERR_OOM, "RESOURCE_EXHAUSTED: out of device memory in %s", what);
  }
  return set_err(c, UPH_ERR_CUDA, "CUDA error in %s: %s", what, cudaGetErrorString(e));
}

#define CK(call, what)                              \
  do {                                              \
    cudaError_t _e = (call);                        \
    if (_e != cudaSuccess) return cuda_err(ctx, _e, what); \
  } while (0)

int ensure(uph_ctx* ctx, DevBuf& b, size_t bytes, const char* what) {
  if (bytes == 0) bytes = 16;
  if (b.cap >= bytes) return UPH_OK;
  b.release();
  cudaError_t e = cudaMallocAsync(&b.ptr, bytes, ctx->stream);
  if (e != cudaSuccess) {
    b.ptr = nullptr;
    return cuda_err(ctx, e, what);
  }
  b.cap = bytes;
  return UPH_OK;
}

// ensure() for a bindable buffer: a buffer some chunk holds is left to it
int ensure_shared(uph_ctx* ctx, SBuf& b, size_t bytes, const char* what) {
  if (!b || b.use_count() > 1) b = sbuf_new();
  return ensure(ctx, *b, bytes, what);
}

int upload(uph_ctx* ctx, void* dst, const void* src, size_t bytes,
           const char* what) {
  if (bytes == 0) return UPH_OK;
  if (!src) return set_err(ctx, UPH_ERR_INVALID, "null host pointer for %s", what);
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream), what);
  return UPH_OK;
}

int download(uph_ctx* ctx, void* dst, const void* src, size_t bytes,
             const char* what) {
  if (bytes == 0 || !dst) return UPH_OK;
  CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream), what);
  return UPH_OK;
}

}  // namespace

extern "C" {

int uph_create(int device, uph_ctx** out) {
  if (!out) return UPH_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || device < 0 || device >= ndev) return UPH_ERR_CUDA;
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return UPH_ERR_CUDA;
  uph_ctx* ctx = new uph_ctx();
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (ctx->sm_count <= 0) ctx->sm_count = 148;
  {
    // keep freed chunk buffers cached in the device's default pool: a job's
    // teardown then returns memory without synchronising the device and the
    // next job reuses it (the pool is trimmed when a context is destroyed)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t thr = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  }
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return UPH_ERR_CUDA;
  }
  ctx->own_stream = true;
  if (uph_render_setup() != 0 || uph_solve_setup() != 0 || uph_gram_tc_setup() != 0 ||
      sparse_setup() != 0 || gal_fft_setup() != 0) {
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return UPH_ERR_CUDA;
  }
  if (cudaMallocHost((void**)&ctx->h_active, sizeof(int)) != cudaSuccess) {
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return UPH_ERR_CUDA;
  }
  for (auto& ev : ctx->ev) cudaEventCreate(&ev);
  *out = ctx;
  return UPH_OK;
}

int uph_destroy(uph_ctx* ctx) {
  if (!ctx) return UPH_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->dstack.reset();
  ctx->wstack.reset();
  ctx->poly.clear();
  ctx->mog.reset();
  ctx->mog_os.reset();
  ctx->tb_knots.reset();
  ctx->tb_amps.reset();
  ctx->tb_lv.reset();
  ctx->tb_core.reset();
  ctx->exp_amp.reset();
  ctx->exp_var.reset();
  for (auto& b : ctx->sp) b.release();
  ctx->bgc.release();
  for (auto& e : ctx->stage_ev)
    if (e) cudaEventDestroy(e);
  for (auto& b : ctx->isl) b.release();
  for (auto& ev : ctx->ev)
    if (ev) cudaEventDestroy(ev);
  if (ctx->h_active) cudaFreeHost(ctx->h_active);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->stream = nullptr;
  {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess)
      cudaMemPoolTrimTo(pool, 0);
  }
  delete ctx;
  return UPH_OK;
}

const char* uph_last_error(const uph_ctx* ctx) {
  return ctx ? ctx->err.c_str() : "null context";
}

int uph_set_stream(uph_ctx* ctx, void* stream) {
  if (!ctx) return UPH_ERR_INVALID;
  if (stream == nullptr) {
    if (!ctx->own_stream) {
      cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
      ctx->own_stream = true;
    }
    return UPH_OK;
  }
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->stream = (cudaStream_t)stream;
  ctx->own_stream = false;
  return UPH_OK;
}

void* uph_get_stream(const uph_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

static int upload_field_impl(uph_ctx* ctx, const float* d, const float* w,
                             int nb, int Hp, int Wp, int pad,
                             cudaMemcpyKind kind) {
  if (!ctx) return UPH_ERR_INVALID;
  if (!d || !w || nb <= 0 || Hp <= 0 || Wp <= 0 || pad < 0)
    return set_err(ctx, UPH_ERR_INVALID, "invalid field arguments");
  cudaSetDevice(ctx->device);
  size_t bytes = sizeof(float) * (size_t)nb * Hp * Wp;
  int rc = ensure_shared(ctx, ctx->dstack, bytes, "field data");
  if (rc) return rc;
  rc = ensure_shared(ctx, ctx->wstack, bytes, "field invvar");
  if (rc) return rc;
  CK(cudaMemcpyAsync(sptr(ctx->dstack), d, bytes, kind, ctx->stream), "field copy");
  CK(cudaMemcpyAsync(sptr(ctx->wstack), w, bytes, kind, ctx->stream), "field copy");
  CK(cudaStreamSynchronize(ctx->stream), "field copy");
  ctx->nb = nb;
  ctx->Hp = Hp;
  ctx->Wp = Wp;
  ctx->pad = pad;
  return UPH_OK;
}

int uph_upload_field(uph_ctx* ctx, const float* d, const float* w,
                     int32_t nb, int32_t Hp, int32_t Wp, int32_t pad) {
  return upload_field_impl(ctx, d, w, nb, Hp, Wp, pad, cudaMemcpyHostToDevice);
}

// Process-wide pool of pinned staging buffers for field uploads (portable
// across contexts and devices): an upload takes one at least as large as it
// needs, or allocates one, and gives it back, so contexts created per call
// do not pay the page-locking each time and concurrent uploads each get
// their own.
namespace {
std::mutex g_stage_mu;
std::vector<std::pair<float*, size_t>> g_stage_free;

float* stage_take(size_t floats, size_t* got) {
  {
    std::lock_guard<std::mutex> lk(g_stage_mu);
    for (size_t i = 0; i < g_stage_free.size(); ++i)
      if (g_stage_free[i].second >= floats) {
        float* p = g_stage_free[i].first;
        *got = g_stage_free[i].second;
        g_stage_free.erase(g_stage_free.begin() + (long)i);
        return p;
      }
  }
  float* p = nullptr;
  if (cudaHostAlloc((void**)&p, sizeof(float) * floats, cudaHostAllocPortable) != cudaSuccess)
    return nullptr;
  *got = floats;
  return p;
}

void stage_give(float* p, size_t floats) {
  std::lock_guard<std::mutex> lk(g_stage_mu);
  g_stage_free.emplace_back(p, floats);
}
}  // namespace

// Copy n floats from pageable src to pinned dst with up to `threads` host
// threads (contiguous slices).
// Nothing throws out of it: if a thread cannot be started, the calling
// thread copies what no thread took.
static void parallel_copy(float* dst, const float* src, size_t n, int threads) {
  if (threads <= 1 || n < (size_t)1 << 20) {
    std::memcpy(dst, src, n * sizeof(float));
    return;
  }
  std::vector<std::thread> pool;
  const size_t per = (n + threads - 1) / threads;
  size_t taken = 0;   // [0, taken) is handed to started threads
  try {
    pool.reserve((size_t)threads);
    for (int t = 0; t < threads; ++t) {
      const size_t lo = (size_t)t * per, hi = std::min(n, lo + per);
      if (lo >= hi) break;
      pool.emplace_back([=] { std::memcpy(dst + lo, src + lo, (hi - lo) * sizeof(float)); });
      taken = hi;
    }
  } catch (...) {
  }
  if (taken < n) std::memcpy(dst + taken, src + taken, (n - taken) * sizeof(float));
  for (auto& th : pool) th.join();
}

int uph_upload_field_unpadded(uph_ctx* ctx, const float* d, const float* w,
                              int32_t nb, int32_t H, int32_t W, int32_t pad) {
  if (!ctx) return UPH_ERR_INVALID;
  if (!d || !w || nb <= 0 || H <= 0 || W <= 0 || pad < 0)
    return set_err(ctx, UPH_ERR_INVALID, "invalid field arguments");
  cudaSetDevice(ctx->device);
  const int Hp = H + 2 * pad, Wp = W + 2 * pad;
  const size_t bytes = sizeof(float) * (size_t)nb * Hp * Wp;
  int rc = ensure_shared(ctx, ctx->dstack, bytes, "field data");
  if (rc) return rc;
  rc = ensure_shared(ctx, ctx->wstack, bytes, "field invvar");
  if (rc) return rc;
  CK(cudaMemsetAsync(sptr(ctx->dstack), 0, bytes, ctx->stream), "field pad");
  CK(cudaMemsetAsync(sptr(ctx->wstack), 0, bytes, ctx->stream), "field pad");
  // The pageable host arrays go through two pinned slots of one band each:
  // host threads fill one slot while the copy engine drains the other, so
  // the upload runs at the multi-threaded host-copy rate instead of the
  // driver's single-threaded pageable staging.
  const size_t band = (size_t)H * W;
  for (auto& e : ctx->stage_ev)
    if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "field staging");
  size_t got = 0;
  float* stage = stage_take(4 * band, &got);
  if (!stage) return set_err(ctx, UPH_ERR_OOM, "RESOURCE_EXHAUSTED: pinned field staging");
  const int threads = (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  cudaError_t ce = cudaSuccess;
  for (int b = 0; b < nb && ce == cudaSuccess; ++b) {
    const int slot = b & 1;
    float* sd = stage + (size_t)slot * 2 * band;
    float* sw = sd + band;
    if (b >= 2) ce = cudaEventSynchronize(ctx->stage_ev[slot]);
    if (ce != cudaSuccess) break;
    parallel_copy(sd, d + (size_t)b * band, band, threads);
    parallel_copy(sw, w + (size_t)b * band, band, threads);
    const size_t o = ((size_t)b * Hp + pad) * Wp + pad;
    ce = cudaMemcpy2DAsync((float*)sptr(ctx->dstack) + o, sizeof(float) * Wp, sd,
                           sizeof(float) * W, sizeof(float) * W, H, cudaMemcpyHostToDevice,
                           ctx->stream);
    if (ce == cudaSuccess)
      ce = cudaMemcpy2DAsync((float*)sptr(ctx->wstack) + o, sizeof(float) * Wp, sw,
                             sizeof(float) * W, sizeof(float) * W, H, cudaMemcpyHostToDevice,
                             ctx->stream);
    if (ce == cudaSuccess) ce = cudaEventRecord(ctx->stage_ev[slot], ctx->stream);
  }
  // the staging buffer goes back to the pool only once its copies are done
  const cudaError_t se = cudaStreamSynchronize(ctx->stream);
  stage_give(stage, got);
  if (ce != cudaSuccess) return cuda_err(ctx, ce, "field copy");
  if (se != cudaSuccess) return cuda_err(ctx, se, "field copy");
  ctx->nb = nb;
  ctx->Hp = Hp;
  ctx->Wp = Wp;
  ctx->pad = pad;
  return UPH_OK;
}

int uph_upload_field_device(uph_ctx* ctx, const float* d, const float* w,
                            int32_t nb, int32_t Hp, int32_t Wp, int32_t pad) {
  return upload_field_impl(ctx, d, w, nb, Hp, Wp, pad, cudaMemcpyDeviceToDevice);
}

int uph_upload_psf_poly(uph_ctx* ctx, int32_t tier, const float* coefs,
                        const float* os, int32_t nb, int32_t nt) {
  if (!ctx) return UPH_ERR_INVALID;
  if (!coefs || !os || tier <= 0 || (tier % 2) == 0 || nb <= 0 ||
      !(nt == 1 || nt == 3 || nt == 6 || nt == 10 || nt == 15 || nt == 21))
    return set_err(ctx, UPH_ERR_INVALID, "invalid PSF polynomial (tier %d, nt %d)", tier, nt);
  cudaSetDevice(ctx->device);
  PolyPsf& p = ctx->poly[tier];
  size_t bytes = sizeof(float) * (size_t)nb * tier * tier * nt;
  int rc = ensure_shared(ctx, p.coefs, bytes, "psf coefs");
  if (rc) return rc;
  rc = ensure_shared(ctx, p.os, sizeof(float) * 4 * nb, "psf origin");
  if (rc) return rc;
  CK(cudaMemcpyAsync(sptr(p.coefs), coefs, bytes, cudaMemcpyHostToDevice, ctx->stream), "psf");
  CK(cudaMemcpyAsync(sptr(p.os), os, sizeof(float) * 4 * nb, cudaMemcpyHostToDevice, ctx->stream), "psf");
  CK(cudaStreamSynchronize(ctx->stream), "psf");
  p.nt = nt;
  p.nb = nb;
  return UPH_OK;
}

int uph_upload_psf_mog(uph_ctx* ctx, const float* params, const float* os,
                       int32_t nb, int32_t K, int32_t nt) {
  if (!ctx) return UPH_ERR_INVALID;
  if (!params || !os || nb <= 0 || K <= 0 || K > UPH_MAXKPSF ||
      !(nt == 1 || nt == 3 || nt == 6 || nt == 10 || nt == 15 || nt == 21))
    return set_err(ctx, UPH_ERR_INVALID, "invalid MoG PSF (K %d, nt %d)", K, nt);
  cudaSetDevice(ctx->device);
  size_t bytes = sizeof(float) * (size_t)nb * K * 4 * nt;
  int rc = ensure_shared(ctx, ctx->mog, bytes, "mog psf");
  if (rc) return rc;
  rc = ensure_shared(ctx, ctx->mog_os, sizeof(float) * 4 * nb, "mog origin");
  if (rc) return rc;
  CK(cudaMemcpyAsync(sptr(ctx->mog), params, bytes, cudaMemcpyHostToDevice, ctx->stream), "mog");
  CK(cudaMemcpyAsync(sptr(ctx->mog_os), os, sizeof(float) * 4 * nb, cudaMemcpyHostToDevice, ctx->stream), "mog");
  CK(cudaStreamSynchronize(ctx->stream), "mog");
  ctx->mog_k = K;
  ctx->mog_nt = nt;
  ctx->mog_nb = nb;
  return UPH_OK;
}

int uph_upload_sersic_table(uph_ctx* ctx, const double* knots,
                            const double* amps, const double* lv,
                            const double* core, int32_t n, int32_t kmax,
                            double nmin, double nmax) {
  if (!ctx) return UPH_ERR_INVALID;
  if (!knots || !amps || !lv || !core || n < 2 || kmax <= 0 || kmax > UPH_MAXGAL - 1)
    return set_err(ctx, UPH_ERR_INVALID, "invalid Sersic table");
  cudaSetDevice(ctx->device);
  int rc = ensure_shared(ctx, ctx->tb_knots, sizeof(double) * n, "table");
  if (!rc) rc = ensure_shared(ctx, ctx->tb_amps, sizeof(double) * n * kmax, "table");
  if (!rc) rc = ensure_shared(ctx, ctx->tb_lv, sizeof(double) * n * kmax, "table");
  if (!rc) rc = ensure_shared(ctx, ctx->tb_core, sizeof(double) * n, "table");
  if (rc) return rc;
  CK(cudaMemcpyAsync(sptr(ctx->tb_knots), knots, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream), "table");
  CK(cudaMemcpyAsync(sptr(ctx->tb_amps), amps, sizeof(double) * n * kmax, cudaMemcpyHostToDevice, ctx->stream), "table");
  CK(cudaMemcpyAsync(sptr(ctx->tb_lv), lv, sizeof(double) * n * kmax, cudaMemcpyHostToDevice, ctx->stream), "table");
  CK(cudaMemcpyAsync(sptr(ctx->tb_core), core, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream), "table");
  CK(cudaStreamSynchronize(ctx->stream), "table");
  ctx->tb_n = n;
  ctx->tb_k = kmax;
  ctx->tb_nmin = nmin;
  ctx->tb_nmax = nmax;
  return UPH_OK;
}

int uph_subtract_tile_backgrounds(uph_ctx* ctx, int32_t n_tiles, const int32_t* tiles,
                                  const float* coefs, int32_t order, const double* norm) {
  if (!ctx) return UPH_ERR_INVALID;
  if (!sptr(ctx->dstack)) return set_err(ctx, UPH_ERR_STATE, "no field uploaded");
  if (ctx->dstack.use_count() > 1)
    return set_err(ctx, UPH_ERR_STATE,
                   "the field is held by a live job's chunks: upload it again to change it");
  if (n_tiles < 0 || (n_tiles > 0 && (!tiles || !coefs)) || !norm || order < 0 || order > 2)
    return set_err(ctx, UPH_ERR_INVALID, "invalid tile backgrounds (%d tiles, order %d)",
                   n_tiles, order);
  if (norm[1] == 0.0 || norm[3] == 0.0)
    return set_err(ctx, UPH_ERR_INVALID, "zero background normalisation scale");
  const int M = order == 0 ? 1 : (order == 1 ? 3 : 6);
  const int H = ctx->Hp - 2 * ctx->pad, W = ctx->Wp - 2 * ctx->pad;
  for (int t = 0; t < n_tiles; ++t) {
    const int* r = tiles + 4 * (size_t)t;
    if (r[0] < 0 || r[1] < 0 || r[2] < r[0] || r[3] < r[1] || r[2] > W || r[3] > H)
      return set_err(ctx, UPH_ERR_INVALID, "tile %d core (%d, %d, %d, %d) outside the %d x %d field",
                     t, r[0], r[1], r[2], r[3], W, H);
  }
  if (n_tiles == 0) return UPH_OK;
  cudaSetDevice(ctx->device);
  const size_t bytes = sizeof(float) * (size_t)n_tiles * ctx->nb * M;
  int rc = ensure(ctx, ctx->bgc, bytes, "tile backgrounds");
  if (rc) return rc;
  CK(cudaMemcpyAsync(ctx->bgc.ptr, coefs, bytes, cudaMemcpyHostToDevice, ctx->stream),
     "tile backgrounds");
  for (int t = 0; t < n_tiles; ++t) {
    const int* r = tiles + 4 * (size_t)t;
    launch_tile_bg_subtract((float*)sptr(ctx->dstack), ctx->nb, ctx->Hp, ctx->Wp, ctx->pad, r[0],
                            r[1], r[2] - r[0], r[3] - r[1],
                            (const float*)ctx->bgc.ptr + (size_t)t * ctx->nb * M, M, norm,
                            ctx->sm_count, ctx->stream);
  }
  CK(cudaGetLastError(), "tile backgrounds");
  CK(cudaStreamSynchronize(ctx->stream), "tile backgrounds");
  return UPH_OK;
}

// Waves of the ordered stamp subtraction: a source goes one wave after the
// latest earlier source whose T x T stamp (corner ix, iy) overlaps its own
// (corners closer than T on both axes), so each wave's stamps are disjoint
// and every pixel sees its sources in index order; the earlier sources are
// found in the 3 x 3 cells of pitch T.  Returns the number of waves.
static int scene_waves(int n, const int* ix, const int* iy, int T, int* wave) {
  std::map<std::pair<int, int>, std::vector<int>> cells;
  auto cell_of = [&](int v) { return v >= 0 ? v / T : -((-v + T - 1) / T); };
  int nwave = 0;
  for (int i = 0; i < n; ++i) {
    const int cx = cell_of(ix[i]), cy = cell_of(iy[i]);
    int w = 0;
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        auto it = cells.find({cx + dx, cy + dy});
        if (it == cells.end()) continue;
        for (int j : it->second)
          if (std::abs(ix[i] - ix[j]) < T && std::abs(iy[i] - iy[j]) < T)
            w = std::max(w, wave[j] + 1);
      }
    wave[i] = w;
    nwave = std::max(nwave, w + 1);
    cells[{cx, cy}].push_back(i);
  }
  return nwave;
}

int uph_scene_waves(int32_t n, const double* x, const double* y, int32_t T, int32_t* wave) {
  if (n < 0 || (n > 0 && (!x || !y || !wave)) || T <= 0) return -1;
  std::vector<int> ix(n), iy(n);
  for (int i = 0; i < n; ++i) {
    if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || std::fabs(x[i]) > 1e8 ||
        std::fabs(y[i]) > 1e8)
      return -1;
    ix[i] = (int)std::nearbyint(x[i]) - T / 2;
    iy[i] = (int)std::nearbyint(y[i]) - T / 2;
  }
  return scene_waves(n, ix.data(), iy.data(), T, wave);
}

int uph_scene_subtract_stars(uph_ctx* ctx, int32_t n, const double* x, const double* y,
                             const float* flux, int32_t T, int32_t nt, const float* coefs,
                             const float* origin_scale) {
  if (!ctx) return UPH_ERR_INVALID;
  if (!sptr(ctx->dstack)) return set_err(ctx, UPH_ERR_STATE, "no field uploaded");
  if (ctx->dstack.use_count() > 1)
    return set_err(ctx, UPH_ERR_STATE,
                   "the field is held by a live job's chunks: upload it again to change it");
  if (n < 0 || (n > 0 && (!x || !y || !flux || !coefs || !origin_scale)) || T <= 0 ||
      (T % 2) == 0 || !(nt == 1 || nt == 3 || nt == 6 || nt == 10 || nt == 15 || nt == 21))
    return set_err(ctx, UPH_ERR_INVALID, "invalid scene subtraction (n %d, T %d, nt %d)", n, T,
                   nt);
  if (sparse_stamp_smem(T, T) > 200 * 1024)
    return set_err(ctx, UPH_ERR_INVALID, "stamp side %d too large", T);
  if (n == 0) return UPH_OK;
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(x[i]) || !std::isfinite(y[i]) || std::fabs(x[i]) > 1e8 ||
        std::fabs(y[i]) > 1e8)
      return set_err(ctx, UPH_ERR_INVALID, "source %d position not finite or out of range", i);
  cudaSetDevice(ctx->device);
  const int nb = ctx->nb;
  // stamp corners as the reference computes them (round half to even of
  // the float64 position, island_stage.py:2000-2001); the stamps render at
  // the float32 position
  std::vector<int> ix(n), iy(n);
  std::vector<float> xf(n), yf(n);
  for (int i = 0; i < n; ++i) {
    ix[i] = (int)std::nearbyint(x[i]) - T / 2;
    iy[i] = (int)std::nearbyint(y[i]) - T / 2;
    xf[i] = (float)x[i];
    yf[i] = (float)y[i];
  }
  std::vector<int> wave(n, 0);
  const int nwave = scene_waves(n, ix.data(), iy.data(), T, wave.data());
  std::vector<int> srcs(n), off(nwave + 1, 0);
  for (int i = 0; i < n; ++i) ++off[wave[i] + 1];
  for (int w = 0; w < nwave; ++w) off[w + 1] += off[w];
  {
    std::vector<int> pos(off.begin(), off.end() - 1);
    for (int i = 0; i < n; ++i) srcs[pos[wave[i]]++] = i;
  }
  std::vector<float> fl((size_t)nb * n);
  for (int i = 0; i < n; ++i)
    for (int b = 0; b < nb; ++b) fl[(size_t)b * n + i] = flux[(size_t)i * nb + b];
  DevBuf dx, dy, dfl, dcf, dos, dst, dix, diy, dscr, dsrc;
  auto release = [&] {
    for (DevBuf* b : {&dx, &dy, &dfl, &dcf, &dos, &dst, &dix, &diy, &dscr, &dsrc}) b->release();
  };
  int rc = UPH_OK;
  const size_t TT = (size_t)T * T;
  if (!rc) rc = ensure(ctx, dx, sizeof(float) * n, "scene");
  if (!rc) rc = ensure(ctx, dy, sizeof(float) * n, "scene");
  if (!rc) rc = ensure(ctx, dfl, sizeof(float) * nb * (size_t)n, "scene");
  if (!rc) rc = ensure(ctx, dcf, sizeof(float) * nb * TT * nt, "scene");
  if (!rc) rc = ensure(ctx, dos, sizeof(float) * 4 * nb, "scene");
  if (!rc) rc = ensure(ctx, dst, sizeof(float) * TT * n, "scene");
  if (!rc) rc = ensure(ctx, dix, sizeof(int) * n, "scene");
  if (!rc) rc = ensure(ctx, diy, sizeof(int) * n, "scene");
  if (!rc) rc = ensure(ctx, dscr, sizeof(int) * 2 * n, "scene");
  if (!rc) rc = ensure(ctx, dsrc, sizeof(int) * n, "scene");
  if (!rc) rc = upload(ctx, dx.ptr, xf.data(), sizeof(float) * n, "scene");
  if (!rc) rc = upload(ctx, dy.ptr, yf.data(), sizeof(float) * n, "scene");
  if (!rc) rc = upload(ctx, dfl.ptr, fl.data(), sizeof(float) * nb * (size_t)n, "scene");
  if (!rc) rc = upload(ctx, dcf.ptr, coefs, sizeof(float) * nb * TT * nt, "scene");
  if (!rc) rc = upload(ctx, dos.ptr, origin_scale, sizeof(float) * 4 * nb, "scene");
  if (!rc) rc = upload(ctx, dix.ptr, ix.data(), sizeof(int) * n, "scene");
  if (!rc) rc = upload(ctx, diy.ptr, iy.data(), sizeof(int) * n, "scene");
  if (!rc) rc = upload(ctx, dsrc.ptr, srcs.data(), sizeof(int) * n, "scene");
  if (rc) {
    cudaStreamSynchronize(ctx->stream);
    release();
    return rc;
  }
  const size_t plane = (size_t)ctx->Hp * ctx->Wp;
  for (int b = 0; b < nb; ++b) {
    // the band's stamps (their own corners go to scratch: the corners above
    // come from the float64 positions)
    launch_star_stamps(n, T, T, (const float*)dcf.ptr + (size_t)b * TT * nt, nt,
                       (const float*)dos.ptr + 4 * b, (const float*)dx.ptr,
                       (const float*)dy.ptr, (float*)dst.ptr, (int*)dscr.ptr,
                       (int*)dscr.ptr + n, ctx->stream);
    for (int w = 0; w < nwave; ++w)
      launch_scene_sub_wave((float*)sptr(ctx->dstack) + b * plane, ctx->Hp, ctx->Wp, ctx->pad,
                            T, (const int*)dsrc.ptr + off[w], off[w + 1] - off[w],
                            (const float*)dst.ptr, (const int*)dix.ptr, (const int*)diy.ptr,
                            (const float*)dfl.ptr + (size_t)b * n, ctx->stream);
  }
  cudaError_t e = cudaGetLastError();
  const cudaError_t se = cudaStreamSynchronize(ctx->stream);
  release();
  if (e != cudaSuccess) return cuda_err(ctx, e, "scene subtraction");
  if (se != cudaSuccess) return cuda_err(ctx, se, "scene subtraction");
  return UPH_OK;
}

int uph_download_field(uph_ctx* ctx, float* data, float* invvar) {
  if (!ctx) return UPH_ERR_INVALID;
  if (!sptr(ctx->dstack)) return set_err(ctx, UPH_ERR_STATE, "no field uploaded");
  cudaSetDevice(ctx->device);
  const size_t bytes = sizeof(float) * (size_t)ctx->nb * ctx->Hp * ctx->Wp;
  int rc = download(ctx, data, sptr(ctx->dstack), bytes, "field");
  if (!rc) rc = download(ctx, invvar, sptr(ctx->wstack), bytes, "field");
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->stream), "field");
  return UPH_OK;
}

int uph_upload_exp_mog(uph_ctx* ctx, const float* amp, const float* var, int32_t k) {
  if (!ctx) return UPH_ERR_INVALID;
  if (!amp || !var || k <= 0 || k > UPH_MAXGAL)
    return set_err(ctx, UPH_ERR_INVALID, "invalid exponential mixture (%d components)", k);
  cudaSetDevice(ctx->device);
  int rc = ensure_shared(ctx, ctx->exp_amp, sizeof(float) * k, "exp mixture");
  if (!rc) rc = ensure_shared(ctx, ctx->exp_var, sizeof(float) * k, "exp mixture");
  if (rc) return rc;
  CK(cudaMemcpyAsync(sptr(ctx->exp_amp), amp, sizeof(float) * k, cudaMemcpyHostToDevice,
                     ctx->stream), "exp mixture");
  CK(cudaMemcpyAsync(sptr(ctx->exp_var), var, sizeof(float) * k, cudaMemcpyHostToDevice,
                     ctx->stream), "exp mixture");
  CK(cudaStreamSynchronize(ctx->stream), "exp mixture");
  ctx->exp_k = k;
  return UPH_OK;
}

int uph_last_timing(const uph_ctx* ctx, float* ms4) {
  if (!ctx || !ms4) return UPH_ERR_INVALID;
  for (int i = 0; i < 4; ++i) ms4[i] = ctx->timing[i];
  return UPH_OK;
}

int64_t uph_last_launch_count(const uph_ctx* ctx) { return ctx ? ctx->launches : -1; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Chunks and jobs
// ---------------------------------------------------------------------------

struct Chunk {
  ClassDev c{};
  std::map<std::string, DevBuf> bufs;
  int n = 0, N = 0, nb = 0, nP = 0;
  bool fresh = true;
  std::vector<int> h_nst0;
  std::vector<uint8_t> h_flags0;
  float* d_lam0 = nullptr;
  float* d_chi20 = nullptr;
  int* d_consec0 = nullptr;
  int* d_nrej0 = nullptr;
  int* d_nst0 = nullptr;
  uint8_t* d_flags0 = nullptr;
  int* d_nsame0 = nullptr;     // "changed" tracker at the chunk's start
  float* d_prej0 = nullptr;
  uint8_t* d_divl0 = nullptr;
  float* d_p0 = nullptr;
  uint8_t* d_div = nullptr;
  uint8_t* d_rail = nullptr;       // trust region: bound-pinned islands
  float* d_cjac = nullptr;         // flux sensitivities (flux_marg only)
  // scene subtract: the field stacks and window origins the private
  // windows are copied from, the seeds and S1 fluxes of the add-back
  bool scene = false;
  const float* fd = nullptr;
  const float* fw = nullptr;
  int fHp = 0, fWp = 0;
  const int* ox_f = nullptr;
  const int* oy_f = nullptr;
  float* d_seed = nullptr;
  float* d_msf = nullptr;
  bool perr_out = false;           // param_errors requested
  std::vector<SBuf> bound;         // the context buffers the chunk reads
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaEvent_t ev_group = nullptr;
  cudaEvent_t ev_done = nullptr;   // end of the chunk's last solve (timed)
  float done_ms = 0.f;             // its time from the solve's start
  bool done = false;
  int iters = 0;
  int slot = 0;
  int graph_kernels = 0;
  ~Chunk() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    if (ev_group) cudaEventDestroy(ev_group);
    if (ev_done) cudaEventDestroy(ev_done);
    for (auto& kv : bufs) kv.second.release();
  }
};

// One lane of the queue engine: a set of chunks on one stream with its own
// work lists (linearisation and trial phases) and iteration graph.
struct QueueLane {
  std::vector<int> chunks;   // chunk indices, heaviest first
  int off = 0, n = 0;        // the lane's islands in the job's order
  QueueList ql[2];
  size_t sm_rlin = 0, sm_rtry = 0, sm_glin = 0, sm_gtc = 0, sm_asm = 0, sm_step = 0,
         sm_trial = 0;
  bool any_tc = false, any_red = false, any_fft = false, any_glr = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int graph_kernels = 0;
  cudaEvent_t ev = nullptr;
  int iters = 0;
  bool live = false, inflight = false;
  void release() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    if (ev) cudaEventDestroy(ev);
    gexec = nullptr;
    graph = nullptr;
    ev = nullptr;
  }
};

struct uph_job {
  uph_ctx* ctx = nullptr;
  std::vector<Chunk*> chunks;
  std::vector<cudaStream_t> streams;
  int* h_active = nullptr;  // pinned, one slot per chunk
  int h_active_cap = 0;
  int* h_stall = nullptr;   // pinned: per chunk, active and stalled islands
  int h_stall_cap = 0;
  bool profile = false;
  float ktime[WK_KINDS] = {};
  int64_t kcount[WK_KINDS] = {};
  double kbytes[WK_KINDS] = {};
  double kflops[WK_KINDS] = {};
  double kexps[WK_KINDS] = {};
  unsigned long long* d_work = nullptr;   // (WK_KINDS, WK_FIELDS) device counters
  // LM loop engine: UPH_ENGINE_QUEUE runs each phase of every chunk as one
  // persistent queue kernel per kind (device-compacted active islands, one
  // CUDA graph per iteration for the whole job); UPH_ENGINE_CHUNKS runs each
  // chunk's iterations as its own graph on one of several streams
  int engine = UPH_ENGINE_CHUNKS;
  DevBuf q_cls, q_order, q_count, q_act[2], q_n[2], q_pre[2], q_next[2];
  std::vector<QueueLane> lanes;
  int lanes_max = 0;        // lanes of the queue engine (0: UPH_QUEUE_LANES)
  bool q_graph_valid = false;
  ~uph_job() {
    for (auto& ln : lanes) ln.release();
    for (DevBuf* b : {&q_cls, &q_order, &q_count, &q_act[0], &q_act[1], &q_n[0], &q_n[1],
                      &q_pre[0], &q_pre[1], &q_next[0], &q_next[1]})
      b->release();
    for (auto* c : chunks) delete c;
    for (auto s : streams) cudaStreamDestroy(s);
    if (h_active) cudaFreeHost(h_active);
    if (h_stall) cudaFreeHost(h_stall);
    if (d_work) cudaFree(d_work);
  }
};

namespace {

template <class T>
T* cbuf(uph_ctx* ctx, Chunk* ch, const char* name, size_t count, int* rc) {
  if (*rc != UPH_OK) return nullptr;
  DevBuf& b = ch->bufs[name];
  *rc = ensure(ctx, b, count * sizeof(T), name);
  return (T*)b.ptr;
}

// Kernel launcher that optionally brackets each launch with events.
struct Launcher {
  uph_job* job;
  cudaStream_t s;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>>* rec;
  template <class F>
  void operator()(int kind, F&& fn, int kernels = 1) {
    if (rec) {
      cudaEvent_t a, b;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, s);
      fn();
      cudaEventRecord(b, s);
      rec->push_back({kind, {a, b}});
    } else {
      fn();
    }
    job->ctx->launches += kernels;
  }
};

void iteration(const ClassDev& c, Launcher& L) {
  cudaStream_t s = L.s;
  L(0, [&] { launch_render(c, c.p, PH_LIN, s); }, 2);
  L(1, [&] { launch_gram_lin(c, s); }, c.gl_split > 1 ? 2 : 1);
  if (c.tc_min_rows < (1 << 30))
    L(WK_GRAM_TC, [&] { launch_gram_tc(c, s); }, c.tc_split > 1 ? 2 : 1);
  L(2, [&] { launch_assemble(c, s); });
  L(3, [&] { launch_step(c, PH_TRIAL, 0, 0.f, 0, s); });
  L(0, [&] { launch_render(c, c.p_try, PH_TRIAL, s); }, 2);
  L(4, [&] { launch_gram_trial(c, c.p_try, PH_TRIAL, 0, c.ftry, c.acond_try, s); });
  L(5, [&] { launch_accept(c, PH_TRIAL, s); });
}

int add_chunk(uph_ctx* ctx, Chunk* ch, const uph_class_desc* cls,
              const uph_chunk_in* in) {
  const int n = in->n_islands, N = cls->nsrc, B = cls->bbox, T = cls->tier;
  if (n <= 0) return set_err(ctx, UPH_ERR_INVALID, "empty chunk");
  if (N <= 0 || N > UPH_MAXN)
    return set_err(ctx, UPH_ERR_INVALID, "nsrc class %d outside 1..%d", N, UPH_MAXN);
  if (B <= 0 || T <= 0 || (T % 2) == 0)
    return set_err(ctx, UPH_ERR_INVALID, "invalid bbox %d / tier %d", B, T);
  if (!sptr(ctx->dstack)) return set_err(ctx, UPH_ERR_STATE, "no field uploaded");
  if (!in->ox || !in->oy || !in->x0b || !in->y0b || !in->stype || !in->n_frozen ||
      !in->free_n || !in->mmask || !in->keep || !in->p0 || !in->lower ||
      !in->upper || !in->prior_mean || !in->prior_inv_sigma)
    return set_err(ctx, UPH_ERR_INVALID, "null input array");
  const int nb = ctx->nb;
  const int mode = cls->render_mode;
  const PolyPsf* pp = nullptr;
  if (mode == UPH_RENDER_REFERENCE) {
    auto it = ctx->poly.find(T);
    if (it == ctx->poly.end())
      return set_err(ctx, UPH_ERR_STATE, "no polynomial PSF uploaded for tier %d", T);
    pp = &it->second;
    if (pp->nb != nb) return set_err(ctx, UPH_ERR_INVALID, "PSF band count mismatch");
  } else if (mode == UPH_RENDER_ANALYTIC) {
    if (!sptr(ctx->mog) || ctx->mog_nb != nb)
      return set_err(ctx, UPH_ERR_STATE, "no analytic PSF uploaded for %d bands", nb);
  } else {
    return set_err(ctx, UPH_ERR_INVALID, "unknown render mode %d", mode);
  }
  const int nP = 6 * N;
  const int nbg = cls->bg_joint ? UPH_MAXBG : 0;
  std::vector<int> nL(n), nr(n);
  int Kmax = 1, nLmax = 1, R = 1;
  bool any_gal = false;
  for (int i = 0; i < n; ++i) {
    int cnt = 0;
    bool seen_pad = false;
    for (int k = 0; k < N; ++k) {
      bool mm = in->mmask[(size_t)i * N + k] != 0;
      if (mm && seen_pad)
        return set_err(ctx, UPH_ERR_INVALID, "island %d: real member slots must come first", i);
      if (!mm) seen_pad = true; else ++cnt;
    }
    if (cnt == 0) return set_err(ctx, UPH_ERR_INVALID, "island %d has no members", i);
    nr[i] = cnt;
    int live = 0;
    for (int k = 0; k < cnt; ++k) {
      const int st = in->stype[(size_t)i * N + k];
      if (st < 0 || st > 3) return set_err(ctx, UPH_ERR_INVALID, "bad source type %d", st);
      const bool gal = st != 0;
      any_gal = any_gal || gal;
      int lk = 0;
      for (int j = 0; j < 6; ++j)
        if (in->keep[((size_t)i * N + k) * 6 + j] && (j < 2 || gal)) ++lk;
      live += lk;
      R = std::max(R, 1 + lk);
    }
    nL[i] = live;
    nLmax = std::max(nLmax, live);
    Kmax = std::max(Kmax, live + cnt + nbg + 1);
    const int ox = in->ox[i], oy = in->oy[i];
    if (ox < 0 || oy < 0 || ox + B > ctx->Wp || oy + B > ctx->Hp)
      return set_err(ctx, UPH_ERR_INVALID, "island %d window outside the padded field", i);
  }
  if (nLmax > UPH_MAXLIVE) return set_err(ctx, UPH_ERR_INVALID, "too many live parameters");
  if (cls->render_direct && mode != UPH_RENDER_REFERENCE)
    return set_err(ctx, UPH_ERR_INVALID, "render_direct needs the reference render mode");
  const bool direct = cls->render_direct && any_gal;
  if (direct) {
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < nr[i]; ++k)
        if (in->stype[(size_t)i * N + k] > 1)
          return set_err(ctx, UPH_ERR_INVALID,
                         "the direct backend renders STAR and EXP sources only");
    if (T > UPH_DIRECT_MAX_T)
      return set_err(ctx, UPH_ERR_INVALID, "the direct backend takes tiers up to %d (tier %d)",
                     UPH_DIRECT_MAX_T, T);
    if (!sptr(ctx->exp_amp) || ctx->exp_k <= 0)
      return set_err(ctx, UPH_ERR_STATE, "no exponential mixture uploaded");
  }
  if (any_gal && !direct && mode == UPH_RENDER_REFERENCE && fft_pad_for(T) > 512)
    return set_err(ctx, UPH_ERR_INVALID,
                   "reference-mode galaxies: tier %d needs a Fourier grid above 512", T);
  if (any_gal && !sptr(ctx->tb_knots))
    return set_err(ctx, UPH_ERR_STATE, "no Sersic table uploaded");
  std::vector<int16_t> row_k((size_t)n * Kmax, 0), row_s((size_t)n * Kmax, -1),
      row_p((size_t)n * Kmax, -1);
  for (int i = 0; i < n; ++i) {
    int r = 0;
    for (int k = 0; k < nr[i]; ++k) {
      const bool gal = in->stype[(size_t)i * N + k] != 0;
      int srow = 1;
      for (int j = 0; j < 6; ++j) {
        if (in->keep[((size_t)i * N + k) * 6 + j] && (j < 2 || gal)) {
          row_k[(size_t)i * Kmax + r] = (int16_t)k;
          row_s[(size_t)i * Kmax + r] = (int16_t)srow++;
          row_p[(size_t)i * Kmax + r] = (int16_t)(6 * k + j);
          ++r;
        }
      }
    }
    for (int k = 0; k < nr[i]; ++k) {
      row_k[(size_t)i * Kmax + r] = (int16_t)k;
      row_s[(size_t)i * Kmax + r] = 0;
      ++r;
    }
    for (int j = 0; j < nbg; ++j) {   // background basis rows: sources -2, -3, -4
      row_k[(size_t)i * Kmax + r] = 0;
      row_s[(size_t)i * Kmax + r] = (int16_t)(-2 - j);
      ++r;
    }
    row_k[(size_t)i * Kmax + r] = 0;
    row_s[(size_t)i * Kmax + r] = -1;
  }
  const int Sz = std::min(T, B);
  ch->n = n; ch->N = N; ch->nb = nb; ch->nP = nP;
  ClassDev& c = ch->c;
  c.n_isl = n; c.nb = nb; c.N = N; c.nP = nP; c.B = B; c.T = T; c.Sz = Sz; c.R = R;
  c.nbg = nbg; c.NL = N + nbg;
  c.dlnp = cls->convergence_dlnp ? 1 : 0;
  c.quantum = 2.0f * cls->plateau_dlnp_tol;
  c.changed = (cls->stall_changed || c.dlnp) ? 1 : 0;
  c.tr = cls->step_tr ? 1 : 0;
  if (c.tr && c.changed)
    return set_err(ctx, UPH_ERR_INVALID,
                   "step_tr excludes stall_changed and convergence_dlnp");
  c.Kmax = Kmax; c.nLmax = nLmax; c.ntile_side = (Sz + UPH_TILE - 1) / UPH_TILE;
  c.mode = mode;
  c.native = (cls->native_stamp > 0 && cls->native_stamp < T) ? (cls->native_stamp | 1) : T;
  c.has_gal = any_gal ? 1 : 0;
  if (cls->precision != UPH_PRECISION_PLAIN && cls->precision != UPH_PRECISION_MIXED)
    return set_err(ctx, UPH_ERR_INVALID, "unknown precision %d", cls->precision);
  c.tc_min_rows = (cls->precision == UPH_PRECISION_MIXED)
                      ? (cls->tc_min_rows < 0 ? UPH_TC_MIN_ROWS_DEFAULT : cls->tc_min_rows)
                      : (1 << 30);
  c.Hp = ctx->Hp; c.Wp = ctx->Wp;
  c.dstack = (const float*)sptr(ctx->dstack);
  c.wstack = (const float*)sptr(ctx->wstack);
  ch->bound = {ctx->dstack, ctx->wstack, ctx->tb_knots, ctx->tb_amps, ctx->tb_lv, ctx->tb_core};
  if (mode == UPH_RENDER_REFERENCE) {
    ch->bound.push_back(pp->coefs);
    ch->bound.push_back(pp->os);
    c.psf_coefs = (const float*)sptr(pp->coefs);
    c.psf_os = (const float*)sptr(pp->os);
    c.nt = pp->nt;
    c.psf_varies = pp->nt > 1;
  } else {
    ch->bound.push_back(ctx->mog);
    ch->bound.push_back(ctx->mog_os);
    c.mog = (const float*)sptr(ctx->mog);
    c.psf_os = (const float*)sptr(ctx->mog_os);
    c.nt = ctx->mog_nt;
    c.kpsf = ctx->mog_k;
    c.psf_varies = ctx->mog_nt > 1;
  }
  c.tb_knots = (const double*)sptr(ctx->tb_knots);
  c.tb_amps = (const double*)sptr(ctx->tb_amps);
  c.tb_lv = (const double*)sptr(ctx->tb_lv);
  c.tb_core = (const double*)sptr(ctx->tb_core);
  c.tb_n = ctx->tb_n; c.tb_k = ctx->tb_k; c.tb_nmin = ctx->tb_nmin; c.tb_nmax = ctx->tb_nmax;
  int rc = UPH_OK;
  int* d_ox = cbuf<int>(ctx, ch, "ox", n, &rc);
  int* d_oy = cbuf<int>(ctx, ch, "oy", n, &rc);
  float* d_x0b = cbuf<float>(ctx, ch, "x0b", n, &rc);
  float* d_y0b = cbuf<float>(ctx, ch, "y0b", n, &rc);
  int* d_st = cbuf<int>(ctx, ch, "stype", (size_t)n * N, &rc);
  float* d_nf = cbuf<float>(ctx, ch, "nfrozen", (size_t)n * N, &rc);
  uint8_t* d_fn = cbuf<uint8_t>(ctx, ch, "freen", (size_t)n * N, &rc);
  uint8_t* d_mm = cbuf<uint8_t>(ctx, ch, "mmask", (size_t)n * N, &rc);
  uint8_t* d_keep = cbuf<uint8_t>(ctx, ch, "keep", (size_t)n * nP, &rc);
  float* d_lo = cbuf<float>(ctx, ch, "lower", (size_t)n * nP, &rc);
  float* d_hi = cbuf<float>(ctx, ch, "upper", (size_t)n * nP, &rc);
  float* d_pm = cbuf<float>(ctx, ch, "pmean", (size_t)n * nP, &rc);
  float* d_pi = cbuf<float>(ctx, ch, "pinv", (size_t)n * nP, &rc);
  int* d_nL = cbuf<int>(ctx, ch, "nL", n, &rc);
  int* d_nr = cbuf<int>(ctx, ch, "nr", n, &rc);
  int16_t* d_rk = cbuf<int16_t>(ctx, ch, "rowk", (size_t)n * Kmax, &rc);
  int16_t* d_rs = cbuf<int16_t>(ctx, ch, "rows", (size_t)n * Kmax, &rc);
  int16_t* d_rp = cbuf<int16_t>(ctx, ch, "rowp", (size_t)n * Kmax, &rc);
  ch->d_p0 = cbuf<float>(ctx, ch, "p0", (size_t)n * nP, &rc);
  ch->d_lam0 = cbuf<float>(ctx, ch, "lam0", n, &rc);
  ch->d_chi20 = cbuf<float>(ctx, ch, "chi20", n, &rc);
  ch->d_consec0 = cbuf<int>(ctx, ch, "consec0", n, &rc);
  ch->d_nrej0 = cbuf<int>(ctx, ch, "nrej0", n, &rc);
  ch->d_nst0 = cbuf<int>(ctx, ch, "nst0", n, &rc);
  ch->d_flags0 = cbuf<uint8_t>(ctx, ch, "flags0", n, &rc);
  c.p = cbuf<float>(ctx, ch, "p", (size_t)n * nP, &rc);
  c.p_try = cbuf<float>(ctx, ch, "ptry", (size_t)n * nP, &rc);
  c.lam = cbuf<float>(ctx, ch, "lam", n, &rc);
  c.chi2 = cbuf<float>(ctx, ch, "chi2", n, &rc);
  c.consec = cbuf<int>(ctx, ch, "consec", n, &rc);
  c.nrej = cbuf<int>(ctx, ch, "nrej", n, &rc);
  c.nst = cbuf<int>(ctx, ch, "nst", n, &rc);
  c.flags = cbuf<uint8_t>(ctx, ch, "flags", n, &rc);
  c.stamps = cbuf<float>(ctx, ch, "stamps", (size_t)n * nb * N * R * Sz * Sz, &rc);
  c.mrec = cbuf<MemberRecord>(ctx, ch, "mrec", (size_t)n * nb * N, &rc);
  c.gram = cbuf<float>(ctx, ch, "gram", (size_t)n * nb * Kmax * Kmax, &rc);
  c.Hb = cbuf<float>(ctx, ch, "Hb", (size_t)n * nb * nLmax * nLmax, &rc);
  c.gb = cbuf<float>(ctx, ch, "gb", (size_t)n * nb * nLmax, &rc);
  c.H = cbuf<float>(ctx, ch, "H", (size_t)n * nLmax * nLmax, &rc);
  c.g = cbuf<float>(ctx, ch, "g", (size_t)n * nLmax, &rc);
  c.lu = cbuf<double>(ctx, ch, "lu", nLmax > UPH_LU_SMEM_N ? (size_t)n * nLmax * (nLmax + 1) : 1, &rc);
  c.chi2b = cbuf<double>(ctx, ch, "chi2b", (size_t)n * nb, &rc);
  c.flux = cbuf<float>(ctx, ch, "flux", (size_t)n * nb * N, &rc);
  c.ferr = cbuf<float>(ctx, ch, "ferr", (size_t)n * nb * N, &rc);
  if (nbg) {
    c.bgout = cbuf<float>(ctx, ch, "bgout", (size_t)n * nb * UPH_MAXBG, &rc);
    c.bgerr = cbuf<float>(ctx, ch, "bgerr", (size_t)n * nb * UPH_MAXBG, &rc);
  }
  c.ngood = cbuf<int>(ctx, ch, "ngood", (size_t)n * nb, &rc);
  c.probe_best = cbuf<float>(ctx, ch, "pbest", n, &rc);
  c.probe_p = cbuf<float>(ctx, ch, "probep", (size_t)n * 4 * nP, &rc);
  c.n_active = cbuf<int>(ctx, ch, "nact", 2, &rc);
  c.err = cbuf<int>(ctx, ch, "err", 1, &rc);
  c.gl_split = gram_lin_splits(B, Kmax);
  if (c.gl_split > 1)
    c.glpart = cbuf<float>(ctx, ch, "glpart", (size_t)c.gl_split * n * nb * Kmax * Kmax, &rc);
  c.tc_split = 1;
  if (c.tc_min_rows < (1 << 30)) {
    c.fcur = cbuf<float>(ctx, ch, "fcur", (size_t)n * nb * c.NL, &rc);
    c.ftry = cbuf<float>(ctx, ch, "ftry", (size_t)n * nb * c.NL, &rc);
    c.acond_cur = cbuf<float>(ctx, ch, "acondc", (size_t)n * nb, &rc);
    c.acond_try = cbuf<float>(ctx, ch, "acondt", (size_t)n * nb, &rc);
    c.tc_cond_max = cls->tc_cond_max < 0.f ? UPH_TC_COND_MAX_DEFAULT : cls->tc_cond_max;
    c.tc_split = gram_tc_splits(n, nb, B, ctx->sm_count);
    if (c.tc_split > 1)
      c.gpart = cbuf<float>(ctx, ch, "gpart", (size_t)c.tc_split * n * nb * Kmax * Kmax, &rc);
  }
  ch->d_div = cbuf<uint8_t>(ctx, ch, "div", n, &rc);
  if (c.dlnp) c.chi2d = cbuf<double>(ctx, ch, "chi2d", n, &rc);
  if (c.tr) {
    c.trs = cbuf<double>(ctx, ch, "trs", (size_t)n * 4, &rc);
    ch->d_rail = cbuf<uint8_t>(ctx, ch, "railed", n, &rc);
  }
  if (cls->param_errors || cls->flux_marg) {
    c.perr = cbuf<float>(ctx, ch, "perr", (size_t)n * N * 13, &rc);
    c.ews = cbuf<double>(ctx, ch, "ews", (size_t)n * nLmax * 2 * nLmax, &rc);
  }
  if (cls->param_errors || cls->flux_marg || cls->re_profile)
    c.flsave = cbuf<uint8_t>(ctx, ch, "flsave", n, &rc);
  if (any_gal && mode == UPH_RENDER_REFERENCE) {
    // galaxy stamps by the Fourier-domain convolution with the pixel PSF,
    // or by the direct backend's float64 convolution
    c.fft_P = fft_pad_for(T);
    c.gfft_floats = direct ? gal_direct_floats(T) : gal_fft_floats(T, c.fft_P);
    c.gfft_smem = direct ? gal_direct_smem(T) : gal_fft_smem(T, c.fft_P);
    c.gdirect = direct ? 1 : 0;
    if (direct) {
      c.exp_k = ctx->exp_k;
      c.exp_amp = (const float*)sptr(ctx->exp_amp);
      c.exp_var = (const float*)sptr(ctx->exp_var);
      ch->bound.push_back(ctx->exp_amp);
      ch->bound.push_back(ctx->exp_var);
    }
    // concurrent chunks each hold a work space: half an SM's worth of CTAs
    // per chunk keeps the device busy without multiplying the memory
    c.gfft_ctas = (int)std::min<long long>((long long)n * nb * N,
                                           std::max(16, ctx->sm_count / 2));
    c.gstamp = cbuf<float>(ctx, ch, "gstamp", (size_t)n * nb * N * 7 * T * T, &rc);
    c.gfft_ws = cbuf<float>(ctx, ch, "gfftws", (size_t)c.gfft_ctas * c.gfft_floats, &rc);
  }
  if (cls->scene_subtract) {
    if (!in->member_s1_flux)
      return set_err(ctx, UPH_ERR_INVALID, "scene_subtract needs member_s1_flux");
    ch->scene = true;
    ch->d_seed = cbuf<float>(ctx, ch, "seed", (size_t)n * nP, &rc);
    ch->d_msf = cbuf<float>(ctx, ch, "msf", (size_t)n * N * nb, &rc);
  }
  if (cls->re_profile) c.reprof = cbuf<float>(ctx, ch, "reprof", (size_t)n * N * UPH_REPROF_K, &rc);
  if (cls->residual) {
    c.resid = cbuf<float>(ctx, ch, "resid", (size_t)n * B * B, &rc);
    c.resid_w = cbuf<float>(ctx, ch, "residw", (size_t)n * B * B, &rc);
  }
  if (cls->flux_marg) {
    ch->d_cjac = cbuf<float>(ctx, ch, "cjac", (size_t)n * nb * nLmax * UPH_MAXLIN, &rc);
    c.femarg = cbuf<float>(ctx, ch, "femarg", (size_t)n * nb * N, &rc);
  }
  ch->perr_out = cls->param_errors != 0;
  if (cls->source_metrics) {
    c.smom = cbuf<double>(ctx, ch, "smom", (size_t)n * nb * N * 5, &rc);
    c.smet = cbuf<float>(ctx, ch, "smet", (size_t)n * N * 4, &rc);
    c.swin = cbuf<float>(ctx, ch, "swin", (size_t)n * nb * N, &rc);
  }
  if (c.changed) {
    c.n_same = cbuf<int>(ctx, ch, "nsame", n, &rc);
    c.prej = cbuf<float>(ctx, ch, "prej", (size_t)n * nP, &rc);
    c.div_live = cbuf<uint8_t>(ctx, ch, "divl", n, &rc);
    ch->d_nsame0 = cbuf<int>(ctx, ch, "nsame0", n, &rc);
    ch->d_prej0 = cbuf<float>(ctx, ch, "prej0", (size_t)n * nP, &rc);
    ch->d_divl0 = cbuf<uint8_t>(ctx, ch, "divl0", n, &rc);
  }
  float* d_dwin = nullptr;
  float* d_wwin = nullptr;
  int* d_ox2 = nullptr;
  int* d_oy2 = nullptr;
  if (ch->scene) {
    d_dwin = cbuf<float>(ctx, ch, "dwin", (size_t)nb * n * B * B, &rc);
    d_wwin = cbuf<float>(ctx, ch, "wwin", (size_t)nb * n * B * B, &rc);
    d_ox2 = cbuf<int>(ctx, ch, "ox2", n, &rc);
    d_oy2 = cbuf<int>(ctx, ch, "oy2", n, &rc);
  }
  if (rc) return rc;
  c.ox = d_ox; c.oy = d_oy; c.x0b = d_x0b; c.y0b = d_y0b; c.stype = d_st;
  c.n_frozen = d_nf; c.free_n = d_fn; c.mmask = d_mm; c.keep = d_keep;
  c.lower = d_lo; c.upper = d_hi; c.prior_mean = d_pm; c.prior_inv = d_pi;
  c.has_priors = cls->has_priors ? 1 : 0;
  c.isl_nL = d_nL; c.isl_nr = d_nr; c.row_k = d_rk; c.row_s = d_rs; c.row_p = d_rp;
  c.reg = cls->reg; c.pos_step_max = cls->pos_step_max; c.ftol_rel = cls->chi2_ftol_rel;
  c.step_tol = cls->step_tol_pix; c.un_freeze = cls->un_freeze_steps;
  // the trust radius starts unset (0): the first step seeds it
  std::vector<float> h_lam(n, c.tr ? 0.f : 1e-3f), h_chi2(n, 0.f);
  std::vector<int> h_consec(n, 0), h_nrej(n, 0);
  ch->h_nst0.assign(n, 0);
  ch->h_flags0.assign(n, FL_NEEDLIN | FL_REAL);
  ch->fresh = (in->init_lam == nullptr);
  if (!ch->fresh) {
    if (!in->init_chi2 || !in->init_consec || !in->init_nrej || !in->init_nst)
      return set_err(ctx, UPH_ERR_INVALID, "partial init state");
    for (int i = 0; i < n; ++i) {
      h_lam[i] = in->init_lam[i];
      h_chi2[i] = in->init_chi2[i];
      h_consec[i] = in->init_consec[i];
      h_nrej[i] = in->init_nrej[i];
      ch->h_nst0[i] = in->init_nst[i];
    }
  }
  if ((rc = upload(ctx, d_ox, in->ox, sizeof(int) * n, "ox"))) return rc;
  if ((rc = upload(ctx, d_oy, in->oy, sizeof(int) * n, "oy"))) return rc;
  if (ch->scene) {
    // the solve reads the private windows: island isl at rows isl*B of a
    // B-wide stack per band
    std::vector<int> zx(n, 0), wy(n);
    for (int i = 0; i < n; ++i) wy[i] = i * B;
    if ((rc = upload(ctx, d_ox2, zx.data(), sizeof(int) * n, "ox"))) return rc;
    if ((rc = upload(ctx, d_oy2, wy.data(), sizeof(int) * n, "oy"))) return rc;
    if ((rc = upload(ctx, ch->d_msf, in->member_s1_flux, sizeof(float) * n * N * nb, "msf")))
      return rc;
    if ((rc = upload(ctx, ch->d_seed, in->seed_p ? in->seed_p : in->p0,
                     sizeof(float) * n * nP, "seed")))
      return rc;
    ch->fd = c.dstack; ch->fw = c.wstack; ch->fHp = c.Hp; ch->fWp = c.Wp;
    ch->ox_f = d_ox; ch->oy_f = d_oy;
    c.dstack = d_dwin; c.wstack = d_wwin; c.Hp = n * B; c.Wp = B;
    c.ox = d_ox2; c.oy = d_oy2;
  }
  if ((rc = upload(ctx, d_x0b, in->x0b, sizeof(float) * n, "x0b"))) return rc;
  if ((rc = upload(ctx, d_y0b, in->y0b, sizeof(float) * n, "y0b"))) return rc;
  if ((rc = upload(ctx, d_st, in->stype, sizeof(int) * n * N, "stype"))) return rc;
  if ((rc = upload(ctx, d_nf, in->n_frozen, sizeof(float) * n * N, "n_frozen"))) return rc;
  if ((rc = upload(ctx, d_fn, in->free_n, (size_t)n * N, "free_n"))) return rc;
  if ((rc = upload(ctx, d_mm, in->mmask, (size_t)n * N, "mmask"))) return rc;
  if ((rc = upload(ctx, d_keep, in->keep, (size_t)n * nP, "keep"))) return rc;
  if ((rc = upload(ctx, d_lo, in->lower, sizeof(float) * n * nP, "lower"))) return rc;
  if ((rc = upload(ctx, d_hi, in->upper, sizeof(float) * n * nP, "upper"))) return rc;
  if ((rc = upload(ctx, d_pm, in->prior_mean, sizeof(float) * n * nP, "prior_mean"))) return rc;
  if ((rc = upload(ctx, d_pi, in->prior_inv_sigma, sizeof(float) * n * nP, "prior_inv"))) return rc;
  if ((rc = upload(ctx, ch->d_p0, in->p0, sizeof(float) * n * nP, "p0"))) return rc;
  if ((rc = upload(ctx, d_nL, nL.data(), sizeof(int) * n, "nL"))) return rc;
  if ((rc = upload(ctx, d_nr, nr.data(), sizeof(int) * n, "nr"))) return rc;
  if ((rc = upload(ctx, d_rk, row_k.data(), sizeof(int16_t) * n * Kmax, "rows"))) return rc;
  if ((rc = upload(ctx, d_rs, row_s.data(), sizeof(int16_t) * n * Kmax, "rows"))) return rc;
  if ((rc = upload(ctx, d_rp, row_p.data(), sizeof(int16_t) * n * Kmax, "rows"))) return rc;
  if ((rc = upload(ctx, ch->d_lam0, h_lam.data(), sizeof(float) * n, "lam"))) return rc;
  if ((rc = upload(ctx, ch->d_chi20, h_chi2.data(), sizeof(float) * n, "chi2"))) return rc;
  if ((rc = upload(ctx, ch->d_consec0, h_consec.data(), sizeof(int) * n, "consec"))) return rc;
  if ((rc = upload(ctx, ch->d_nrej0, h_nrej.data(), sizeof(int) * n, "nrej"))) return rc;
  if ((rc = upload(ctx, ch->d_nst0, ch->h_nst0.data(), sizeof(int) * n, "nst"))) return rc;
  if ((rc = upload(ctx, ch->d_flags0, ch->h_flags0.data(), n, "flags"))) return rc;
  if (c.changed) {
    // tracker carry (a re-queued chunk) or zeros
    if (in->init_n_same) {
      if ((rc = upload(ctx, ch->d_nsame0, in->init_n_same, sizeof(int) * n, "n_same"))) return rc;
    } else {
      CK(cudaMemsetAsync(ch->d_nsame0, 0, sizeof(int) * n, ctx->stream), "n_same");
    }
    if (in->init_prej) {
      if ((rc = upload(ctx, ch->d_prej0, in->init_prej, sizeof(float) * n * nP, "prej"))) return rc;
    } else {
      CK(cudaMemsetAsync(ch->d_prej0, 0, sizeof(float) * n * nP, ctx->stream), "prej");
    }
    if (in->init_diverged) {
      if ((rc = upload(ctx, ch->d_divl0, in->init_diverged, n, "diverged"))) return rc;
    } else {
      CK(cudaMemsetAsync(ch->d_divl0, 0, n, ctx->stream), "diverged");
    }
  }
  CK(cudaMemsetAsync(c.stamps, 0, sizeof(float) * (size_t)n * nb * N * R * Sz * Sz,
                     ctx->stream), "memset");
  CK(cudaEventCreateWithFlags(&ch->ev_group, cudaEventDisableTiming), "event");
  CK(cudaEventCreate(&ch->ev_done), "event");
  return UPH_OK;
}

// Reset a chunk's LM state from its uploaded inputs (stream s).
int reset_chunk(uph_ctx* ctx, Chunk* ch, cudaStream_t s) {
  const ClassDev& c = ch->c;
  const int n = ch->n;
  CK(cudaMemcpyAsync(c.p, ch->d_p0, sizeof(float) * n * ch->nP, cudaMemcpyDeviceToDevice, s), "reset");
  CK(cudaMemcpyAsync(c.lam, ch->d_lam0, sizeof(float) * n, cudaMemcpyDeviceToDevice, s), "reset");
  CK(cudaMemcpyAsync(c.chi2, ch->d_chi20, sizeof(float) * n, cudaMemcpyDeviceToDevice, s), "reset");
  CK(cudaMemcpyAsync(c.consec, ch->d_consec0, sizeof(int) * n, cudaMemcpyDeviceToDevice, s), "reset");
  CK(cudaMemcpyAsync(c.nrej, ch->d_nrej0, sizeof(int) * n, cudaMemcpyDeviceToDevice, s), "reset");
  CK(cudaMemcpyAsync(c.nst, ch->d_nst0, sizeof(int) * n, cudaMemcpyDeviceToDevice, s), "reset");
  CK(cudaMemcpyAsync(c.flags, ch->d_flags0, n, cudaMemcpyDeviceToDevice, s), "reset");
  if (c.changed) {
    CK(cudaMemcpyAsync(c.n_same, ch->d_nsame0, sizeof(int) * n, cudaMemcpyDeviceToDevice, s),
       "reset");
    CK(cudaMemcpyAsync(c.prej, ch->d_prej0, sizeof(float) * n * ch->nP,
                       cudaMemcpyDeviceToDevice, s), "reset");
    CK(cudaMemcpyAsync(c.div_live, ch->d_divl0, n, cudaMemcpyDeviceToDevice, s), "reset");
  }
  CK(cudaMemsetAsync(c.err, 0, sizeof(int), s), "reset");
  ch->done = false;
  ch->iters = 0;
  return UPH_OK;
}

// probes: whether the chunk may hold stalled islands (the diverged and
// plateau probes act on stalled islands only, and the outputs of the others
// do not read them: with none, their launches are skipped)
void post_loop(Chunk* ch, Launcher& L, bool probes = true) {
  const ClassDev& c = ch->c;
  cudaStream_t s = L.s;
  launch_set_probe(c, s);
  if (c.changed) {
    // "changed" mode reports the loop's own diverged flag; no post-hoc probe
    cudaMemcpyAsync(ch->d_div, c.div_live, c.n_isl, cudaMemcpyDeviceToDevice, s);
    L.job->ctx->launches += 1;
  } else if (probes) {
    for (int j = 0; j < 4; ++j) L(3, [&] { launch_step(c, PH_PROBE, j, 0.f, 1, s); });
    launch_diverged_compare(c, ch->d_div, s);
    L.job->ctx->launches += 2;
  }
  if (c.tr) {
    launch_railed(c, ch->d_rail, s);
    L.job->ctx->launches += 1;
  }
  if (c.perr) {
    // covariance at the final parameters: one more linearisation of every
    // island, then the float64 inversion
    // (the assembly also keeps the flux sensitivities when the
    // marginalised flux variance is wanted)
    ClassDev ce = c;
    ce.cjac = ch->d_cjac;
    launch_errors_begin(c, s);
    L(0, [&] { launch_render(c, c.p, PH_LIN, s); }, 2);
    L(1, [&] { launch_gram_lin(c, s); }, c.gl_split > 1 ? 2 : 1);
    if (c.tc_min_rows < (1 << 30))
      L(WK_GRAM_TC, [&] { launch_gram_tc(c, s); }, c.tc_split > 1 ? 2 : 1);
    L(2, [&] { launch_assemble(ce, s); });
    L(3, [&] { launch_final_errors(c, s); });
    if (c.femarg) L(3, [&] { launch_flux_marg(ce, s); });
    launch_errors_end(c, s);
    L.job->ctx->launches += 2;
  }
  if (probes) {
    launch_fill_float(c.probe_best, INFINITY, c.n_isl, s);
    L.job->ctx->launches += 1;
    for (int e = -9; e <= 6; ++e) {
      const float lamj = (float)std::pow(10.0, (double)e);
      L(3, [&] { launch_step(c, PH_PROBE, 0, lamj, 2, s); });
      L(0, [&] { launch_render(c, c.p_try, PH_PROBE, s); }, 2);
      L(4, [&] { launch_gram_trial(c, c.p_try, PH_PROBE, 0, nullptr, nullptr, s); });
      L(5, [&] { launch_accept(c, PH_PROBE, s); });
    }
  }
  if (c.reprof) {
    // Re profile: one trial pass per (member slot, offset) on the islands
    // whose slot holds an extended member; flags saved around it
    static const float kDeltas[UPH_REPROF_K] = UPH_REPROF_DELTAS;
    launch_errors_begin(c, s);
    for (int n = 0; n < c.N; ++n)
      for (int j = 0; j < UPH_REPROF_K; ++j) {
        L(3, [&] { launch_reprof_set(c, n, j, kDeltas[j], s); });
        L(0, [&] { launch_render(c, c.p_try, PH_PROBE, s); }, 2);
        L(4, [&] { launch_gram_trial(c, c.p_try, PH_PROBE, 0, nullptr, nullptr, s); });
        L(5, [&] { launch_reprof_store(c, n, j, s); });
      }
    launch_errors_end(c, s);
    L.job->ctx->launches += 2;
  }
  L(0, [&] { launch_render(c, c.p, PH_ALL, s); }, 2);
  L(4, [&] { launch_gram_trial(c, c.p, PH_ALL, 1, nullptr, nullptr, s); });
  // source metrics and the residual read the final pass's model rows and
  // fluxes
  if (c.smet) L(4, [&] { launch_source_metrics(c, s); }, 2);
  if (c.resid) L(4, [&] { launch_residual_coadd(c, s); });
}

using LaunchRecords = std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>>;

// End of a solve (everything joined on the library stream): wait for it,
// turn device error flags into status codes, record the timings and, for an
// instrumented solve, the per-kind times and work counters.
int job_finish(uph_job* job, LaunchRecords& rec) {
  uph_ctx* ctx = job->ctx;
  const int nch = (int)job->chunks.size();
  CK(cudaEventRecord(ctx->ev[2], ctx->stream), "event");
  CK(cudaStreamSynchronize(ctx->stream), "solve");
  for (int i = 0; i < nch; ++i) {
    int e = 0;
    CK(cudaMemcpy(&e, job->chunks[i]->c.err, sizeof(int), cudaMemcpyDeviceToHost), "err");
    if (e == 1)
      return set_err(ctx, UPH_ERR_TIMEOUT,
                     "a bounded device wait expired in chunk %d (tensor-core Gram)", i);
    if (e)
      return set_err(ctx, UPH_ERR_CUDA,
                     "chunk %d: a kernel was launched with less shared memory than its "
                     "tiles need (device check %d)", i, e);
  }
  cudaEventElapsedTime(&ctx->timing[1], ctx->ev[0], ctx->ev[2]);
  for (auto* ch : job->chunks) cudaEventElapsedTime(&ch->done_ms, ctx->ev[0], ch->ev_done);
  ctx->timing[2] = 0.f;
  for (auto* ch : job->chunks) ch->c.work = nullptr;
  if (job->profile) {
    unsigned long long w[WK_FIELDS * WK_KINDS];
    CK(cudaMemcpy(w, job->d_work, sizeof w, cudaMemcpyDeviceToHost), "work");
    for (int k = 0; k < WK_KINDS; ++k) {
      job->ktime[k] = 0.f;
      job->kcount[k] = 0;
      job->kbytes[k] = (double)w[WK_FIELDS * k];
      job->kflops[k] = (double)w[WK_FIELDS * k + 1];
      job->kexps[k] = (double)w[WK_FIELDS * k + 2];
    }
    for (auto& r : rec) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, r.second.first, r.second.second);
      job->ktime[r.first] += ms;
      job->kcount[r.first] += 1;
      cudaEventDestroy(r.second.first);
      cudaEventDestroy(r.second.second);
    }
  }
  return UPH_OK;
}

int job_solve(uph_job* job, int max_steps) {
  uph_ctx* ctx = job->ctx;
  cudaSetDevice(ctx->device);
  if (max_steps < 0) return set_err(ctx, UPH_ERR_INVALID, "max_steps < 0");
  const int nch = (int)job->chunks.size();
  if (nch == 0) return UPH_OK;
  ctx->launches = 0;
  // instrumented solves run on one stream so that per-launch event times
  // are not inflated by other streams' kernels
  const int nstreams = job->profile ? 1 : std::min(nch, UPH_MAX_STREAMS);
  if ((int)job->streams.size() < nstreams) {
    int prio_lo = 0, prio_hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi), "stream priorities");
    while ((int)job->streams.size() < nstreams) {
      // the first streams take the heaviest chunks (the critical path) and
      // get the highest priority
      const int prio = (int)job->streams.size() < UPH_HIGH_PRIORITY_STREAMS ? prio_hi : prio_lo;
      cudaStream_t st;
      CK(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio), "stream");
      job->streams.push_back(st);
    }
  }
  // heaviest chunks first, each onto the least-loaded stream (longest
  // processing time first); cost ~ one iteration's Gram and render work
  std::vector<int> order(nch);
  std::vector<double> cost(nch);
  for (int i = 0; i < nch; ++i) {
    const ClassDev& c = job->chunks[i]->c;
    order[i] = i;
    cost[i] = (double)c.n_isl * c.nb *
              ((double)c.B * c.B * c.Kmax + (double)c.N * c.T * c.T * c.R);
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  {
    std::vector<double> load(nstreams, 0.0);
    for (int i : order) {
      const int j = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      job->chunks[i]->slot = j;
      load[j] += cost[i];
    }
  }
  if (job->h_active_cap < 2 * nch) {
    if (job->h_active) cudaFreeHost(job->h_active);
    CK(cudaMallocHost((void**)&job->h_active, sizeof(int) * 2 * nch), "pinned");
    job->h_active_cap = 2 * nch;
  }
  std::vector<char> counted(nch, 0);
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> rec;
  auto* recp = job->profile ? &rec : nullptr;
  if (job->profile) {
    if (!job->d_work)
      CK(cudaMalloc((void**)&job->d_work, sizeof(unsigned long long) * WK_FIELDS * WK_KINDS),
         "work");
    CK(cudaMemsetAsync(job->d_work, 0, sizeof(unsigned long long) * WK_FIELDS * WK_KINDS,
                       ctx->stream), "work");
  }
  for (auto* ch : job->chunks) ch->c.work = job->profile ? job->d_work : nullptr;
  CK(cudaEventRecord(ctx->ev[0], ctx->stream), "event");
  for (auto st : job->streams) CK(cudaStreamWaitEvent(st, ctx->ev[0], 0), "wait");
  for (int i : order) {
    Chunk* ch = job->chunks[i];
    cudaStream_t s = job->streams[ch->slot];
    int rc = reset_chunk(ctx, ch, s);
    if (rc) return rc;
    Launcher L{job, s, recp};
    if (ch->scene) {
      // scene subtract: fresh private windows plus the members at their seeds
      launch_copy_windows(ch->c, ch->fd, ch->fw, ch->fHp, ch->fWp, ch->ox_f, ch->oy_f, s);
      L(0, [&] { launch_render(ch->c, ch->d_seed, PH_ALL, s); }, 2);
      launch_addback(ch->c, ch->d_seed, ch->d_msf, s);
      ctx->launches += 2;
    }
    // initial chi2 (fresh chunks) and, for the tensor-core Gram, the fluxes
    // at the starting parameters that its residual row needs
    // (dlnp: the float64 chi2 carry is recomputed at the starting point)
    if (ch->fresh || ch->c.fcur || ch->c.dlnp) {
      L(0, [&] { launch_render(ch->c, ch->c.p, PH_ALL, s); }, 2);
      L(4, [&] { launch_gram_trial(ch->c, ch->c.p, PH_ALL, 0, ch->c.fcur, ch->c.acond_cur,
                                   s); });
      if (ch->fresh || ch->c.dlnp) L(5, [&] { launch_accept(ch->c, PH_ALL, s); });
    }
    if (max_steps > 0 && !job->profile && !ch->gexec) {
      Launcher Lc{job, s, nullptr};
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "capture");
      const int64_t before = ctx->launches;
      iteration(ch->c, Lc);
      ch->graph_kernels = (int)(ctx->launches - before);
      ctx->launches = before;
      cudaError_t ce = cudaStreamEndCapture(s, &ch->graph);
      if (ce != cudaSuccess) return cuda_err(ctx, ce, "end capture");
      CK(cudaGraphInstantiate(&ch->gexec, ch->graph, 0), "graph instantiate");
    }
    if (max_steps == 0) ch->done = true;
  }
  CK(cudaGetLastError(), "launch");
  // LM loop: every chunk advances in groups of UPH_CHECK_EVERY iterations;
  // as soon as a group's active count reaches the host, that chunk's next
  // group -- or, once it has finished, its post-loop probes and final pass --
  // is enqueued, so no chunk waits for another.
  std::vector<char> inflight(nch, 0);
  auto enqueue_group = [&](int i) -> int {
    Chunk* ch = job->chunks[i];
    cudaStream_t s = job->streams[ch->slot];
    const int group = std::min(UPH_CHECK_EVERY, max_steps - ch->iters);
    for (int j = 0; j < group; ++j) {
      if (job->profile) {
        Launcher L{job, s, recp};
        iteration(ch->c, L);
      } else {
        CK(cudaGraphLaunch(ch->gexec, s), "graph launch");
        ctx->launches += ch->graph_kernels;
      }
    }
    ch->iters += group;
    launch_count_active(ch->c, s);
    ctx->launches += 1;
    CK(cudaMemcpyAsync(job->h_active + 2 * i, ch->c.n_active, 2 * sizeof(int),
                       cudaMemcpyDeviceToHost, s), "count");
    counted[i] = 1;
    CK(cudaEventRecord(ch->ev_group, s), "event");
    inflight[i] = 1;
    return UPH_OK;
  };
  auto finish = [&](int i) {
    Chunk* ch = job->chunks[i];
    ch->done = true;
    Launcher L{job, job->streams[ch->slot], recp};
    post_loop(ch, L, !counted[i] || job->h_active[2 * i + 1] > 0);
    cudaEventRecord(ch->ev_done, job->streams[ch->slot]);
  };
  int live = 0;
  for (int i : order) {
    if (job->chunks[i]->done) {
      finish(i);
      continue;
    }
    int rc = enqueue_group(i);
    if (rc) return rc;
    ++live;
  }
  while (live > 0) {
    bool progress = false;
    for (int i : order) {
      if (!inflight[i]) continue;
      Chunk* ch = job->chunks[i];
      const cudaError_t q = cudaEventQuery(ch->ev_group);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) return cuda_err(ctx, q, "lm loop");
      inflight[i] = 0;
      progress = true;
      if (job->h_active[2 * i] == 0 || ch->iters >= max_steps) {
        finish(i);
        --live;
      } else {
        int rc = enqueue_group(i);
        if (rc) return rc;
      }
    }
    if (!progress) std::this_thread::yield();
  }
  CK(cudaGetLastError(), "post-loop");
  for (auto st : job->streams) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    CK(cudaEventRecord(e, st), "event");
    CK(cudaStreamWaitEvent(ctx->stream, e, 0), "join");
    cudaEventDestroy(e);
  }
  return job_finish(job, rec);
}

// Streams of a job (created once; the first ones get the highest priority)
// and each chunk's slot: heaviest chunks first onto the least-loaded stream
// (longest processing time first); cost ~ one iteration's Gram and render.
int job_streams(uph_job* job, int nstreams, std::vector<int>& order) {
  uph_ctx* ctx = job->ctx;
  const int nch = (int)job->chunks.size();
  if ((int)job->streams.size() < nstreams) {
    int prio_lo = 0, prio_hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi), "stream priorities");
    while ((int)job->streams.size() < nstreams) {
      const int prio = (int)job->streams.size() < UPH_HIGH_PRIORITY_STREAMS ? prio_hi : prio_lo;
      cudaStream_t st;
      CK(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio), "stream");
      job->streams.push_back(st);
    }
  }
  order.resize(nch);
  std::vector<double> cost(nch);
  for (int i = 0; i < nch; ++i) {
    const ClassDev& c = job->chunks[i]->c;
    order[i] = i;
    cost[i] = (double)c.n_isl * c.nb *
              ((double)c.B * c.B * c.Kmax + (double)c.N * c.T * c.T * c.R);
  }
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<double> load(nstreams, 0.0);
  for (int i : order) {
    const int j = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    job->chunks[i]->slot = j;
    load[j] += cost[i];
  }
  return UPH_OK;
}

// Lanes of the queue engine by footprint: a queue kernel launches with the
// largest shared-memory footprint among its lane's chunks, so chunks of like
// size share a lane -- sorted by window side, Gram rows and stamp tier, then
// cut into nl runs of about equal cost, every lane non-empty -- instead of
// the longest-processing-time deal, which puts a heavy chunk in every lane
// and runs every unit at the heavy chunk's occupancy.
void queue_lanes(uph_job* job, int nl) {
  const int nch = (int)job->chunks.size();
  std::vector<int> byfp(nch);
  std::vector<double> cost(nch);
  double total = 0.0;
  for (int i = 0; i < nch; ++i) {
    const ClassDev& c = job->chunks[i]->c;
    byfp[i] = i;
    cost[i] = (double)c.n_isl * c.nb *
              ((double)c.B * c.B * c.Kmax + (double)c.N * c.T * c.T * c.R);
    total += cost[i];
  }
  std::stable_sort(byfp.begin(), byfp.end(), [&](int a, int b) {
    const ClassDev& x = job->chunks[a]->c;
    const ClassDev& y = job->chunks[b]->c;
    if (x.B != y.B) return x.B > y.B;
    if (x.Kmax != y.Kmax) return x.Kmax > y.Kmax;
    return x.T > y.T;
  });
  int lane = 0;
  double acc = 0.0;
  for (int j = 0; j < nch; ++j) {
    // move on when this lane has its share, or when the chunks left are
    // only enough to give every remaining lane one
    if (j > 0 && lane < nl - 1 &&
        (acc >= total * (lane + 1) / nl || nch - j <= nl - 1 - lane))
      ++lane;
    job->chunks[byfp[j]]->slot = lane;
    acc += cost[byfp[j]];
  }
}

// Every stream of the job waits for the work enqueued so far on `from`.
int job_fork(uph_job* job, cudaStream_t from, int nstreams) {
  uph_ctx* ctx = job->ctx;
  cudaEvent_t e;
  CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
  CK(cudaEventRecord(e, from), "event");
  for (int i = 0; i < nstreams; ++i) CK(cudaStreamWaitEvent(job->streams[i], e, 0), "fork");
  cudaEventDestroy(e);
  return UPH_OK;
}

// `to` waits for the work enqueued so far on every stream of the job.
int job_join(uph_job* job, cudaStream_t to, int nstreams) {
  uph_ctx* ctx = job->ctx;
  for (int i = 0; i < nstreams; ++i) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    CK(cudaEventRecord(e, job->streams[i]), "event");
    CK(cudaStreamWaitEvent(to, e, 0), "join");
    cudaEventDestroy(e);
  }
  return UPH_OK;
}

// The LM loop of the whole job on the work queues (UPH_ENGINE_QUEUE).  The
// chunks are dealt to up to UPH_QUEUE_LANES lanes, longest processing time
// first; each lane runs on its own stream, with its own device work lists
// and a CUDA graph of one LM iteration: the device compacts the lane's
// islands still active in the linearisation and trial phases, then one
// persistent kernel per kernel kind works through their units.  Lanes
// overlap on the device the way the per-chunk streams did, with a few
// launches per iteration per lane instead of one graph per chunk.  The
// per-chunk set-up (state reset, scene add-back, initial chi2) and the
// post-loop passes (probes, final fluxes) run per chunk on the lane's
// stream.  Every per-island computation is the per-chunk kernels' own, so
// the results are bitwise those of job_solve.
int job_solve_queue(uph_job* job, int max_steps) {
  uph_ctx* ctx = job->ctx;
  cudaSetDevice(ctx->device);
  if (max_steps < 0) return set_err(ctx, UPH_ERR_INVALID, "max_steps < 0");
  const int nch = (int)job->chunks.size();
  if (nch == 0) return UPH_OK;
  ctx->launches = 0;
  cudaStream_t s = ctx->stream;
  const int nl = job->profile ? 1 : std::min(nch, job->lanes_max > 0 ? job->lanes_max
                                                                      : UPH_QUEUE_LANES);
  std::vector<int> order;
  int rc = job_streams(job, nl, order);
  if (rc) return rc;
  queue_lanes(job, nl);
  if (job->h_active_cap < std::max(nch, nl)) {
    if (job->h_active) cudaFreeHost(job->h_active);
    CK(cudaMallocHost((void**)&job->h_active, sizeof(int) * std::max(nch, nl)), "pinned");
    job->h_active_cap = std::max(nch, nl);
  }
  if (job->h_stall_cap < 2 * nch) {
    if (job->h_stall) cudaFreeHost(job->h_stall);
    CK(cudaMallocHost((void**)&job->h_stall, sizeof(int) * 2 * nch), "pinned");
    job->h_stall_cap = 2 * nch;
  }
  LaunchRecords rec;
  auto* recp = job->profile ? &rec : nullptr;
  if (job->profile) {
    if (!job->d_work)
      CK(cudaMalloc((void**)&job->d_work, sizeof(unsigned long long) * WK_FIELDS * WK_KINDS),
         "work");
    CK(cudaMemsetAsync(job->d_work, 0, sizeof(unsigned long long) * WK_FIELDS * WK_KINDS, s),
       "work");
  }
  for (auto* ch : job->chunks) ch->c.work = job->profile ? job->d_work : nullptr;
  // lanes: the chunks of each stream slot, heaviest first, and their islands'
  // range in the job's order
  if ((int)job->lanes.size() != nl || !job->q_graph_valid) {
    for (auto& ln : job->lanes) ln.release();
    job->lanes.assign(nl, QueueLane{});
    job->q_graph_valid = false;
  }
  int n_total = 0;
  for (auto& ln : job->lanes) ln.chunks.clear();
  for (int i : order) job->lanes[job->chunks[i]->slot].chunks.push_back(i);
  std::vector<int2> hord;
  for (auto& ln : job->lanes) {
    ln.off = n_total;
    for (int i : ln.chunks)
      for (int j = 0; j < job->chunks[i]->c.n_isl; ++j) hord.push_back(make_int2(i, j));
    ln.n = (int)hord.size() - ln.off;
    n_total = (int)hord.size();
  }
  std::vector<ClassDev> hcls(nch);
  for (int i = 0; i < nch; ++i) hcls[i] = job->chunks[i]->c;
  if ((rc = ensure(ctx, job->q_cls, sizeof(ClassDev) * nch, "queue"))) return rc;
  if ((rc = ensure(ctx, job->q_order, sizeof(int2) * n_total, "queue"))) return rc;
  if ((rc = ensure(ctx, job->q_count, sizeof(int) * nl, "queue"))) return rc;
  for (int k = 0; k < 2; ++k) {
    if ((rc = ensure(ctx, job->q_act[k], sizeof(int2) * n_total, "queue"))) return rc;
    if ((rc = ensure(ctx, job->q_n[k], sizeof(int) * nl, "queue"))) return rc;
    if ((rc = ensure(ctx, job->q_pre[k], sizeof(int) * (size_t)QK_KINDS * (n_total + nl),
                     "queue")))
      return rc;
    if ((rc = ensure(ctx, job->q_next[k], sizeof(int) * QK_KINDS * nl, "queue"))) return rc;
  }
  const ClassDev* dcls = (const ClassDev*)job->q_cls.ptr;
  const int2* dord = (const int2*)job->q_order.ptr;
  int* dcount = (int*)job->q_count.ptr;
  const bool bg = job->chunks[0]->c.nbg > 0;
  for (int l = 0; l < nl; ++l) {
    QueueLane& ln = job->lanes[l];
    for (int k = 0; k < 2; ++k) {
      QueueList& q = ln.ql[k];
      q.cls = dcls;
      q.act = (int2*)job->q_act[k].ptr + ln.off;
      q.n_act = (int*)job->q_n[k].ptr + l;
      q.pre = (int*)job->q_pre[k].ptr + (size_t)QK_KINDS * (ln.off + l);
      q.stride = ln.n + 1;
      q.next = (int*)job->q_next[k].ptr + QK_KINDS * l;
      q.per_cta = job->engine == UPH_ENGINE_QUEUE_PER_CTA ? 1 : 0;
      for (int kind = 0; kind < QK_KINDS; ++kind) {
        long long cap = 0;
        for (int i : ln.chunks)
          cap += (long long)job->chunks[i]->c.n_isl * queue_units(job->chunks[i]->c, kind);
        q.cap[kind] = (int)std::min<long long>(cap, 1 << 30);
      }
    }
    // launch shapes: the largest footprint over the lane's chunks
    ln.sm_rlin = ln.sm_rtry = ln.sm_glin = ln.sm_gtc = ln.sm_asm = ln.sm_step = ln.sm_trial = 0;
    ln.any_tc = ln.any_red = ln.any_fft = ln.any_glr = false;
    for (int i : ln.chunks) {
      const ClassDev& c = job->chunks[i]->c;
      ln.sm_rlin = std::max(ln.sm_rlin, render_phase_smem(c, PH_LIN));
      ln.sm_rtry = std::max(ln.sm_rtry, render_phase_smem(c, PH_TRIAL));
      ln.sm_glin = std::max(ln.sm_glin, gram_lin_smem_bytes(c.Kmax));
      ln.any_glr = ln.any_glr || c.gl_split > 1;
      ln.sm_asm = std::max(ln.sm_asm, assemble_smem_bytes(c.nLmax, c.N));
      ln.sm_step = std::max(ln.sm_step, step_smem_bytes(c.nLmax));
      ln.sm_trial = std::max(ln.sm_trial, gram_trial_smem_bytes(c.N));
      if (c.tc_min_rows < (1 << 30)) {
        ln.any_tc = true;
        ln.any_red = ln.any_red || c.tc_split > 1;
        ln.sm_gtc = std::max(ln.sm_gtc,
                             gram_tc_smem_bytes(c.Kmax < UPH_MAXK ? c.Kmax : UPH_MAXK));
      }
      ln.any_fft = ln.any_fft || (c.mode == 0 && c.gstamp);
    }
    ln.iters = 0;
    ln.live = max_steps > 0;
    ln.inflight = false;
  }
  CK(cudaEventRecord(ctx->ev[0], s), "event");
  CK(cudaMemcpyAsync(job->q_cls.ptr, hcls.data(), sizeof(ClassDev) * nch,
                     cudaMemcpyHostToDevice, s), "queue");
  CK(cudaMemcpyAsync(job->q_order.ptr, hord.data(), sizeof(int2) * n_total,
                     cudaMemcpyHostToDevice, s), "queue");
  if ((rc = job_fork(job, s, nl))) return rc;
  // per-chunk set-up on the lanes' streams
  for (int i : order) {
    Chunk* ch = job->chunks[i];
    cudaStream_t cs = job->streams[ch->slot];
    if ((rc = reset_chunk(ctx, ch, cs))) return rc;
    Launcher L{job, cs, recp};
    if (ch->scene) {
      launch_copy_windows(ch->c, ch->fd, ch->fw, ch->fHp, ch->fWp, ch->ox_f, ch->oy_f, cs);
      L(0, [&] { launch_render(ch->c, ch->d_seed, PH_ALL, cs); }, 2);
      launch_addback(ch->c, ch->d_seed, ch->d_msf, cs);
      ctx->launches += 2;
    }
    if (ch->fresh || ch->c.fcur || ch->c.dlnp) {
      L(0, [&] { launch_render(ch->c, ch->c.p, PH_ALL, cs); }, 2);
      L(4, [&] { launch_gram_trial(ch->c, ch->c.p, PH_ALL, 0, ch->c.fcur, ch->c.acond_cur,
                                   cs); });
      if (ch->fresh || ch->c.dlnp) L(5, [&] { launch_accept(ch->c, PH_ALL, cs); });
    }
  }
  CK(cudaGetLastError(), "launch");
  const int sms = ctx->sm_count;
  auto iteration = [&](QueueLane& ln, cudaStream_t ls, Launcher& L) {
    const int2* lord = dord + ln.off;
    launch_q_build(dcls, lord, ln.n, ln.ql[0], PH_LIN, ls);
    launch_q_build(dcls, lord, ln.n, ln.ql[1], PH_TRIAL, ls);
    ctx->launches += 2;
    auto gal_fft = [&](int phase, bool p_try) {
      if (!ln.any_fft) return;
      for (int i : ln.chunks) {
        const ClassDev& c = job->chunks[i]->c;
        if (c.mode == 0 && c.gstamp) {
          launch_gal_fft(c, p_try ? c.p_try : c.p, phase, ls);
          ctx->launches += 1;
        }
      }
    };
    L(0, [&] {
      launch_q_setup(ln.ql[0], PH_LIN, false, sms, ls);
      gal_fft(PH_LIN, false);
      launch_q_render(ln.ql[0], PH_LIN, true, false, ln.sm_rlin, sms, ls);
    }, 2);
    L(1, [&] { launch_q_gram_lin(ln.ql[0], bg, ln.any_glr, ln.sm_glin, sms, ls); },
      ln.any_glr ? 2 : 1);
    if (ln.any_tc)
      L(WK_GRAM_TC, [&] { launch_q_gram_tc(ln.ql[0], ln.sm_gtc, ln.any_red, sms, ls); },
        ln.any_red ? 2 : 1);
    L(2, [&] { launch_q_assemble(ln.ql[0], ln.sm_asm, sms, ls); });
    L(3, [&] { launch_q_step(ln.ql[1], ln.sm_step, sms, ls); });
    L(0, [&] {
      launch_q_setup(ln.ql[1], PH_TRIAL, true, sms, ls);
      gal_fft(PH_TRIAL, true);
      launch_q_render(ln.ql[1], PH_TRIAL, false, true, ln.sm_rtry, sms, ls);
    }, 2);
    L(4, [&] { launch_q_trial(ln.ql[1], bg, ln.sm_trial, sms, ls); });
    L(5, [&] { launch_q_accept(ln.ql[1], sms, ls); });
  };
  if (max_steps > 0 && !job->profile && !job->q_graph_valid) {
    for (int l = 0; l < nl; ++l) {
      QueueLane& ln = job->lanes[l];
      cudaStream_t ls = job->streams[l];
      Launcher Lc{job, ls, nullptr};
      CK(cudaStreamBeginCapture(ls, cudaStreamCaptureModeThreadLocal), "capture");
      const int64_t before = ctx->launches;
      iteration(ln, ls, Lc);
      ln.graph_kernels = (int)(ctx->launches - before);
      ctx->launches = before;
      cudaError_t ce = cudaStreamEndCapture(ls, &ln.graph);
      if (ce != cudaSuccess) return cuda_err(ctx, ce, "end capture");
      CK(cudaGraphInstantiate(&ln.gexec, ln.graph, 0), "graph instantiate");
    }
    job->q_graph_valid = true;
  }
  for (auto& ln : job->lanes)
    if (!ln.ev) CK(cudaEventCreateWithFlags(&ln.ev, cudaEventDisableTiming), "event");
  // LM loop: each lane advances in groups of UPH_CHECK_EVERY iterations; as
  // soon as a group's count of islands still iterating reaches the host, the
  // lane's next group -- or, once it has finished, its chunks' post-loop
  // passes -- is enqueued, so no lane waits for another
  auto enqueue_group = [&](int l) -> int {
    QueueLane& ln = job->lanes[l];
    cudaStream_t ls = job->streams[l];
    const int group = std::min(UPH_CHECK_EVERY, max_steps - ln.iters);
    for (int j = 0; j < group; ++j) {
      if (job->profile) {
        Launcher L{job, ls, recp};
        iteration(ln, ls, L);
      } else {
        CK(cudaGraphLaunch(ln.gexec, ls), "graph launch");
        ctx->launches += ln.graph_kernels;
      }
    }
    ln.iters += group;
    launch_q_count(dcls, dord + ln.off, ln.n, dcount + l, ls);
    ctx->launches += 1;
    CK(cudaMemcpyAsync(job->h_active + l, dcount + l, sizeof(int), cudaMemcpyDeviceToHost, ls),
       "count");
    CK(cudaEventRecord(ln.ev, ls), "event");
    ln.inflight = true;
    return UPH_OK;
  };
  auto finish_lane = [&](int l) -> int {
    QueueLane& ln = job->lanes[l];
    cudaStream_t ls = job->streams[l];
    ln.live = false;
    // which chunks hold stalled islands (the post-loop probes' subjects)
    const bool counted = max_steps > 0;
    if (counted) {
      for (int i : ln.chunks) {
        launch_count_active(job->chunks[i]->c, ls);
        CK(cudaMemcpyAsync(job->h_stall + 2 * i, job->chunks[i]->c.n_active, 2 * sizeof(int),
                           cudaMemcpyDeviceToHost, ls), "count");
      }
      ctx->launches += (int64_t)ln.chunks.size();
      CK(cudaStreamSynchronize(ls), "count");
    }
    for (int i : ln.chunks) {
      Chunk* ch = job->chunks[i];
      ch->iters = ln.iters;
      ch->done = true;
      Launcher L{job, ls, recp};
      post_loop(ch, L, !counted || job->h_stall[2 * i + 1] > 0);
      cudaEventRecord(ch->ev_done, ls);
    }
    return UPH_OK;
  };
  int live = 0;
  for (int l = 0; l < nl; ++l) {
    if (!job->lanes[l].live) {
      if ((rc = finish_lane(l))) return rc;
      continue;
    }
    if ((rc = enqueue_group(l))) return rc;
    ++live;
  }
  while (live > 0) {
    bool progress = false;
    for (int l = 0; l < nl; ++l) {
      QueueLane& ln = job->lanes[l];
      if (!ln.inflight) continue;
      const cudaError_t q = cudaEventQuery(ln.ev);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) return cuda_err(ctx, q, "lm loop");
      ln.inflight = false;
      progress = true;
      if (job->h_active[l] == 0 || ln.iters >= max_steps) {
        if ((rc = finish_lane(l))) return rc;
        --live;
      } else if ((rc = enqueue_group(l))) {
        return rc;
      }
    }
    if (!progress) std::this_thread::yield();
  }
  CK(cudaGetLastError(), "post-loop");
  if ((rc = job_join(job, s, nl))) return rc;
  return job_finish(job, rec);
}

int job_read(uph_job* job, int id, uph_chunk_out* out) {
  uph_ctx* ctx = job->ctx;
  if (id < 0 || id >= (int)job->chunks.size())
    return set_err(ctx, UPH_ERR_INVALID, "bad chunk id %d", id);
  if (!out) return set_err(ctx, UPH_ERR_INVALID, "null output");
  Chunk* ch = job->chunks[id];
  const ClassDev& c = ch->c;
  const int n = ch->n, N = ch->N, nb = ch->nb, nP = ch->nP;
  std::vector<uint8_t> fl(n);
  std::vector<int> ng((size_t)n * nb);
  std::vector<float> pbest(n);
  std::vector<int> nst(n);
  int rc;
  if ((rc = download(ctx, out->p, c.p, sizeof(float) * n * nP, "p"))) return rc;
  if ((rc = download(ctx, out->fluxes, c.flux, sizeof(float) * n * nb * N, "flux"))) return rc;
  if ((rc = download(ctx, out->ferr, c.ferr, sizeof(float) * n * nb * N, "ferr"))) return rc;
  if (c.changed) {
    if ((rc = download(ctx, out->n_same, c.n_same, sizeof(int) * n, "n_same"))) return rc;
    if ((rc = download(ctx, out->prej, c.prej, sizeof(float) * n * ch->nP, "prej"))) return rc;
  } else {
    if (out->n_same) std::memset(out->n_same, 0, sizeof(int) * n);
    if (out->prej) std::memset(out->prej, 0, sizeof(float) * n * ch->nP);
  }
  if (c.nbg) {
    if ((rc = download(ctx, out->bg, c.bgout, sizeof(float) * n * nb * UPH_MAXBG, "bg"))) return rc;
    if ((rc = download(ctx, out->bg_err, c.bgerr, sizeof(float) * n * nb * UPH_MAXBG, "bg")))
      return rc;
  } else {
    if (out->bg) std::memset(out->bg, 0, sizeof(float) * n * nb * UPH_MAXBG);
    if (out->bg_err) std::memset(out->bg_err, 0, sizeof(float) * n * nb * UPH_MAXBG);
  }
  if ((rc = download(ctx, out->chi2, c.chi2, sizeof(float) * n, "chi2"))) return rc;
  if ((rc = download(ctx, nst.data(), c.nst, sizeof(int) * n, "nst"))) return rc;
  if ((rc = download(ctx, out->lam, c.lam, sizeof(float) * n, "lam"))) return rc;
  if ((rc = download(ctx, out->consec, c.consec, sizeof(int) * n, "consec"))) return rc;
  if ((rc = download(ctx, out->nrej, c.nrej, sizeof(int) * n, "nrej"))) return rc;
  if ((rc = download(ctx, out->diverged, ch->d_div, n, "diverged"))) return rc;
  if (out->reprof) {
    if (c.reprof) {
      if ((rc = download(ctx, out->reprof, c.reprof, sizeof(float) * n * N * UPH_REPROF_K,
                         "reprof")))
        return rc;
    } else {
      for (size_t e = 0; e < (size_t)n * N * UPH_REPROF_K; ++e) out->reprof[e] = NAN;
    }
  }
  if (out->acond) {
    if (c.acond_cur) {
      if ((rc = download(ctx, out->acond, c.acond_cur, sizeof(float) * n * nb, "acond")))
        return rc;
    } else {
      for (size_t e = 0; e < (size_t)n * nb; ++e) out->acond[e] = NAN;
    }
  }
  for (int q = 0; q < 2; ++q) {
    float* dst = q ? out->resid_w : out->resid;
    const float* src = q ? c.resid_w : c.resid;
    if (!dst) continue;
    const size_t cnt = (size_t)n * c.B * c.B;
    if (src) {
      if ((rc = download(ctx, dst, src, sizeof(float) * cnt, "residual"))) return rc;
    } else {
      for (size_t e = 0; e < cnt; ++e) dst[e] = NAN;
    }
  }
  if (out->smetrics) {
    if (c.smet) {
      if ((rc = download(ctx, out->smetrics, c.smet, sizeof(float) * n * N * 4, "smetrics")))
        return rc;
    } else {
      for (size_t e = 0; e < (size_t)n * N * 4; ++e) out->smetrics[e] = NAN;
    }
  }
  if (out->swin) {
    if (c.swin) {
      if ((rc = download(ctx, out->swin, c.swin, sizeof(float) * n * nb * N, "swin"))) return rc;
    } else {
      for (size_t e = 0; e < (size_t)n * nb * N; ++e) out->swin[e] = NAN;
    }
  }
  if (out->femarg) {
    if (c.femarg) {
      if ((rc = download(ctx, out->femarg, c.femarg, sizeof(float) * n * nb * N, "femarg")))
        return rc;
    } else {
      for (size_t e = 0; e < (size_t)n * nb * N; ++e) out->femarg[e] = NAN;
    }
  }
  if (out->perr) {
    if (c.perr && ch->perr_out) {
      if ((rc = download(ctx, out->perr, c.perr, sizeof(float) * n * N * 13, "perr"))) return rc;
    } else {
      for (size_t e = 0; e < (size_t)n * N * 13; ++e) out->perr[e] = NAN;
    }
  }
  if (out->railed) {
    if (c.tr) {
      if ((rc = download(ctx, out->railed, ch->d_rail, n, "railed"))) return rc;
    } else {
      std::memset(out->railed, 0, n);
    }
  }
  if ((rc = download(ctx, fl.data(), c.flags, n, "flags"))) return rc;
  if ((rc = download(ctx, ng.data(), c.ngood, sizeof(int) * n * nb, "ngood"))) return rc;
  if ((rc = download(ctx, pbest.data(), c.probe_best, sizeof(float) * n, "probe"))) return rc;
  CK(cudaStreamSynchronize(ctx->stream), "read");
  int steps_run = 0;
  for (int i = 0; i < n; ++i) {
    const bool st = (fl[i] & FL_STALL) != 0;
    // dlnp: a reject-exit whose plateau certificate passes (the best damped
    // step gains less than one quantum) converged on the plateau
    const bool certified = c.dlnp && st && std::isfinite(pbest[i]) && pbest[i] > -c.quantum;
    if (out->nst) out->nst[i] = nst[i];
    if (out->conv) out->conv[i] = (fl[i] & FL_CONV) ? 1 : 0;
    if (out->stall) out->stall[i] = (st && !certified) ? 1 : 0;
    if (out->stall_dchi2) out->stall_dchi2[i] = st ? pbest[i] : NAN;
    // the legacy probe only runs on stalled islands; "changed" mode's flag
    // is the loop's sticky tracker and stands as it is
    if (out->diverged && !st && !c.changed) out->diverged[i] = 0;
    if (out->n_good) {
      int64_t t = 0;
      for (int b = 0; b < nb; ++b) t += ng[(size_t)i * nb + b];
      out->n_good[i] = t;
    }
    steps_run = std::max(steps_run, nst[i] - ch->h_nst0[i]);
  }
  out->steps_run = steps_run;
  return UPH_OK;
}

}  // namespace

extern "C" {

int uph_job_create(uph_ctx* ctx, uph_job** out) {
  if (!ctx || !out) return UPH_ERR_INVALID;
  uph_job* j = new uph_job();
  j->ctx = ctx;
  *out = j;
  return UPH_OK;
}

int uph_job_destroy(uph_job* job) {
  if (!job) return UPH_OK;
  cudaSetDevice(job->ctx->device);
  cudaStreamSynchronize(job->ctx->stream);
  for (auto s : job->streams) cudaStreamSynchronize(s);
  delete job;
  return UPH_OK;
}

int uph_job_add_chunk(uph_job* job, const uph_class_desc* cls,
                      const uph_chunk_in* in, int32_t* chunk_id) {
  if (!job) return UPH_ERR_INVALID;
  uph_ctx* ctx = job->ctx;
  if (!cls || !in) return set_err(ctx, UPH_ERR_INVALID, "null argument");
  cudaSetDevice(ctx->device);
  Chunk* ch = new Chunk();
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, ctx->stream);
  int rc = add_chunk(ctx, ch, cls, in);
  if (rc) {
    cudaStreamSynchronize(ctx->stream);
    delete ch;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc;
  }
  cudaEventRecord(b, ctx->stream);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (job->chunks.empty()) ctx->timing[0] = 0.f;
  ctx->timing[0] += ms;
  job->chunks.push_back(ch);
  job->q_graph_valid = false;   // the queue engine's graph covers the old chunk set
  if (chunk_id) *chunk_id = (int32_t)job->chunks.size() - 1;
  return UPH_OK;
}

int uph_job_solve(uph_job* job, int32_t max_steps) {
  if (!job) return UPH_ERR_INVALID;
  if ((job->engine == UPH_ENGINE_QUEUE || job->engine == UPH_ENGINE_QUEUE_PER_CTA) &&
      !job->chunks.empty()) {
    // the queue kernels are instantiated per background setting: every chunk
    // of the job must share it (else the per-chunk engine runs)
    bool same_bg = true;
    for (auto* ch : job->chunks)
      same_bg = same_bg && ((ch->c.nbg > 0) == (job->chunks[0]->c.nbg > 0));
    if (same_bg) return job_solve_queue(job, max_steps);
  }
  return job_solve(job, max_steps);
}

int uph_job_set_engine(uph_job* job, int32_t engine, int32_t lanes) {
  if (!job) return UPH_ERR_INVALID;
  if (engine != UPH_ENGINE_QUEUE && engine != UPH_ENGINE_CHUNKS &&
      engine != UPH_ENGINE_QUEUE_PER_CTA)
    return set_err(job->ctx, UPH_ERR_INVALID, "unknown engine %d", engine);
  if (lanes < 0 || lanes > UPH_MAX_STREAMS)
    return set_err(job->ctx, UPH_ERR_INVALID, "lanes %d outside 0..%d", lanes, UPH_MAX_STREAMS);
  if (lanes != job->lanes_max || engine != job->engine) job->q_graph_valid = false;
  job->engine = engine;
  job->lanes_max = lanes;
  return UPH_OK;
}

int uph_job_read(uph_job* job, int32_t chunk_id, uph_chunk_out* out) {
  if (!job) return UPH_ERR_INVALID;
  cudaSetDevice(job->ctx->device);
  cudaEvent_t a = job->ctx->ev[3], b = job->ctx->ev[4];
  cudaEventRecord(a, job->ctx->stream);
  int rc = job_read(job, chunk_id, out);
  cudaEventRecord(b, job->ctx->stream);
  cudaEventSynchronize(b);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  job->ctx->timing[3] = (chunk_id == 0 ? 0.f : job->ctx->timing[3]) + ms;
  return rc;
}

int uph_job_set_profile(uph_job* job, int32_t on) {
  if (!job) return UPH_ERR_INVALID;
  job->profile = on != 0;
  return UPH_OK;
}

int uph_job_kernel_time(const uph_job* job, int32_t kind, float* ms,
                        int64_t* launches) {
  if (!job || kind < 0 || kind >= WK_KINDS) return UPH_ERR_INVALID;
  if (ms) *ms = job->ktime[kind];
  if (launches) *launches = job->kcount[kind];
  return UPH_OK;
}

int uph_sparse_band_solve(uph_ctx* ctx, const uph_sparse_band* in, uph_sparse_out* out) {
  if (!ctx || !in || !out) return UPH_ERR_INVALID;
  const int n = in->n_sources, H = in->psf_h, W = in->psf_w, h = in->band_h, w = in->band_w;
  const int kmax = in->k_max;
  if (n < 0 || h <= 0 || w <= 0 || H <= 0 || W <= 0 || kmax < 0 || in->psf_nterms <= 0 ||
      in->psf_nterms > UPH_MAXNT || in->bg_order < 0 || in->bg_order > 2)
    return set_err(ctx, UPH_ERR_INVALID, "invalid sparse band shape");
  if (!in->data || !in->invvar || !in->pix_good || !in->psf_coefs ||
      (n > 0 && (!in->pos_x || !in->pos_y)) ||
      (n > 0 && kmax > 0 && (!in->neighbor_idx || !in->neighbor_mask)))
    return set_err(ctx, UPH_ERR_INVALID, "null sparse band input");
  if (sparse_stamp_smem(H, W) > 200 * 1024)
    return set_err(ctx, UPH_ERR_INVALID, "PSF stamp %dx%d too large", H, W);
  if (!(in->psf_x_scale != 0.f && in->psf_y_scale != 0.f && in->bg_x_scale != 0.0 &&
        in->bg_y_scale != 0.0))
    return set_err(ctx, UPH_ERR_INVALID, "zero normalisation scale");
  for (size_t e = 0; e < (size_t)n * kmax; ++e)
    if (in->neighbor_mask[e] && (in->neighbor_idx[e] < 0 || in->neighbor_idx[e] >= n))
      return set_err(ctx, UPH_ERR_INVALID, "neighbour index out of range");
  bool any_gal = false;
  const bool direct = in->render_direct != 0;
  if (in->source_type) {
    if (!in->logre || !in->ee1 || !in->ee2 || !in->sersic_n)
      return set_err(ctx, UPH_ERR_INVALID, "source types without shapes");
    for (int i = 0; i < n; ++i) {
      if (in->source_type[i] < 0 || in->source_type[i] > (direct ? 1 : 3))
        return set_err(ctx, UPH_ERR_INVALID, "source type %d not rendered by the %s backend",
                       in->source_type[i], direct ? "direct" : "fft");
      any_gal = any_gal || in->source_type[i] != 0;
    }
  }
  if (direct && (in->exp_k < 1 || in->exp_k > 16 || !in->exp_amp || !in->exp_var))
    return set_err(ctx, UPH_ERR_INVALID, "direct backend needs 1..16 mixture components");
  const int fftP = fft_pad_for(std::max(H, W));
  if (any_gal && !direct && !sptr(ctx->tb_knots))
    return set_err(ctx, UPH_ERR_STATE, "no Sersic table uploaded");
  if (any_gal && !direct && fftP > 512)
    return set_err(ctx, UPH_ERR_INVALID, "PSF stamp %dx%d needs a Fourier grid above 512", H, W);
  cudaSetDevice(ctx->device);
  const int M = in->bg_order == 0 ? 1 : (in->bg_order == 1 ? 3 : 6);
  const int nt = n + M;
  const size_t npix = (size_t)h * w;
  const int nparts = (int)std::max<size_t>(1, std::min<size_t>(2 * (size_t)ctx->sm_count,
                                                            (npix + 255) / 256));
  const size_t nq = (size_t)M * M + M;
  const size_t sizes[] = {
      sizeof(float) * npix, sizeof(float) * npix, npix, sizeof(float) * npix,
      sizeof(float) * (size_t)std::max(n, 1), sizeof(float) * (size_t)std::max(n, 1),
      sizeof(float) * (size_t)H * W * in->psf_nterms, sizeof(float) * 4, sizeof(double) * 4,
      sizeof(int) * std::max<size_t>((size_t)n * kmax, 1), std::max<size_t>((size_t)n * kmax, 1),
      sizeof(float) * std::max<size_t>((size_t)n * H * W, 1),
      sizeof(int) * (size_t)std::max(n, 1), sizeof(int) * (size_t)std::max(n, 1),
      sizeof(float) * (size_t)std::max(n, 1), sizeof(float) * (size_t)std::max(n, 1),
      sizeof(float) * std::max<size_t>((size_t)n * M, 1),
      sizeof(float) * std::max<size_t>((size_t)n * kmax, 1), sizeof(double) * nparts * nq,
      sizeof(float) * (size_t)nt * nt, sizeof(double) * (size_t)nt * (2 * (size_t)nt + 1),
      sizeof(int), sizeof(float) * nt, sizeof(float) * nt,
      // extended sources
      sizeof(int) * (size_t)std::max(n, 1), sizeof(float) * (size_t)std::max(n, 1),
      sizeof(float) * (size_t)std::max(n, 1), sizeof(float) * (size_t)std::max(n, 1),
      sizeof(float) * (size_t)std::max(n, 1),
      any_gal ? sizeof(float) * (size_t)n * H * W : 16,
      any_gal && !direct ? sizeof(float) * std::min<size_t>((size_t)n, 2 * (size_t)ctx->sm_count) *
                               sparse_gal_floats(H, W, fftP)
                         : 16,
      direct ? sizeof(float) * 2 * (size_t)in->exp_k : 16};
  for (int i = 0; i < 32; ++i) {
    int rc = ensure(ctx, ctx->sp[i], sizes[i], "sparse solve");
    if (rc) return rc;
  }
  SparseDev d{};
  d.n = n; d.H = H; d.W = W; d.nterms = in->psf_nterms; d.M = M; d.h = h; d.w = w;
  d.gx0 = in->grid_x0; d.gy0 = in->grid_y0; d.renorm = in->renorm ? 1 : 0; d.kmax = kmax;
  d.nparts = nparts; d.reg = in->reg;
  float* data = (float*)ctx->sp[0].ptr;
  float* invvar = (float*)ctx->sp[1].ptr;
  uint8_t* good = (uint8_t*)ctx->sp[2].ptr;
  d.wgrid = (float*)ctx->sp[3].ptr;
  float* px = (float*)ctx->sp[4].ptr;
  float* py = (float*)ctx->sp[5].ptr;
  float* coefs = (float*)ctx->sp[6].ptr;
  float* os = (float*)ctx->sp[7].ptr;
  double* bn = (double*)ctx->sp[8].ptr;
  int* nidx = (int*)ctx->sp[9].ptr;
  uint8_t* nmask = (uint8_t*)ctx->sp[10].ptr;
  d.data = data; d.invvar = invvar; d.good = good; d.px = px; d.py = py; d.coefs = coefs;
  d.os = os; d.bn = bn; d.nidx = nidx; d.nmask = nmask;
  d.stamps = (float*)ctx->sp[11].ptr;
  d.ixt = (int*)ctx->sp[12].ptr;
  d.iyt = (int*)ctx->sp[13].ptr;
  d.diag = (float*)ctx->sp[14].ptr;
  d.twd = (float*)ctx->sp[15].ptr;
  d.twb = (float*)ctx->sp[16].ptr;
  d.off = (float*)ctx->sp[17].ptr;
  d.part = (double*)ctx->sp[18].ptr;
  d.Af = (float*)ctx->sp[19].ptr;
  d.G = (double*)ctx->sp[20].ptr;
  d.prow = (int*)ctx->sp[21].ptr;
  d.x = (float*)ctx->sp[22].ptr;
  d.var = (float*)ctx->sp[23].ptr;
  if (any_gal) {
    d.stype = (const int*)ctx->sp[24].ptr;
    d.lr = (const float*)ctx->sp[25].ptr;
    d.e1 = (const float*)ctx->sp[26].ptr;
    d.e2 = (const float*)ctx->sp[27].ptr;
    d.sn = (const float*)ctx->sp[28].ptr;
    d.gal = (float*)ctx->sp[29].ptr;
    d.gws = (float*)ctx->sp[30].ptr;
    d.fft_P = fftP;
    d.gal_floats = sparse_gal_floats(H, W, fftP);
    d.gal_ctas = direct ? 0 : (int)std::min<long long>(n, 2LL * ctx->sm_count);
    d.direct = direct ? 1 : 0;
    d.exp_k = direct ? in->exp_k : 0;
    d.exp_mog = (const float*)ctx->sp[31].ptr;
    d.tb_knots = (const double*)sptr(ctx->tb_knots);
    d.tb_amps = (const double*)sptr(ctx->tb_amps);
    d.tb_lv = (const double*)sptr(ctx->tb_lv);
    d.tb_core = (const double*)sptr(ctx->tb_core);
    d.tb_n = ctx->tb_n;
    d.tb_k = ctx->tb_k;
    d.tb_nmin = ctx->tb_nmin;
    d.tb_nmax = ctx->tb_nmax;
    d.renorm = 0;   // the reference's mixed renderer does not renormalise
  }
  const float osh[4] = {in->psf_x_origin, in->psf_x_scale, in->psf_y_origin, in->psf_y_scale};
  const double bnh[4] = {in->bg_x_origin, in->bg_x_scale, in->bg_y_origin, in->bg_y_scale};
  int rc;
  if ((rc = upload(ctx, data, in->data, sizeof(float) * npix, "data"))) return rc;
  if ((rc = upload(ctx, invvar, in->invvar, sizeof(float) * npix, "invvar"))) return rc;
  if ((rc = upload(ctx, good, in->pix_good, npix, "pix_good"))) return rc;
  if (n > 0) {
    if ((rc = upload(ctx, px, in->pos_x, sizeof(float) * n, "pos_x"))) return rc;
    if ((rc = upload(ctx, py, in->pos_y, sizeof(float) * n, "pos_y"))) return rc;
  }
  if ((rc = upload(ctx, coefs, in->psf_coefs, sizeof(float) * (size_t)H * W * in->psf_nterms,
                   "psf")))
    return rc;
  if ((rc = upload(ctx, os, osh, sizeof(osh), "psf origin"))) return rc;
  if ((rc = upload(ctx, bn, bnh, sizeof(bnh), "bg origin"))) return rc;
  if (any_gal) {
    if ((rc = upload(ctx, ctx->sp[24].ptr, in->source_type, sizeof(int) * n, "types"))) return rc;
    if ((rc = upload(ctx, ctx->sp[25].ptr, in->logre, sizeof(float) * n, "logre"))) return rc;
    if ((rc = upload(ctx, ctx->sp[26].ptr, in->ee1, sizeof(float) * n, "ee1"))) return rc;
    if ((rc = upload(ctx, ctx->sp[27].ptr, in->ee2, sizeof(float) * n, "ee2"))) return rc;
    if ((rc = upload(ctx, ctx->sp[28].ptr, in->sersic_n, sizeof(float) * n, "sersic_n")))
      return rc;
    if (direct) {
      const size_t kb = sizeof(float) * (size_t)in->exp_k;
      if ((rc = upload(ctx, ctx->sp[31].ptr, in->exp_amp, kb, "exp_amp"))) return rc;
      if ((rc = upload(ctx, (char*)ctx->sp[31].ptr + kb, in->exp_var, kb, "exp_var"))) return rc;
    }
  }
  if (n > 0 && kmax > 0) {
    if ((rc = upload(ctx, nidx, in->neighbor_idx, sizeof(int) * (size_t)n * kmax, "nbr")))
      return rc;
    if ((rc = upload(ctx, nmask, in->neighbor_mask, (size_t)n * kmax, "nbr"))) return rc;
  }
  launch_sparse_band(d, ctx->stream);
  CK(cudaGetLastError(), "sparse launch");
  std::vector<float> x(nt), var(nt);
  if ((rc = download(ctx, x.data(), d.x, sizeof(float) * nt, "x"))) return rc;
  if ((rc = download(ctx, var.data(), d.var, sizeof(float) * nt, "var"))) return rc;
  CK(cudaStreamSynchronize(ctx->stream), "sparse solve");
  bool fin = true;
  for (int i = 0; i < nt; ++i) fin = fin && std::isfinite(x[i]);
  for (int i = 0; i < n; ++i) {
    if (out->fluxes) out->fluxes[i] = x[i];
    if (out->flux_var) out->flux_var[i] = var[i];
  }
  for (int m = 0; m < M; ++m) {
    if (out->bg_coefs) out->bg_coefs[m] = x[n + m];
    if (out->bg_var) out->bg_var[m] = var[n + m];
  }
  out->converged = fin ? 1 : 0;
  return UPH_OK;
}

int uph_island_roots(uph_ctx* ctx, const double* pos_x, const double* pos_y,
                     const double* radius, const uint8_t* forced_singleton,
                     int32_t n, int32_t* root_out) {
  if (!ctx) return UPH_ERR_INVALID;
  if (n < 0) return set_err(ctx, UPH_ERR_INVALID, "negative source count");
  if (n == 0) return UPH_OK;
  if (!pos_x || !pos_y || !radius || !root_out)
    return set_err(ctx, UPH_ERR_INVALID, "null island input");
  double xmin = INFINITY, xmax = -INFINITY, ymin = INFINITY, ymax = -INFINITY, rmax = 0.0;
  for (int i = 0; i < n; ++i) {
    if (!std::isfinite(pos_x[i]) || !std::isfinite(pos_y[i]) || !std::isfinite(radius[i]) ||
        !(radius[i] > 0.0))
      return set_err(ctx, UPH_ERR_INVALID, "non-finite position or radius at %d", i);
    xmin = std::min(xmin, pos_x[i]);
    xmax = std::max(xmax, pos_x[i]);
    ymin = std::min(ymin, pos_y[i]);
    ymax = std::max(ymax, pos_y[i]);
    rmax = std::max(rmax, radius[i]);
  }
  // coupled sources lie in the same or adjacent cells of pitch >= 2 r_max;
  // the grid is capped at 4096 cells a side
  const double span = std::max(xmax - xmin, ymax - ymin);
  const double cell = std::max(2.0 * rmax, span / 4096.0);
  const int ncx = (int)std::floor((xmax - xmin) / cell) + 1;
  const int ncy = (int)std::floor((ymax - ymin) / cell) + 1;
  const size_t ncell = (size_t)ncx * ncy;
  cudaSetDevice(ctx->device);
  const size_t sizes[13] = {sizeof(double) * n, sizeof(double) * n, sizeof(double) * n,
                            (size_t)n, sizeof(int) * n, sizeof(int) * ncell,
                            sizeof(int) * (ncell + 1), sizeof(int) * ncell, sizeof(int) * n,
                            sizeof(int) * n, sizeof(int) * n, sizeof(int), 16};
  for (int i = 0; i < 13; ++i) {
    int rc = ensure(ctx, ctx->isl[i], sizes[i], "island decomposition");
    if (rc) return rc;
  }
  IslandDev d{};
  d.n = n; d.ncx = ncx; d.ncy = ncy; d.x0 = xmin; d.y0 = ymin; d.cell = cell;
  d.tries = ctx->isl_tries;
  double* x = (double*)ctx->isl[0].ptr;
  double* y = (double*)ctx->isl[1].ptr;
  double* r = (double*)ctx->isl[2].ptr;
  uint8_t* single = (uint8_t*)ctx->isl[3].ptr;
  d.x = x; d.y = y; d.r = r; d.single = forced_singleton ? single : nullptr;
  d.cid = (int*)ctx->isl[4].ptr;
  d.count = (int*)ctx->isl[5].ptr;
  d.start = (int*)ctx->isl[6].ptr;
  d.cursor = (int*)ctx->isl[7].ptr;
  d.bucket = (int*)ctx->isl[8].ptr;
  d.parent = (int*)ctx->isl[9].ptr;
  d.root = (int*)ctx->isl[10].ptr;
  d.err = (int*)ctx->isl[11].ptr;
  int rc;
  if ((rc = upload(ctx, x, pos_x, sizeof(double) * n, "pos_x"))) return rc;
  if ((rc = upload(ctx, y, pos_y, sizeof(double) * n, "pos_y"))) return rc;
  if ((rc = upload(ctx, r, radius, sizeof(double) * n, "radius"))) return rc;
  if (forced_singleton && (rc = upload(ctx, single, forced_singleton, (size_t)n, "singleton")))
    return rc;
  CK(cudaMemsetAsync(d.count, 0, sizeof(int) * ncell, ctx->stream), "island counts");
  CK(cudaMemsetAsync(d.err, 0, sizeof(int), ctx->stream), "island flag");
  launch_island_roots(d, ctx->stream);
  CK(cudaGetLastError(), "island launch");
  int err = 0;
  if ((rc = download(ctx, root_out, d.root, sizeof(int) * n, "roots"))) return rc;
  if ((rc = download(ctx, &err, d.err, sizeof(int), "island flag"))) return rc;
  CK(cudaStreamSynchronize(ctx->stream), "island decomposition");
  if (err)
    return set_err(ctx, UPH_ERR_TIMEOUT,
                   "union-find retries exhausted (%d attempts per coupled pair)",
                   ctx->isl_tries);
  return UPH_OK;
}

int uph_set_island_retry_limit(uph_ctx* ctx, int32_t tries) {
  if (!ctx) return UPH_ERR_INVALID;
  if (tries < 0) return set_err(ctx, UPH_ERR_INVALID, "negative retry limit");
  ctx->isl_tries = tries;
  return UPH_OK;
}

int uph_job_chunk_time(const uph_job* job, int32_t chunk_id, float* ms) {
  if (!job || !ms || chunk_id < 0 || chunk_id >= (int)job->chunks.size())
    return UPH_ERR_INVALID;
  *ms = job->chunks[chunk_id]->done_ms;
  return UPH_OK;
}

int uph_job_kernel_work(const uph_job* job, int32_t kind, double* bytes,
                        double* flops) {
  if (!job || kind < 0 || kind >= WK_KINDS) return UPH_ERR_INVALID;
  if (bytes) *bytes = job->kbytes[kind];
  if (flops) *flops = job->kflops[kind];
  return UPH_OK;
}

int uph_job_kernel_exps(const uph_job* job, int32_t kind, double* exps) {
  if (!job || !exps || kind < 0 || kind >= WK_KINDS) return UPH_ERR_INVALID;
  *exps = job->kexps[kind];
  return UPH_OK;
}

int uph_measure_peaks(uph_ctx* ctx, double* out) {
  if (!ctx) return UPH_ERR_INVALID;
  if (!out) return set_err(ctx, UPH_ERR_INVALID, "null output");
  cudaSetDevice(ctx->device);
  const int rc = measure_peaks(ctx->stream, ctx->sm_count, out);
  if (rc) return cuda_err(ctx, (cudaError_t)rc, "peak kernels");
  return UPH_OK;
}

int uph_run_chunk(uph_ctx* ctx, const uph_class_desc* cls,
                  const uph_chunk_in* in, int32_t max_steps,
                  uph_chunk_out* out) {
  if (!ctx) return UPH_ERR_INVALID;
  if (!out) return set_err(ctx, UPH_ERR_INVALID, "null output");
  uph_job* job = nullptr;
  int rc = uph_job_create(ctx, &job);
  if (rc) return rc;
  rc = uph_job_add_chunk(job, cls, in, nullptr);
  if (!rc) rc = uph_job_solve(job, max_steps);
  if (!rc) rc = uph_job_read(job, 0, out);
  uph_job_destroy(job);
  return rc;
}

}  // extern "C"

// Allocation-free final-flux pass (uph_fluxes_noalloc).
//
// Some callers of this library cannot call cudaMalloc: a host that runs
// inside a framework owning the whole device memory pool (foreign
// allocations would fragment or exceed its budget), or a serving process
// that must not allocate once it has started (fixed memory budget, no
// allocator calls on the request path).  They already hold device buffers
// for the field, the PSF and the island parameters, and want fluxes back in
// buffers they own.  uph_fluxes_noalloc gives them the star-island final-flux
// pass -- render every member at fixed parameters (reference render mode),
// solve the per-band VarPro fluxes and compute the island chi2 -- using the
// same kernels as the solver, with every intermediate (stamps, per-band
// chi2, good-pixel counts, island flags, per-member render set-up records)
// in the file-scope device array
// below instead of memory allocated per call.
//
// Limits and sharing rules:
//  * the array holds UPH_NOALLOC_SCRATCH_BYTES; a call whose intermediates
//    do not fit is rejected with UPH_ERR_INVALID and a message;
//  * every GPU that loads the library keeps the array until the process
//    exits;
//  * every call uses the same array and leaves its contents behind; each
//    call writes every intermediate it later reads, so no state carries
//    over, but two calls that overlap on the GPU (different streams, or
//    different host threads) race on the array and must be serialised by
//    the caller;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) and sets the kernels' shared-memory limits, with
//    that device current; make that first call before any stream capture.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/uniphot_b200.h"
#include "uph_internal.cuh"

int uph_render_setup();
int uph_solve_setup();

namespace {

static __device__ __align__(256) unsigned char
    g_noalloc_scratch[UPH_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

void put_err(const uph_noalloc_args* a, const char* msg) {
  if (a && a->err_buf && a->err_len > 0) {
    std::snprintf(a->err_buf, (size_t)a->err_len, "%s", msg);
  }
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Per-island validation and set-up.  An island is solved only when its
// real members occupy the leading member slots (at least one), every real
// member is a point source, its window lies inside the padded field and
// every real member's position is finite and near the window; such an
// island gets the flags of an active island.  Any other island is marked
// converged, which the render and flux kernels skip (they run in the trial
// phase), and k_noalloc_finish sets its outputs to NaN.
__global__ void k_noalloc_prepare(int n, int N, int B, int T, int Hp, int Wp,
                                  const uint8_t* mmask, const int32_t* stype,
                                  const int32_t* ox, const int32_t* oy,
                                  const float* x0b, const float* y0b,
                                  const float* p, uint8_t* flags, int* nr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int cnt = 0;
  while (cnt < N && mmask[(size_t)i * N + cnt]) ++cnt;
  bool ok = cnt >= 1;
  for (int k = cnt; k < N; ++k) ok = ok && !mmask[(size_t)i * N + k];
  // the window (B x B at ox, oy) inside the padded field
  ok = ok && ox[i] >= 0 && oy[i] >= 0 && ox[i] <= Wp - B && oy[i] <= Hp - B;
  // positions relative to the window origin: finite and within a stamp of
  // the window, so that the stamp placement arithmetic stays in range
  const float lo = -(float)(T + B), hi = (float)(2 * B + T);
  for (int k = 0; k < cnt && ok; ++k) {
    const float gx = p[(size_t)i * 6 * N + 6 * k] - x0b[i];
    const float gy = p[(size_t)i * 6 * N + 6 * k + 1] - y0b[i];
    ok = stype[(size_t)i * N + k] == 0 && gx >= lo && gx <= hi && gy >= lo && gy <= hi;
  }
  nr[i] = ok ? cnt : 0;
  flags[i] = ok ? FL_REAL : (FL_REAL | FL_CONV);
}

// Island chi2: per-band sums (formed exactly) accumulated in float32 in band
// order, as the solver's accept step does; NaN outputs for the islands that
// k_noalloc_prepare rejected.
__global__ void k_noalloc_finish(int n, int nb, int N, const uint8_t* flags,
                                 const double* chi2b, float* chi2, float* flux,
                                 float* ferr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (flags[i] & FL_CONV) {
    chi2[i] = __int_as_float(0x7fc00000);
    for (int j = 0; j < nb * N; ++j) {
      flux[(size_t)i * nb * N + j] = __int_as_float(0x7fc00000);
      ferr[(size_t)i * nb * N + j] = __int_as_float(0x7fc00000);
    }
    return;
  }
  float c = 0.f;
  for (int b = 0; b < nb; ++b) c = __fadd_rn(c, (float)chi2b[(size_t)i * nb + b]);
  chi2[i] = c;
}

}  // namespace

extern "C" int uph_fluxes_noalloc(const uph_noalloc_args* a) {
  if (!a) return UPH_ERR_INVALID;
  const int n = a->n_islands, N = a->nsrc, B = a->bbox, T = a->tier, nb = a->n_bands;
  if (n <= 0 || N <= 0 || N > UPH_MAXN || B <= 0 || T <= 0 || (T % 2) == 0 ||
      nb <= 0 || a->Hp <= 0 || a->Wp <= 0 ||
      !(a->nt == 1 || a->nt == 3 || a->nt == 6 || a->nt == 10 || a->nt == 15 ||
        a->nt == 21)) {
    put_err(a, "uph_fluxes_noalloc: invalid sizes");
    return UPH_ERR_INVALID;
  }
  if (!a->data || !a->invvar || !a->psf_coefs || !a->psf_origin_scale || !a->ox ||
      !a->oy || !a->x0b || !a->y0b || !a->stype || !a->mmask || !a->p ||
      !a->fluxes || !a->ferr || !a->chi2) {
    put_err(a, "uph_fluxes_noalloc: null device pointer");
    return UPH_ERR_INVALID;
  }
  const int Sz = B < T ? B : T;
  size_t off = 0;
  const size_t o_flags = off;
  off = align256(off + (size_t)n);
  const size_t o_nr = off;
  off = align256(off + sizeof(int) * (size_t)n);
  const size_t o_chi2b = off;
  off = align256(off + sizeof(double) * (size_t)n * nb);
  const size_t o_ngood = off;
  off = align256(off + sizeof(int) * (size_t)n * nb);
  const size_t o_stamps = off;
  off = align256(off + sizeof(float) * (size_t)n * nb * N * Sz * Sz);
  const size_t o_mrec = off;
  off = align256(off + sizeof(MemberRecord) * (size_t)n * nb * N);
  if (off > (size_t)UPH_NOALLOC_SCRATCH_BYTES) {
    char msg[256];
    std::snprintf(msg, sizeof msg,
                  "uph_fluxes_noalloc: chunk needs %zu bytes of scratch, the "
                  "fixed array holds %u; pass fewer islands",
                  off, (unsigned)UPH_NOALLOC_SCRATCH_BYTES);
    put_err(a, msg);
    return UPH_ERR_INVALID;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    put_err(a, "uph_fluxes_noalloc: no current CUDA device");
    return UPH_ERR_CUDA;
  }
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        put_err(a, "uph_fluxes_noalloc: cudaGetSymbolAddress failed");
        return UPH_ERR_CUDA;
      }
      if (uph_render_setup() != 0 || uph_solve_setup() != 0) {
        put_err(a, "uph_fluxes_noalloc: kernel attribute setup failed");
        return UPH_ERR_CUDA;
      }
      g_scratch_ptr[dev] = p;
    }
    base = (unsigned char*)g_scratch_ptr[dev];
  }
  cudaStream_t s = (cudaStream_t)a->stream;
  ClassDev c;
  std::memset(&c, 0, sizeof c);
  c.n_isl = n; c.nb = nb; c.N = N; c.nP = 6 * N; c.B = B; c.T = T; c.Sz = Sz; c.R = 1;
  c.Kmax = N + 1; c.nLmax = 1; c.ntile_side = (Sz + UPH_TILE - 1) / UPH_TILE;
  c.mode = UPH_RENDER_REFERENCE; c.nt = a->nt; c.psf_varies = a->nt > 1;
  c.native = (a->native_stamp > 0 && a->native_stamp < T) ? (a->native_stamp | 1) : T;
  c.has_gal = 0;
  c.Hp = a->Hp; c.Wp = a->Wp;
  c.dstack = a->data; c.wstack = a->invvar;
  c.psf_coefs = a->psf_coefs; c.psf_os = a->psf_origin_scale;
  c.ox = a->ox; c.oy = a->oy; c.x0b = a->x0b; c.y0b = a->y0b;
  c.stype = a->stype; c.mmask = a->mmask;
  c.p = const_cast<float*>(a->p);
  c.flags = base + o_flags;
  c.isl_nr = (const int*)(base + o_nr);
  c.chi2b = (double*)(base + o_chi2b);
  c.ngood = (int*)(base + o_ngood);
  c.stamps = (float*)(base + o_stamps);
  c.mrec = (MemberRecord*)(base + o_mrec);
  c.flux = a->fluxes;
  c.ferr = a->ferr;
  c.reg = a->reg;
  k_noalloc_prepare<<<(n + 127) / 128, 128, 0, s>>>(
      n, N, B, T, a->Hp, a->Wp, a->mmask, a->stype, a->ox, a->oy, a->x0b, a->y0b,
      a->p, c.flags, (int*)(base + o_nr));
  // trial phase: every island without the converged flag, i.e. every
  // island that passed the checks above
  launch_render(c, c.p, PH_TRIAL, s);
  launch_gram_trial(c, c.p, PH_TRIAL, 1, nullptr, nullptr, s);
  k_noalloc_finish<<<(n + 127) / 128, 128, 0, s>>>(n, nb, N, c.flags, c.chi2b, a->chi2,
                                                  a->fluxes, a->ferr);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char msg[256];
    std::snprintf(msg, sizeof msg, "uph_fluxes_noalloc: %s", cudaGetErrorString(e));
    put_err(a, msg);
    return UPH_ERR_CUDA;
  }
  return UPH_OK;
}

// Per-grid, per-band sparse forced photometry of point sources
// (forced_phot_sparse.py:342-562): fixed-position PSF stamps, the weighted
// normal matrix of stamps and a polynomial background, an element-wise
// ridge, a float64 solve and the diagonal of the inverse.
//
//   k_sp_gal      galaxies (the "fft" backend, source_model.py:304-318):
//                 the PSF at the source, the Sersic mixture's transform
//                 times the padded PSF's (sersic_mog.py:153-194) by radix-2
//                 shared-memory FFTs, cropped to the stamp, plus the core
//                 times the PSF
//   k_sp_exp_direct  EXP galaxies on the "direct" backend (source_model.py:
//                 218-256, 298-303), one CTA per source: the PSF stamp and
//                 the exponential mixture at pixel centres in shared memory,
//                 the profile normalised, their same-size convolution
//                 renormalised to unit sum
//   k_sp_stamps   one CTA per source: PSF polynomial at the source (or the
//                 galaxy stamp), unit-sum renormalisation on the all-star
//                 path, Lanczos-3 x then y pass in shared memory
//   k_sp_self     one CTA per source: sum w s^2, sum w s d, sum w s B_m over
//                 the stamp (zero weight outside the grid)
//   k_sp_pairs    one warp per neighbour slot: sum w_s s_s s_t over the
//                 stamps' overlap
//   k_sp_bg       grid-stride partial sums of w B_m B_n and w B_m d per CTA
//   k_sp_assemble the (n + M)^2 system in float as the reference assembles
//                 it (pairs scatter-added), ridge, promoted to float64 with
//                 the identity and the right-hand side beside it
//   k_gj_pivot / k_gj_elim  Gauss-Jordan with partial pivoting on
//                 [A | I | b], one pivot column per launch pair, rows
//                 eliminated across the whole grid
//
// The background basis X^m Y^n is evaluated per pixel in float64 and
// rounded once, X = (grid x0 + column - x_origin) / x_scale.

#include "uph_internal.cuh"

namespace {

constexpr int ST = 256;

__device__ __forceinline__ float bg_term(int t, int gx, int gy, const double* bn) {
  // terms (0,0), (1,0), (0,1), (2,0), (1,1), (0,2)
  const double X = ((double)gx - bn[0]) / bn[1];
  const double Y = ((double)gy - bn[2]) / bn[3];
  switch (t) {
    case 0: return 1.f;
    case 1: return (float)X;
    case 2: return (float)Y;
    case 3: return (float)(X * X);
    case 4: return (float)(X * Y);
    default: return (float)(Y * Y);
  }
}

__device__ void psf_basis_at(float x, float y, const float* os, int nt, float* beta) {
  const float X = __fdiv_rn(__fsub_rn(x, os[0]), os[1]);
  const float Y = __fdiv_rn(__fsub_rn(y, os[2]), os[3]);
  for (int t = 0; t < nt; ++t) {
    int m, q;
    term_mn(t, m, q);
    float xm = 1.f, yq = 1.f;
    for (int i = 0; i < m; ++i) xm *= X;
    for (int i = 0; i < q; ++i) yq *= Y;
    beta[t] = xm * yq;
  }
}

constexpr int MAXPS = 512;

// Unshifted galaxy stamps (H x W) of the extended sources; a grid of CTAs
// loops over the sources with a work space each of sparse_gal_floats and a
// shared line buffer for the radix-2 FFTs.
constexpr int SP_FFT_SMEM = 32768;

__host__ __device__ inline size_t sp_align64(size_t f) { return (f + 63) & ~(size_t)63; }

__global__ void __launch_bounds__(ST)
k_sp_gal(const SparseDev d) {
  extern __shared__ float2 fbuf[];
  __shared__ float cw[MAXPS], sw[MAXPS];
  __shared__ float beta[UPH_MAXNT];
  __shared__ double ga[UPH_MAXGAL], gv[UPH_MAXGAL];
  __shared__ double gcore;
  __shared__ float cg[3];
  const int tid = threadIdx.x;
  const int H = d.H, W = d.W, PP = d.fft_P, Hf = PP / 2 + 1;
  const int logP = 31 - __clz(PP);
  const int lb = SP_FFT_SMEM / (8 * PP);
  for (int m = tid; m < PP; m += ST) {
    double sn, cs;
    sincospi(2.0 * (double)m / (double)PP, &sn, &cs);
    cw[m] = (float)cs;
    sw[m] = (float)sn;
  }
  float* ws = d.gws + (size_t)blockIdx.x * d.gal_floats;
  const size_t PH = (size_t)PP * Hf;
  float* img = ws;                                            // H x W
  float2* R = (float2*)(ws + sp_align64((size_t)H * W));      // H x Hf
  float2* X = R + (size_t)H * Hf;                             // P x Hf
  float* Fs = (float*)(X + PH);                               // P x Hf
  float2* Cc = (float2*)(Fs + sp_align64(PH));                // H x Hf
  for (int s = blockIdx.x; s < d.n; s += gridDim.x) {
    __syncthreads();
    if (d.stype[s] == 0) continue;     // stars take the PSF itself
    if (tid == 0) {
      psf_basis_at(d.px[s], d.py[s], d.os, d.nterms, beta);
      // Sersic mixture at the source's index (sersic_mog.py:81-100)
      int seg;
      double t, dt;
      sersic_segment(d.tb_knots, d.tb_n, d.tb_nmin, d.tb_nmax, (double)d.sn[s], &seg, &t, &dt);
      for (int g = 0; g < d.tb_k; ++g) {
        ga[g] = (1 - t) * d.tb_amps[seg * d.tb_k + g] + t * d.tb_amps[(seg + 1) * d.tb_k + g];
        gv[g] = exp((1 - t) * d.tb_lv[seg * d.tb_k + g] + t * d.tb_lv[(seg + 1) * d.tb_k + g]);
      }
      gcore = (1 - t) * d.tb_core[seg] + t * d.tb_core[seg + 1];
      float dc[3][3];
      cov_terms((double)d.lr[s], (double)d.e1[s], (double)d.e2[s], cg, dc);
    }
    __syncthreads();
    for (int e = tid; e < H * W; e += ST) {
      const float* cf = d.coefs + (size_t)e * d.nterms;
      float v = 0.f;
      for (int t = 0; t < d.nterms; ++t) v = fmaf(cf[t], beta[t], v);
      img[e] = v;
    }
    __syncthreads();
    fft2_forward(img, H, W, PP, logP, R, X, fbuf, lb, cw, sw);
    // the mixture's transform in float32, as the reference evaluates it
    const float kk = -(float)UPH_TWO_PI2;
    for (int e = tid; e < (int)PH; e += ST) {
      const int w = e / Hf, u = e - (e / Hf) * Hf;
      const float nu = (float)u / (float)PP;
      const float nw = (float)(w < PP / 2 ? w : w - PP) / (float)PP;
      const float ex = kk * (cg[0] * nu * nu + cg[1] * nw * nw + 2.f * cg[2] * nu * nw);
      float F = 0.f;
      for (int g = 0; g < d.tb_k; ++g) F = fmaf((float)ga[g], expf((float)gv[g] * ex), F);
      Fs[e] = F;
    }
    __syncthreads();
    fft2_inverse_cols(X, Fs, false, 0.f, 0.f, 0.f, H, PP, logP, Cc, fbuf, lb, cw, sw);
    float* o = d.gal + (size_t)s * H * W;
    fft2_inverse_rows(Cc, H, W, PP, logP, o, fbuf, lb, cw, sw);
    for (int e = tid; e < H * W; e += ST) o[e] = (float)((double)o[e] + gcore * (double)img[e]);
  }
}

__device__ __forceinline__ double block_sum_sp(double v, double* red) {
  // red: ST / 32 doubles; every thread returns the CTA's sum
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < ST / 32; ++w) t += red[w];
  return t;
}

// "direct" EXP stamps, unshifted (H x W) into d.gal; dynamic shared memory
// sparse_stamp_smem(H, W): the profile then the PSF stamp.
__global__ void __launch_bounds__(ST)
k_sp_exp_direct(const SparseDev d) {
  extern __shared__ float sm[];
  __shared__ float beta[UPH_MAXNT];
  __shared__ float shp[4];
  __shared__ double red[ST / 32];
  const int s = blockIdx.x;
  if (s >= d.n || d.stype[s] != 1) return;   // one source per CTA: uniform exit
  const int tid = threadIdx.x, H = d.H, W = d.W, HW = H * W;
  float* prof = sm;
  float* psf = sm + HW;
  if (tid == 0) {
    psf_basis_at(d.px[s], d.py[s], d.os, d.nterms, beta);
    // the shape matrix rows (a, b), (c, d) of source_model.py:226-237
    const float re = fminf(fmaxf(expf(d.lr[s]), 0.1f), 1000.f);
    const float e1 = d.e1[s], e2 = d.e2[s];
    const float e = 1.f - expf(-hypotf(e1, e2));
    const float inv_ba = fminf((1.f + e) / fmaxf(1.f - e, 1e-4f), 1000.f);
    float st, ct;
    sincosf(0.5f * atan2f(e2, e1), &st, &ct);
    shp[0] = re * ct / inv_ba;
    shp[1] = re * st;
    shp[2] = -re * st / inv_ba;
    shp[3] = re * ct;
  }
  __syncthreads();
  const float* amp = d.exp_mog;
  const float* var = d.exp_mog + d.exp_k;
  const float a = shp[0], b = shp[1], c = shp[2], dd = shp[3];
  double acc = 0.0;
  for (int e = tid; e < HW; e += ST) {
    const float* cf = d.coefs + (size_t)e * d.nterms;
    float v = 0.f;
    for (int t = 0; t < d.nterms; ++t) v = fmaf(cf[t], beta[t], v);
    psf[e] = v;
    const float y = (float)(e / W - H / 2), x = (float)(e % W - W / 2);
    float p = 0.f;
    for (int k = 0; k < d.exp_k; ++k) {
      const float vk = var[k];
      const float sxx = vk * (a * a + b * b), sxy = vk * (a * c + b * dd);
      const float syy = vk * (c * c + dd * dd);
      const float det = fmaxf(sxx * syy - sxy * sxy, 1e-12f);
      const float q = (syy * x * x - 2.f * sxy * x * y + sxx * y * y) / det;
      p += amp[k] / (2.f * 3.14159265358979f * sqrtf(det)) * expf(-0.5f * fminf(q, 200.f));
    }
    prof[e] = p;
    acc += (double)p;
  }
  const double tp = block_sum_sp(acc, red);
  if (tp > 0.0)
    for (int e = tid; e < HW; e += ST) prof[e] = (float)((double)prof[e] / tp);
  __syncthreads();
  // out[y][x] = sum_{i,j} psf[i][j] prof[y + oy - i][x + ox - j] over the
  // profile's extent: the full convolution's window from ((H-1)/2, (W-1)/2)
  const int oy = (H - 1) / 2, ox = (W - 1) / 2;
  float* o = d.gal + (size_t)s * HW;
  acc = 0.0;
  for (int e = tid; e < HW; e += ST) {
    const int y = e / W, x = e - (e / W) * W;
    const int i0 = max(0, y + oy - (H - 1)), i1 = min(H - 1, y + oy);
    const int j0 = max(0, x + ox - (W - 1)), j1 = min(W - 1, x + ox);
    float v = 0.f;
    for (int i = i0; i <= i1; ++i) {
      const int r = (y + oy - i) * W + x + ox;     // r - j indexes the profile
      for (int j = j0; j <= j1; ++j) v = fmaf(psf[i * W + j], prof[r - j], v);
    }
    o[e] = v;
    acc += (double)v;
  }
  const double tc = block_sum_sp(acc, red);
  if (tc > 0.0)
    for (int e = tid; e < HW; e += ST) o[e] = (float)((double)o[e] / tc);
}

__global__ void __launch_bounds__(ST)
k_sp_stamps(int n, int H, int W, const float* __restrict__ coefs, int nt,
            const float* __restrict__ os, const float* __restrict__ px,
            const float* __restrict__ py, float gx0, float gy0, int renorm,
            float* __restrict__ out, int* __restrict__ ixt, int* __restrict__ iyt,
            const int* __restrict__ stype, const float* __restrict__ gal) {
  extern __shared__ float sm[];
  __shared__ float beta[UPH_MAXNT];
  __shared__ float Lx[7], Ly[7], dL[7];
  __shared__ double red[ST / 32];
  __shared__ float norm;
  const int s = blockIdx.x;
  if (s >= n) return;
  const int tid = threadIdx.x;
  float* raw = sm;            // H x W
  float* tmp = sm + H * W;    // H x W
  const bool is_gal = stype && stype[s] != 0;
  if (tid == 0) {
    psf_basis_at(px[s], py[s], os, nt, beta);
    const float xg = __fsub_rn(px[s], gx0), yg = __fsub_rn(py[s], gy0);
    lanczos_taps((double)__fsub_rn(xg, rintf(xg)), Lx, dL);
    lanczos_taps((double)__fsub_rn(yg, rintf(yg)), Ly, dL);
    // stamp_top_left (forced_phot_sparse.py:255-269)
    ixt[s] = (int)rintf(xg) - W / 2;
    iyt[s] = (int)rintf(yg) - H / 2;
  }
  __syncthreads();
  double acc = 0.0;
  for (int e = tid; e < H * W; e += ST) {
    float v;
    if (is_gal) {
      v = gal[(size_t)s * H * W + e];
    } else {
      const float* cf = coefs + (size_t)e * nt;
      v = 0.f;
      for (int t = 0; t < nt; ++t) v = fmaf(cf[t], beta[t], v);
    }
    raw[e] = v;
    acc += (double)v;
  }
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if ((tid & 31) == 0) red[tid >> 5] = acc;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < ST / 32; ++w) t += red[w];
    norm = renorm ? (float)fmax(t, 1e-12) : 1.f;
  }
  __syncthreads();
  if (renorm)
    for (int e = tid; e < H * W; e += ST) raw[e] = __fdiv_rn(raw[e], norm);
  __syncthreads();
  // x pass: tmp[i][j] = sum_q Lx[q] raw[i][j + q - 3], zero border
  for (int e = tid; e < H * W; e += ST) {
    const int i = e / W, j = e - (e / W) * W;
    float a = 0.f;
    bool first = true;
    for (int q = 0; q < 7; ++q) {
      const int jj = j + q - 3;
      const float v = (jj >= 0 && jj < W) ? raw[i * W + jj] : 0.f;
      a = first ? Lx[q] * v : fmaf(Lx[q], v, a);
      first = false;
    }
    tmp[e] = a;
  }
  __syncthreads();
  float* o = out + (size_t)s * H * W;
  for (int e = tid; e < H * W; e += ST) {
    const int i = e / W, j = e - (e / W) * W;
    float a = 0.f;
    bool first = true;
    for (int q = 0; q < 7; ++q) {
      const int ii = i + q - 3;
      const float v = (ii >= 0 && ii < H) ? tmp[ii * W + j] : 0.f;
      a = first ? Ly[q] * v : fmaf(Ly[q], v, a);
      first = false;
    }
    o[e] = a;
  }
}

__global__ void __launch_bounds__(ST)
k_sp_self(int n, int H, int W, const float* __restrict__ st, const int* __restrict__ ixt,
          const int* __restrict__ iyt, const float* __restrict__ data,
          const float* __restrict__ wgrid, int h, int w, int gx0, int gy0, const double* bn4,
          int M, float* __restrict__ diag, float* __restrict__ twd, float* __restrict__ twb) {
  __shared__ double red[2 + 6][ST / 32];
  __shared__ double bn[4];
  const int s = blockIdx.x;
  if (s >= n) return;
  const int tid = threadIdx.x;
  if (tid < 4) bn[tid] = bn4[tid];
  __syncthreads();
  double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const float* S = st + (size_t)s * H * W;
  for (int e = tid; e < H * W; e += ST) {
    const int ky = e / W, kx = e - (e / W) * W;
    const int gy = iyt[s] + ky, gx = ixt[s] + kx;
    if (gy < 0 || gy >= h || gx < 0 || gx >= w) continue;
    const float wv = wgrid[(size_t)gy * w + gx];
    const float ws = __fmul_rn(wv, S[e]);
    a[0] += (double)__fmul_rn(ws, S[e]);
    a[1] += (double)__fmul_rn(ws, data[(size_t)gy * w + gx]);
    for (int m = 0; m < M; ++m) a[2 + m] += (double)__fmul_rn(ws, bg_term(m, gx0 + gx, gy0 + gy, bn));
  }
  for (int q = 0; q < 2 + M; ++q) {
    double v = a[q];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((tid & 31) == 0) red[q][tid >> 5] = v;
  }
  __syncthreads();
  if (tid < 2 + M) {
    double t = 0.0;
    for (int w2 = 0; w2 < ST / 32; ++w2) t += red[tid][w2];
    if (tid == 0) diag[s] = (float)t;
    else if (tid == 1) twd[s] = (float)t;
    else twb[(size_t)s * M + tid - 2] = (float)t;
  }
}

__global__ void __launch_bounds__(ST)
k_sp_pairs(int n, int H, int W, int kmax, const int* __restrict__ nidx,
           const uint8_t* __restrict__ nmask, const float* __restrict__ st,
           const int* __restrict__ ixt, const int* __restrict__ iyt,
           const float* __restrict__ wgrid, int h, int w, float* __restrict__ off) {
  const int gw = (blockIdx.x * ST + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (gw >= n * kmax) return;
  const int s = gw / kmax;
  if (!nmask[gw]) {
    if (lane == 0) off[gw] = 0.f;
    return;
  }
  const int t = nidx[gw];
  const int di = iyt[s] - iyt[t], dj = ixt[s] - ixt[t];
  const float* Ss = st + (size_t)s * H * W;
  const float* Sv = st + (size_t)t * H * W;
  double a = 0.0;
  for (int e = lane; e < H * W; e += 32) {
    const int ky = e / W, kx = e - (e / W) * W;
    const int ty = ky + di, tx = kx + dj;
    if (ty < 0 || ty >= H || tx < 0 || tx >= W) continue;
    const int gy = iyt[s] + ky, gx = ixt[s] + kx;
    if (gy < 0 || gy >= h || gx < 0 || gx >= w) continue;
    // the t stamp at a pixel of s inside the grid is inside the grid too
    const float v = __fmul_rn(__fmul_rn(wgrid[(size_t)gy * w + gx], Ss[e]), Sv[ty * W + tx]);
    a += (double)v;
  }
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if (lane == 0) off[gw] = (float)a;
}

__global__ void __launch_bounds__(ST)
k_sp_bg(int h, int w, int gx0, int gy0, const double* bn4, int M,
        const float* __restrict__ data, const float* __restrict__ wgrid,
        double* __restrict__ part) {
  __shared__ double red[27][ST / 32];
  __shared__ double bn[4];
  const int tid = threadIdx.x;
  if (tid < 4) bn[tid] = bn4[tid];
  __syncthreads();
  const int nq = M * M + M;
  double a[42];
#pragma unroll
  for (int q = 0; q < 42; ++q) a[q] = 0.0;
  for (size_t pix = (size_t)blockIdx.x * ST + tid; pix < (size_t)h * w;
       pix += (size_t)gridDim.x * ST) {
    const int gy = (int)(pix / w), gx = (int)(pix - (pix / w) * w);
    const float wv = wgrid[pix];
    if (wv == 0.f) continue;
    float B[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) B[m] = m < M ? bg_term(m, gx0 + gx, gy0 + gy, bn) : 0.f;
    const float d = data[pix];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      if (m >= M) break;
      const float bw = __fmul_rn(B[m], wv);
#pragma unroll
      for (int q = 0; q < 6; ++q)
        if (q < M) a[m * M + q] += (double)__fmul_rn(bw, B[q]);
      a[M * M + m] += (double)__fmul_rn(bw, d);
    }
  }
  // block reduction in chunks of 27 sums, fixed order
  for (int base = 0; base < nq; base += 27) {
    const int cnt = min(27, nq - base);
    for (int q = 0; q < cnt; ++q) {
      double v = a[base + q];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if ((tid & 31) == 0) red[q][tid >> 5] = v;
    }
    __syncthreads();
    if (tid < cnt) {
      double t = 0.0;
      for (int w2 = 0; w2 < ST / 32; ++w2) t += red[tid][w2];
      part[(size_t)blockIdx.x * nq + base + tid] = t;
    }
    __syncthreads();
  }
}

// [A | I | b] in float64, row pitch ld = 2 nt + 1, nt = n + M.
__global__ void k_sp_assemble(int n, int M, int kmax, const float* __restrict__ diag,
                              const float* __restrict__ off, const int* __restrict__ nidx,
                              const uint8_t* __restrict__ nmask,
                              const float* __restrict__ twd, const float* __restrict__ twb,
                              const double* __restrict__ part, int nparts, float reg,
                              float* __restrict__ Af, double* __restrict__ G) {
  // one thread block builds the float matrix (small rows loop), then all
  // threads promote it; launched with one CTA per row of the system
  const int nt = n + M;
  const int r = blockIdx.x;
  if (r >= nt) return;
  const int tid = threadIdx.x;
  const size_t ld = 2 * (size_t)nt + 1;
  float* Ar = Af + (size_t)r * nt;
  for (int j = tid; j < nt; j += blockDim.x) Ar[j] = 0.f;
  __syncthreads();
  const int nq = M * M + M;
  if (tid == 0) {
    if (r < n) {
      Ar[r] = diag[r];
      for (int k = 0; k < kmax; ++k)
        if (nmask[(size_t)r * kmax + k]) {
          const int t = nidx[(size_t)r * kmax + k];
          Ar[t] = __fadd_rn(Ar[t], off[(size_t)r * kmax + k]);
        }
      for (int m = 0; m < M; ++m) Ar[n + m] = twb[(size_t)r * M + m];
    } else {
      const int m = r - n;
      for (int s = 0; s < n; ++s) Ar[s] = twb[(size_t)s * M + m];
      for (int q = 0; q < M; ++q) {
        double t = 0.0;
        for (int p = 0; p < nparts; ++p) t += part[(size_t)p * nq + m * M + q];
        Ar[n + q] = (float)t;
      }
    }
    Ar[r] = __fadd_rn(Ar[r], __fmul_rn(reg, fmaxf(fabsf(Ar[r]), 1e-30f)));
  }
  __syncthreads();
  double* Gr = G + (size_t)r * ld;
  for (int j = tid; j < (int)ld; j += blockDim.x) {
    double v;
    if (j < nt) v = (double)Ar[j];
    else if (j < 2 * nt) v = (j - nt == r) ? 1.0 : 0.0;
    else {
      if (r < n) {
        v = (double)twd[r];
      } else {
        double t = 0.0;
        for (int p = 0; p < nparts; ++p) t += part[(size_t)p * nq + M * M + (r - n)];
        v = (double)(float)t;
      }
    }
    Gr[j] = v;
  }
}

// pivot search in column col (first maximum of |G[r][col]|, r >= col),
// row swap, pivot row scaled to a unit pivot
__global__ void k_gj_pivot(int nt, int col, double* __restrict__ G, int* __restrict__ prow) {
  __shared__ double bv[1024];
  __shared__ int bi[1024];
  const int tid = threadIdx.x;
  const size_t ld = 2 * (size_t)nt + 1;
  double best = -1.0;
  int bidx = col;
  for (int r = col + tid; r < nt; r += blockDim.x) {
    const double v = fabs(G[(size_t)r * ld + col]);
    if (v > best) {
      best = v;
      bidx = r;
    }
  }
  bv[tid] = best;
  bi[tid] = bidx;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (tid < st) {
      const double o = bv[tid + st];
      const int oi = bi[tid + st];
      if (o > bv[tid] || (o == bv[tid] && oi < bi[tid])) {
        bv[tid] = o;
        bi[tid] = oi;
      }
    }
    __syncthreads();
  }
  const int p = bi[0];
  if (p != col)
    for (size_t j = tid; j < ld; j += blockDim.x) {
      const double t = G[(size_t)col * ld + j];
      G[(size_t)col * ld + j] = G[(size_t)p * ld + j];
      G[(size_t)p * ld + j] = t;
    }
  __syncthreads();
  const double inv = 1.0 / G[(size_t)col * ld + col];
  __syncthreads();
  for (size_t j = tid; j < ld; j += blockDim.x) G[(size_t)col * ld + j] *= inv;
  if (tid == 0) *prow = p;
}

// eliminate column col from every other row (the factor of row r is read
// before any thread of that row writes it: one thread block per row)
__global__ void k_gj_elim(int nt, int col, double* __restrict__ G) {
  const int r = blockIdx.x;
  if (r >= nt || r == col) return;
  const size_t ld = 2 * (size_t)nt + 1;
  __shared__ double f;
  if (threadIdx.x == 0) f = G[(size_t)r * ld + col];
  __syncthreads();
  if (f == 0.0) return;
  const double* Pc = G + (size_t)col * ld;
  double* Gr = G + (size_t)r * ld;
  for (size_t j = threadIdx.x; j < ld; j += blockDim.x) Gr[j] -= f * Pc[j];
}

__global__ void k_sp_out(int n, int M, const double* __restrict__ G, float* __restrict__ x,
                         float* __restrict__ var) {
  const int nt = n + M;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nt) return;
  const size_t ld = 2 * (size_t)nt + 1;
  x[r] = (float)G[(size_t)r * ld + 2 * nt];
  var[r] = (float)G[(size_t)r * ld + nt + r];
}

}  // namespace

__global__ void k_sp_wgrid(size_t npix, const float* __restrict__ invvar,
                           const uint8_t* __restrict__ good, float* __restrict__ wgrid) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < npix) wgrid[i] = good[i] ? invvar[i] : 0.f;
}

size_t sparse_stamp_smem(int H, int W) { return 2 * sizeof(float) * (size_t)H * W; }

size_t sparse_gal_floats(int H, int W, int P) {
  const size_t Hf = (size_t)P / 2 + 1;
  return sp_align64((size_t)H * W) + sp_align64(2 * (size_t)H * Hf) + 2 * (size_t)P * Hf +
         sp_align64((size_t)P * Hf) + sp_align64(2 * (size_t)H * Hf) + 64;
}

int sparse_setup() {
  const int rc = (int)cudaFuncSetAttribute(k_sp_stamps,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           200 * 1024);
  if (rc) return rc;
  return (int)cudaFuncSetAttribute(k_sp_exp_direct, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   200 * 1024);
}

// Raw (not renormalised) Lanczos-shifted polynomial-PSF stamps of n point
// sources at (px, py) in field pixels, H x W each, into out, with their
// stamp top-left corners (round(x) - W/2, round(y) - H/2) in ixt / iyt.
void launch_star_stamps(int n, int H, int W, const float* coefs, int nt, const float* os,
                        const float* px, const float* py, float* out, int* ixt, int* iyt,
                        cudaStream_t s) {
  if (n > 0)
    k_sp_stamps<<<(unsigned)n, ST, sparse_stamp_smem(H, W), s>>>(
        n, H, W, coefs, nt, os, px, py, 0.f, 0.f, 0, out, ixt, iyt, nullptr, nullptr);
}

void launch_sparse_band(const SparseDev& d, cudaStream_t s) {
  const int n = d.n, H = d.H, W = d.W, M = d.M, nt = d.n + d.M;
  const size_t npix = (size_t)d.h * d.w;
  k_sp_wgrid<<<(unsigned)((npix + 255) / 256), 256, 0, s>>>(npix, d.invvar, d.good, d.wgrid);
  if (n > 0) {
    if (d.direct)
      k_sp_exp_direct<<<(unsigned)n, ST, sparse_stamp_smem(H, W), s>>>(d);
    else if (d.gal_ctas > 0)
      k_sp_gal<<<(unsigned)d.gal_ctas, ST, SP_FFT_SMEM, s>>>(d);
    k_sp_stamps<<<(unsigned)n, ST, sparse_stamp_smem(H, W), s>>>(
        n, H, W, d.coefs, d.nterms, d.os, d.px, d.py, (float)d.gx0, (float)d.gy0, d.renorm,
        d.stamps, d.ixt, d.iyt, d.stype, d.gal);
    k_sp_self<<<(unsigned)n, ST, 0, s>>>(n, H, W, d.stamps, d.ixt, d.iyt, d.data, d.wgrid,
                                         d.h, d.w, d.gx0, d.gy0, d.bn, M, d.diag, d.twd,
                                         d.twb);
    if (d.kmax > 0) {
      const long long warps = (long long)n * d.kmax;
      k_sp_pairs<<<(unsigned)((warps * 32 + ST - 1) / ST), ST, 0, s>>>(
          n, H, W, d.kmax, d.nidx, d.nmask, d.stamps, d.ixt, d.iyt, d.wgrid, d.h, d.w,
          d.off);
    }
  }
  k_sp_bg<<<(unsigned)d.nparts, ST, 0, s>>>(d.h, d.w, d.gx0, d.gy0, d.bn, M, d.data,
                                            d.wgrid, d.part);
  k_sp_assemble<<<(unsigned)nt, 128, 0, s>>>(n, M, d.kmax, d.diag, d.off, d.nidx, d.nmask,
                                             d.twd, d.twb, d.part, d.nparts, d.reg, d.Af,
                                             d.G);
  for (int col = 0; col < nt; ++col) {
    k_gj_pivot<<<1, 1024, 0, s>>>(nt, col, d.G, d.prow);
    k_gj_elim<<<(unsigned)nt, 256, 0, s>>>(nt, col, d.G);
  }
  k_sp_out<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(n, M, d.G, d.x, d.var);
}

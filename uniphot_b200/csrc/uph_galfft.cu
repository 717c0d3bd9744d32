// Galaxy stamps of the reference render mode (pixelised polynomial PSF):
// the Fourier-domain convolution of the PSF stamp with the galaxy's Sersic
// Gaussian mixture (sersic_mog.py:153-207, source_model.py:264-328),
//
//   S = irfft2(rfft2(pad(psf)) * sum_c a_c exp(v_c e(k)))[:T, :T] + core psf,
//   e(k) = -2 pi^2 (cxx kx^2 + cyy ky^2 + 2 cxy kx ky),
//
// on a P x P grid (P the power of two >= 3T/2), and the partials the Gauss-
// Newton rows need: through the PSF's spatial variation (Sx, Sy: the same
// product with the PSF's position derivatives), the shape (F1 de/dtheta
// with F1 = sum a_c v_c exp(v_c e)) and the Sersic index (sum (da_c + a_c
// dv_c e) exp(v_c e) plus dcore psf, times dn/du).  The mixture's transform
// is real (zero-centred Gaussians), so every product is a complex spectrum
// times a real factor.
//
// The transforms are radix-2 FFTs of whole lines in shared memory (a batch
// of lines per pass: as many as the larger of the T rows and the P/2 + 1
// columns, up to FFT_SMEM_MAX bytes, so a P = 128 grid takes one pass per
// direction): the T non-zero rows of the padded image, then
// the P/2 + 1 columns of their half spectra; on the way back the columns,
// keeping the T rows of the crop, then those rows' real inverses.  One CTA per (island, band, galaxy member), looping over the members
// of a grid sized to the SM count, with its work space in global memory
// (L2-resident per CTA).  The unshifted rows land in c.gstamp, which the
// render's Lanczos passes read in place of the star's polynomial PSF.

#include <algorithm>

#include "../../include/uniphot_b200.h"
#include "uph_internal.cuh"

namespace {

constexpr int GT = 256;
constexpr int MAXP = 512;
// shared line buffer of the FFTs, at most: three CTAs fit an SM beside their
// static shared memory
#ifndef UPH_FFT_SMEM_MAX
#define UPH_FFT_SMEM_MAX (70 * 1024)
#endif
constexpr int FFT_SMEM_MAX = UPH_FFT_SMEM_MAX;

__host__ __device__ inline size_t align64(size_t f) { return (f + 63) & ~(size_t)63; }

__global__ void __launch_bounds__(GT) k_gal_fft(ClassDev c, const float* __restrict__ Pp,
                                                int phase) {
  extern __shared__ float2 fbuf[];          // LB lines of P complex values
  __shared__ float cw[MAXP], sw[MAXP];
  __shared__ int need[7];
  __shared__ int is_gal;
  __shared__ float fa[UPH_MAXGAL], fv[UPH_MAXGAL], fda[UPH_MAXGAL], fdv[UPH_MAXGAL];
  const int tid = threadIdx.x;
  const int T = c.T, PP = c.fft_P, H = PP / 2 + 1;
  const int logP = 31 - __clz(PP);
  const int lb = c.gfft_smem / (8 * PP);
  const int TT = T * T;
  for (int m = tid; m < PP; m += GT) {
    double sn, cs;
    sincospi(2.0 * (double)m / (double)PP, &sn, &cs);
    cw[m] = (float)cs;
    sw[m] = (float)sn;
  }
  float* ws = c.gfft_ws + (size_t)blockIdx.x * c.gfft_floats;
  const size_t PH = (size_t)PP * H;
  float* img = ws;                                          // 3 real T x T
  float2* R = (float2*)(ws + align64(3 * (size_t)TT));      // T x H
  float2* X = R + (size_t)T * H;                            // 3 spectra, P x H
  float* Fs = (float*)(X + 3 * PH);                         // F, F1, dF, P x H
  float2* Cc = (float2*)(Fs + align64(3 * PH));             // T x H
  const int nitems = c.n_isl * c.nb * c.N;
  const bool lin = phase == PH_LIN;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int k = item % c.N;
    const int b = (item / c.N) % c.nb;
    const int isl = item / (c.N * c.nb);
    __syncthreads();
    if (tid == 0) {
      is_gal = isl_active(c.flags[isl], phase) && c.mmask[isl * c.N + k] &&
               c.stype[isl * c.N + k] != 0;
      const uint8_t* kp = c.keep + ((size_t)isl * c.N + k) * 6;
      need[0] = 1;
      need[1] = lin && kp[0] && c.psf_varies;
      need[2] = lin && kp[1] && c.psf_varies;
      for (int q = 0; q < 3; ++q) need[3 + q] = lin && kp[2 + q];
      need[6] = lin && kp[5];
    }
    __syncthreads();
    if (!is_gal) continue;
    const MemberRecord* rec = c.mrec + ((size_t)isl * c.nb + b) * c.N + k;
    for (int g = tid; g < rec->ngal; g += GT) {
      fa[g] = (float)rec->ga[g];
      fv[g] = (float)rec->gv[g];
      fda[g] = (float)rec->gda[g];
      fdv[g] = (float)rec->gdv[g];
    }
    // ---- PSF stamp at the member position and its position partials ----
    for (int e = tid; e < TT; e += GT) {
      const int i = e / T, j = e - (e / T) * T;
      const float* cf = c.psf_coefs + (((size_t)b * T + i) * T + j) * c.nt;
      float v0 = 0.f, v1 = 0.f, v2 = 0.f;
      for (int tt = 0; tt < c.nt; ++tt) {
        const float cv = cf[tt];
        v0 = fmaf(cv, rec->beta[tt], v0);
        v1 = fmaf(cv, rec->betax[tt], v1);
        v2 = fmaf(cv, rec->betay[tt], v2);
      }
      img[e] = v0;
      img[TT + e] = v1;
      img[2 * TT + e] = v2;
    }
    __syncthreads();
    for (int im = 0; im < 3; ++im)
      if (need[im]) fft2_forward(img + im * TT, T, T, PP, logP, R, X + PH * im, fbuf, lb, cw, sw);
    // ---- the mixture's transform and its partials on the grid, in float32
    //      as the reference evaluates it ----
    const float kk = -(float)UPH_TWO_PI2;
    const float cg0 = rec->cg[0], cg1 = rec->cg[1], cg2 = rec->cg[2];
    const int ng = rec->ngal;
    for (int e = tid; e < (int)PH; e += GT) {
      const int w = e / H, u = e - (e / H) * H;
      const float nu = (float)u / (float)PP;
      const float nw = (float)(w < PP / 2 ? w : w - PP) / (float)PP;
      const float ex = kk * (cg0 * nu * nu + cg1 * nw * nw + 2.f * cg2 * nu * nw);
      float F = 0.f, F1 = 0.f, dF = 0.f;
      for (int g = 0; g < ng; ++g) {
        const float E = expf(fv[g] * ex);
        F = fmaf(fa[g], E, F);
        F1 = fmaf(fa[g] * fv[g], E, F1);
        dF = fmaf(fmaf(fa[g] * fdv[g], ex, fda[g]), E, dF);
      }
      Fs[e] = F;
      Fs[PH + e] = F1;
      Fs[2 * PH + e] = dF;
    }
    __syncthreads();
    // ---- inverse transforms of the needed products, cropped to T x T ----
    float* out = c.gstamp + (size_t)item * 7 * TT;
    for (int s = 0; s < 7; ++s) {
      if (!need[s]) continue;
      const float2* Xb = X + PH * (s < 3 ? s : 0);
      const float* fac = Fs + PH * (s < 3 ? 0 : (s < 6 ? 1 : 2));
      const bool shp = s >= 3 && s < 6;
      fft2_inverse_cols(Xb, fac, shp, shp ? rec->dcov[s - 3][0] : 0.f,
                        shp ? rec->dcov[s - 3][1] : 0.f, shp ? rec->dcov[s - 3][2] : 0.f, T, PP,
                        logP, Cc, fbuf, lb, cw, sw);
      float* o = out + (size_t)s * TT;
      fft2_inverse_rows(Cc, T, T, PP, logP, o, fbuf, lb, cw, sw);
      for (int e = tid; e < TT; e += GT) {
        double r = (double)o[e];
        if (s == 0) r += rec->gcore * (double)img[e];
        else if (s == 1) r += rec->gcore * (double)img[TT + e];
        else if (s == 2) r += rec->gcore * (double)img[2 * TT + e];
        else if (s == 6) r = (r + rec->gdcore * (double)img[e]) * (double)rec->dndu;
        o[e] = (float)r;
      }
      __syncthreads();
    }
  }
}

// ---- The legacy "direct" backend for EXP members (source_model.py:218-256,
// 298-303), in float64: the exponential mixture sampled at pixel centres
// and normalised to unit sum, convolved with the PSF stamp ("same": output
// pixel (r, s) sums K[i][j] I[r + o - i][s + o - j], o = T / 2, i and j
// ascending, the order a shifted-add convolution accumulates in), the
// result renormalised to unit sum.  Rows: 0 the stamp; 1-2 its position
// partials through the PSF's spatial variation (the convolution of the
// profile with the PSF's position derivative, through the renormalisation
// by the quotient rule); 3-5 the shape partials (log r_e, e1, e2) by
// central differences of the whole stamp with step DIRECT_FD_STEP; 6 zero
// (no Sersic index).  One CTA per (island, band, member) of a grid-stride
// loop; the PSF stamp and the profile in shared memory, the float64
// intermediates in the CTA's global work space.

constexpr double DIRECT_FD_STEP = 1e-6;
constexpr double DIRECT_PI = 3.141592653589793;

__device__ double direct_block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();                           // red may still be read
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) red[0] = t;
  }
  __syncthreads();
  return red[0];
}

// The exponential mixture at pixel centres of a T x T grid centred at T/2,
// quadratic form clipped at 200, normalised to unit sum (when positive).
__device__ void direct_profile(const ClassDev& c, int T, double lr, double e1, double e2,
                               double* I, double* red) {
  const double re = fmin(fmax(exp(lr), 0.1), 1000.0);
  const double ee = hypot(e1, e2);
  const double e = 1.0 - exp(-ee);
  const double inv_ba = fmin((1.0 + e) / fmax(1.0 - e, 1e-4), 1000.0);
  const double th = 0.5 * atan2(e2, e1);
  const double ct = cos(th), st = sin(th);
  const double a = re * ct / inv_ba, b = re * st, cc = -re * st / inv_ba, d = re * ct;
  const int h = T / 2;
  double part = 0.0;
  for (int q = threadIdx.x; q < T * T; q += blockDim.x) {
    const int i = q / T, j = q - (q / T) * T;
    const double y = (double)(i - h), x = (double)(j - h);
    double v = 0.0;
    for (int g = 0; g < c.exp_k; ++g) {
      const double am = (double)c.exp_amp[g], va = (double)c.exp_var[g];
      const double sxx = va * (a * a + b * b), sxy = va * (a * cc + b * d),
                   syy = va * (cc * cc + d * d);
      const double det = fmax(sxx * syy - sxy * sxy, 1e-12);
      const double qf = (syy * x * x - 2.0 * sxy * x * y + sxx * y * y) / det;
      v += am / (2.0 * DIRECT_PI * sqrt(det)) * exp(-0.5 * fmin(qf, 200.0));
    }
    I[q] = v;
    part += v;
  }
  const double tot = direct_block_sum(part, red);
  if (tot > 0.0)
    for (int q = threadIdx.x; q < T * T; q += blockDim.x) I[q] /= tot;
  __syncthreads();
}

// out = conv_same(I, K) (float64); returns its sum.
__device__ double direct_conv(const double* K, const double* I, int T, double* out,
                              double* red) {
  const int o = T / 2;
  double part = 0.0;
  for (int q = threadIdx.x; q < T * T; q += blockDim.x) {
    const int r = q / T, s = q - (q / T) * T;
    const int ilo = max(0, r + o - (T - 1)), ihi = min(T - 1, r + o);
    const int jlo = max(0, s + o - (T - 1)), jhi = min(T - 1, s + o);
    double acc = 0.0;
    for (int i = ilo; i <= ihi; ++i) {
      const double* Kr = K + i * T;
      const double* Ir = I + (r + o - i) * T + (s + o);
      for (int j = jlo; j <= jhi; ++j) acc = fma(Kr[j], Ir[-j], acc);
    }
    out[q] = acc;
    part += acc;
  }
  return direct_block_sum(part, red);
}

__global__ void __launch_bounds__(GT) k_gal_direct(ClassDev c, const float* __restrict__ Pp,
                                                   int phase) {
  extern __shared__ double dsm[];            // K (T x T), I (T x T)
  __shared__ double red[32];
  __shared__ int need[7];
  __shared__ int is_gal;
  const int tid = threadIdx.x;
  const int T = c.T, TT = T * T;
  double* K = dsm;
  double* I = dsm + TT;
  float* ws = c.gfft_ws + (size_t)blockIdx.x * c.gfft_floats;
  float* img = ws;                                          // 3 float T x T
  double* C = (double*)(ws + align64(3 * (size_t)TT));      // 3 double T x T
  double* S0 = C + TT;
  double* Sp = S0 + TT;
  const int nitems = c.n_isl * c.nb * c.N;
  const bool lin = phase == PH_LIN;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int k = item % c.N;
    const int b = (item / c.N) % c.nb;
    const int isl = item / (c.N * c.nb);
    __syncthreads();
    if (tid == 0) {
      is_gal = isl_active(c.flags[isl], phase) && c.mmask[isl * c.N + k] &&
               c.stype[isl * c.N + k] != 0;
      const uint8_t* kp = c.keep + ((size_t)isl * c.N + k) * 6;
      need[0] = 1;
      need[1] = lin && kp[0] && c.psf_varies;
      need[2] = lin && kp[1] && c.psf_varies;
      for (int q = 0; q < 3; ++q) need[3 + q] = lin && kp[2 + q];
      need[6] = lin && kp[5];
    }
    __syncthreads();
    if (!is_gal) continue;
    const MemberRecord* rec = c.mrec + ((size_t)isl * c.nb + b) * c.N + k;
    for (int e = tid; e < TT; e += GT) {
      const int i = e / T, j = e - (e / T) * T;
      const float* cf = c.psf_coefs + (((size_t)b * T + i) * T + j) * c.nt;
      float v0 = 0.f, v1 = 0.f, v2 = 0.f;
      for (int tt = 0; tt < c.nt; ++tt) {
        const float cv = cf[tt];
        v0 = fmaf(cv, rec->beta[tt], v0);
        v1 = fmaf(cv, rec->betax[tt], v1);
        v2 = fmaf(cv, rec->betay[tt], v2);
      }
      img[e] = v0;
      img[TT + e] = v1;
      img[2 * TT + e] = v2;
      K[e] = (double)v0;
    }
    const float* pm = Pp + (size_t)isl * c.nP + 6 * k;
    const double lr = (double)pm[2], e1 = (double)pm[3], e2 = (double)pm[4];
    float* out = c.gstamp + (size_t)item * 7 * TT;
    // the stamp
    direct_profile(c, T, lr, e1, e2, I, red);
    const double tot0 = direct_conv(K, I, T, C, red);
    for (int e = tid; e < TT; e += GT) {
      const double v = tot0 > 0.0 ? C[e] / tot0 : C[e];
      S0[e] = v;
      out[e] = (float)v;
    }
    __syncthreads();
    // position partials through the PSF's variation (profile in I)
    for (int q = 1; q <= 2; ++q) {
      if (!need[q]) continue;
      for (int e = tid; e < TT; e += GT) K[e] = (double)img[q * TT + e];
      __syncthreads();
      const double sd = direct_conv(K, I, T, C, red);
      for (int e = tid; e < TT; e += GT)
        out[(size_t)q * TT + e] = tot0 > 0.0 ? (float)((C[e] - S0[e] * sd) / tot0) : 0.f;
      __syncthreads();
    }
    // shape partials by central differences of the stamp
    if (need[3] || need[4] || need[5]) {
      for (int e = tid; e < TT; e += GT) K[e] = (double)img[e];
      __syncthreads();
      for (int j = 0; j < 3; ++j) {
        if (!need[3 + j]) continue;
        for (int sg = 0; sg < 2; ++sg) {
          const double hh = sg == 0 ? DIRECT_FD_STEP : -DIRECT_FD_STEP;
          direct_profile(c, T, lr + (j == 0 ? hh : 0.0), e1 + (j == 1 ? hh : 0.0),
                         e2 + (j == 2 ? hh : 0.0), I, red);
          const double t = direct_conv(K, I, T, C, red);
          for (int e = tid; e < TT; e += GT) {
            const double v = t > 0.0 ? C[e] / t : C[e];
            if (sg == 0)
              Sp[e] = v;
            else
              out[(size_t)(3 + j) * TT + e] = (float)((Sp[e] - v) / (2.0 * DIRECT_FD_STEP));
          }
          __syncthreads();
        }
      }
    }
    if (need[6])
      for (int e = tid; e < TT; e += GT) out[(size_t)6 * TT + e] = 0.f;
  }
}

}  // namespace

size_t gal_direct_floats(int T) {
  return align64(3 * (size_t)T * T) + 6 * (size_t)T * T + 64;
}

int gal_direct_smem(int T) { return (int)(2 * sizeof(double) * (size_t)T * T); }

int fft_pad_for(int T) {
  int n = 1;
  while (n < T + T / 2) n <<= 1;
  return n;
}

int gal_fft_smem(int T, int P) {
  const int lines = std::max(P / 2 + 1, T);
  return 8 * P * std::min(lines, FFT_SMEM_MAX / (8 * P));
}

int gal_fft_setup() {
  cudaError_t e = cudaFuncSetAttribute(k_gal_fft, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       FFT_SMEM_MAX);
  if (e != cudaSuccess) return (int)e;
  return (int)cudaFuncSetAttribute(k_gal_direct, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   gal_direct_smem(UPH_DIRECT_MAX_T));
}

size_t gal_fft_floats(int T, int P) {
  const size_t H = (size_t)P / 2 + 1;
  // img, R (complex), X (3 complex), Fs (3 real), Cc (complex), each aligned
  return align64(3 * (size_t)T * T) + align64(2 * (size_t)T * H) + 6 * (size_t)P * H +
         align64(3 * (size_t)P * H) + align64(2 * (size_t)T * H) + 64;
}

void launch_gal_fft(const ClassDev& c, const float* P, int phase, cudaStream_t s) {
  if (c.gfft_ctas > 0 && c.gdirect)
    k_gal_direct<<<(unsigned)c.gfft_ctas, GT, (size_t)c.gfft_smem, s>>>(c, P, phase);
  else if (c.gfft_ctas > 0)
    k_gal_fft<<<(unsigned)c.gfft_ctas, GT, (size_t)c.gfft_smem, s>>>(c, P, phase);
}

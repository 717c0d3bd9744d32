// Internal device-side descriptors and helpers of the uniphot_b200 solver.
//
// Layout in HBM (one solver class, one chunk of n_isl islands):
//   field stacks   dstack/wstack          (nb, Hp, Wp) f32, read in place
//   stamps         (n_isl, nb, N, R, Sz*Sz) f32 -- member m and d m/d theta
//                  on the member's footprint box clipped to the window
//   gram           (n_isl, nb, Kmax*Kmax) f32 -- weighted Gram of the rows
//                  [dM/dtheta (nL); M (nr); data (1)]
//   Hb, gb         (n_isl, nb, nLmax^2), (n_isl, nb, nLmax) f32 -- per-band
//                  Gauss-Newton blocks of the VarPro residual
//   H, g           (n_isl, nLmax^2), (n_isl, nLmax) f32 -- band sums
//   chi2b          (n_isl, nb) f64, flux/ferr (n_isl, nb, N) f32
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define UPH_MAXN 32          // member slots per island handled on the device
#define UPH_MAXLIVE 192      // live nonlinear parameters per island
#define UPH_MAXBG 3           // planar background rows (1, X, Y) per band
#define UPH_MAXLIN (UPH_MAXN + UPH_MAXBG)   // linear unknowns per band
#define UPH_MAXK (UPH_MAXLIVE + UPH_MAXLIN + 1)
#define UPH_LU_SMEM_N 160    // damped systems up to this size factor in shared memory
#define UPH_MAXKPSF 8        // Gaussian components of an analytic PSF
#define UPH_MAXNT 21         // polynomial terms (order 5)
#define UPH_MAXGAL 16        // Sersic table components + delta core
#define UPH_TILE 32          // render output tile side
#define UPH_HALO (UPH_TILE + 6)

// island flag bits
#define FL_CONV 1
#define FL_STALL 2
#define FL_NEEDLIN 4
#define FL_PROBE 8
#define FL_REAL 16           // a real island (chunk rows are all real)

// kernel phases
#define PH_LIN 0      // linearisation at p of islands that need it
#define PH_TRIAL 1    // trial point of every non-converged island
#define PH_PROBE 2    // post-hoc probes of stalled islands
#define PH_ALL 3      // every island (initial chi2, final fluxes)

// One Gaussian term of an analytic member stamp: PSF component q convolved
// with galaxy component g (covariances add), with what the derivative
// stamps need.
struct GComp {
  float ia, ib, ic;          // inverse covariance
  float A, B, C, det;        // covariance xx, xy, yy; det holds 0.5/det
  float nrm, nx, ny, nu;     // weight * amplitude / (2 pi sqrt det) (+ d/dx, d/dy, d/dn)
  float v, dv;               // galaxy variance scale and d v / d n
  float dAx, dBx, dCx, dAy, dBy, dCy;
};

// Per (island, band, member) render set-up at the current parameters,
// computed once by k_member_setup and read by every render tile.
struct MemberRecord {
  float Lx[7], dLx[7], Ly[7], dLy[7];            // Lanczos taps, d/d shift
  float beta[UPH_MAXNT], betax[UPH_MAXNT], betay[UPH_MAXNT];  // PSF basis
  float dcov[3][3];                              // d(cxx,cyy,cxy)/d(lr,e1,e2)
  float cg[3];                                   // unit galaxy covariance
  float dndu;
  int ncomp;
  GComp comps[UPH_MAXKPSF * UPH_MAXGAL];
  // reference render mode, galaxies: the Sersic mixture at the member's
  // index (amplitude, variance in units of the galaxy covariance, their
  // derivatives in n; the zero-variance core apart), for the Fourier-
  // domain convolution with the pixelised PSF
  int ngal;
  double ga[UPH_MAXGAL], gv[UPH_MAXGAL], gda[UPH_MAXGAL], gdv[UPH_MAXGAL];
  double gcore, gdcore;
};

struct ClassDev {
  int n_isl, nb, N, nP, B, T, Sz, R, Kmax, nLmax, ntile_side;
  int mode, nt, kpsf, psf_varies;
  int native;              // star support side (odd, <= T)
  int has_gal;             // some member of the chunk is extended
  int Hp, Wp;
  const float* dstack;
  const float* wstack;
  const float* psf_coefs;  // (nb, T, T, nt)
  const float* psf_os;     // (nb, 4)
  const float* mog;        // (nb, kpsf, 4, nt)
  const double* tb_knots;
  const double* tb_amps;
  const double* tb_lv;
  const double* tb_core;
  int tb_n, tb_k;
  double tb_nmin, tb_nmax;
  const int* ox;
  const int* oy;
  const float* x0b;
  const float* y0b;
  const int* stype;
  const float* n_frozen;
  const uint8_t* free_n;
  const uint8_t* mmask;
  const uint8_t* keep;
  const float* lower;
  const float* upper;
  const float* prior_mean;
  const float* prior_inv;
  int has_priors;
  const int* isl_nL;       // live parameters per island
  const int* isl_nr;       // real members per island (slots 0..nr-1)
  const int16_t* row_k;    // (n_isl, Kmax) member slot of Gram row
  const int16_t* row_s;    // stamp row (0 = model, >0 derivative, -1 data)
  const int16_t* row_p;    // parameter index 6k+j of derivative rows
  float* p;
  float* p_try;
  float* lam;
  float* chi2;
  int* consec;
  int* nrej;
  int* nst;
  uint8_t* flags;
  float* stamps;
  MemberRecord* mrec;      // (n_isl, nb, N)
  float* gram;
  float* Hb;
  float* gb;
  float* H;
  float* g;
  double* lu;
  double* chi2b;
  float* flux;
  float* ferr;
  int* ngood;
  // Fluxes solved at p (fcur) and at p_try (ftry), (n_isl, nb, N); only
  // allocated when some island uses the tensor-core Gram, whose last row is
  // the residual d - M^T fcur instead of the data.
  // Linear solution per band: nr member fluxes, then nbg background
  // coefficients (nbg = 3 when the planar background is solved jointly,
  // else 0); arrays of it have stride NL = N + nbg.
  int nbg;
  int NL;
  // "changed" stall counting: identical-proposal reject runs (n_same), the
  // last rejected proposal (prej, n_isl x nP) and the sticky diverged flag
  int changed;
  // convergence "dlnp": chi2 carried in float64 (chi2d), absolute
  // sub-quantum prongs (quantum = 2 plateau_dlnp_tol), reject-exits at the
  // lam cap or on a no-move proposal; implies the "changed" counting
  int dlnp;
  float quantum;
  double* chi2d;
  int* n_same;
  float* prej;
  uint8_t* div_live;
  // trust-region step: the radius lives in lam; k_step leaves per island
  // (predicted gain, radius used, radius cap, step reached the boundary)
  // in trs for k_accept's radius update
  int tr;
  double* trs;             // (n_isl, 4)
  // marginal covariance at the final parameters (param_errors): output
  // (n_isl, N, 13), float64 work space for the inversion (n_isl, nLmax,
  // 2 nLmax) and the flags saved around the relinearisation
  float* perr;
  double* ews;
  uint8_t* flsave;
  // shape-marginalised flux variance (flux_marg): the flux sensitivities
  // d f / d theta of the relinearisation, (n_isl, nb, nLmax, UPH_MAXLIN),
  // written by k_assemble only when non-null, and the output (n_isl, nb, N)
  float* cjac;
  float* femarg;
  // source metrics (source_metrics): per (island, band, member) moments
  // (n_isl, nb, N, 5), combined metrics (n_isl, N, 4), window fluxes
  // (n_isl, nb, N)
  double* smom;
  float* smet;
  float* swin;
  // Re profile (n_isl, N, 12) chi2 differences; band-coadded residual and
  // weight (n_isl, B, B)
  float* reprof;
  float* resid;
  float* resid_w;
  // reference render mode with galaxies: the unshifted galaxy stamp and its
  // partials (S, Sx, Sy, S_lr, S_e1, S_e2, S_u) per (island, band, member),
  // (n_isl, nb, N, 7, T, T), from the Fourier-domain convolution; its work
  // space per resident CTA (gfft_ctas of gfft_floats floats); the pad size;
  // the shared line buffer's bytes (gal_fft_smem)
  int fft_P;
  int gfft_ctas;
  int gfft_smem;
  size_t gfft_floats;
  // the legacy "direct" backend instead of the Fourier-domain convolution
  // (EXP members only): its exponential mixture
  int gdirect;
  int exp_k;
  const float* exp_amp;
  const float* exp_var;
  float* gstamp;
  float* gfft_ws;
  float* bgout;            // (n_isl, nb, 3) final background coefficients
  float* bgerr;            // (n_isl, nb, 3) and their errors
  float* fcur;
  float* ftry;
  // (n_isl, nb) conditioning indicator of the members' scaled normal matrix
  // at p (acond_cur) and p_try (acond_try), from the trial pass's f64
  // elimination; an island whose indicator exceeds tc_cond_max in any band
  // forms its Gram in FP32
  float* acond_cur;
  float* acond_try;
  float tc_cond_max;
  float* probe_best;       // (n_isl) plateau certificate
  float* probe_p;          // (n_isl, 4, nP) diverged-probe proposals
  int* n_active;
  int* err;                // device error flag: 1 a bounded wait expired,
                           // 2 a launch had too little shared memory
  // (WK_KINDS, WK_FIELDS) algorithmic bytes, flops and exponentials per
  // kernel kind, added by every
  // working CTA; non-null only during instrumented solves
  unsigned long long* work;
  int tc_min_rows;         // islands with more Gram rows use the tensor-core Gram
  int tc_split;            // CTAs per (island, band) of the tensor-core Gram,
                           // each over a contiguous range of pixel chunks
  float* gpart;            // (tc_split, n_isl, nb, Kmax, Kmax) partial Grams
                           // (tc_split > 1), summed in split order
  int gl_split;            // CTAs per (island, band, block set) of the FP32
                           // Gram, each over a contiguous range of pixel tiles
                           // (a function of the window side only)
  float* glpart;           // (gl_split, n_isl, nb, Kmax, Kmax) its partial
                           // Grams (gl_split > 1), summed in split order
  float reg, pos_step_max, ftol_rel, step_tol;
  int un_freeze;
};

// Gram rows of island isl: live derivative rows, member model rows,
// background rows, the data (or residual) row.
__device__ __forceinline__ int gram_K(const ClassDev& c, int isl) {
  return c.isl_nL[isl] + c.isl_nr[isl] + c.nbg + 1;
}

// Planar background basis j (0: 1, 1: X, 2: Y) at window pixel (wy, wx):
// X = (wx - c) / s, Y = (wy - c) / s with c = (B - 1) / 2 and s = B / 2,
// evaluated in double and rounded once.
__device__ __forceinline__ float bg_basis(int j, int wy, int wx, int B) {
  if (j == 0) return 1.0f;
  const double cen = 0.5 * (B - 1), sc = 0.5 * B;
  return (float)(((double)(j == 1 ? wx : wy) - cen) / sc);
}

// Whether island isl forms its next Gram on the tensor cores (mixed form):
// more than tc_min_rows rows and a well-conditioned normal matrix of its
// members in every band.  k_gram_lin, k_gram_tc and k_assemble take the same
// decision from the same data.
__device__ __forceinline__ bool tc_island(const ClassDev& c, int isl, int K) {
  if (K <= c.tc_min_rows) return false;
  const float* a = c.acond_cur + (size_t)isl * c.nb;
  for (int b = 0; b < c.nb; ++b)
    if (!(a[b] <= c.tc_cond_max)) return false;
  return true;
}

// Kernel kinds of the instrumented solve (uph_job_kernel_time numbering).
enum { WK_RENDER = 0, WK_GRAM = 1, WK_ASSEMBLE = 2, WK_STEP = 3, WK_TRIAL = 4,
       WK_ACCEPT = 5, WK_GRAM_TC = 6, WK_KINDS = 7 };
// Per kind: algorithmic bytes, floating-point operations (tensor-core or
// FP32 CUDA-core, by kind) and exponential evaluations (SFU).
constexpr int WK_FIELDS = 3;

__device__ __forceinline__ void work_add(const ClassDev& c, int kind,
                                         unsigned long long bytes,
                                         unsigned long long flops,
                                         unsigned long long exps = 0) {
  if (c.work) {
    atomicAdd(c.work + WK_FIELDS * kind, bytes);
    if (flops) atomicAdd(c.work + WK_FIELDS * kind + 1, flops);
    if (exps) atomicAdd(c.work + WK_FIELDS * kind + 2, exps);
  }
}

// Algorithmic work of one (island, band) Gram of K rows: every stamp row
// read over its member's box, data and weights over the window, the K x K
// result written; K (K + 1) flops per pixel (upper triangle, multiply-add).
__device__ __forceinline__ void gram_work(const ClassDev& c, int kind,
                                          const int16_t* rk, const int16_t* rs,
                                          int K, const int4* box) {
  if (!c.work) return;
  unsigned long long px = 0;
  for (int r = 0; r < K; ++r) {
    if (rs[r] < 0) continue;
    const int4 bx = box[rk[r]];
    px += (unsigned long long)max(bx.z, 0) * (unsigned long long)max(bx.w, 0);
  }
  const unsigned long long npix = (unsigned long long)c.B * c.B;
  work_add(c, kind, 4ull * (px + 2 * npix + (unsigned long long)K * K),
           (unsigned long long)K * (K + 1) * npix);
}

__device__ __forceinline__ bool isl_active(uint8_t fl, int phase) {
  switch (phase) {
    case PH_LIN: return !(fl & FL_CONV) && (fl & FL_NEEDLIN);
    case PH_TRIAL: return !(fl & FL_CONV);
    case PH_PROBE: return (fl & FL_PROBE) != 0;
    default: return true;
  }
}

// Stamp placement of member k at parameters P: the window box of its
// footprint.  Positions are float32 as in the reference; rint is
// round-half-to-even like jnp.round.
struct MemberBox {
  int ixt, iyt;      // stamp top-left in window coordinates
  int wx0, wy0;      // clipped box origin in the window
  int bw, bh;        // clipped box size (<= Sz), may be <= 0
  float dx, dy;      // fractional shift
};

__device__ __forceinline__ MemberBox member_box(const ClassDev& c, int isl,
                                                const float* P, int k) {
  MemberBox mb;
  const float x = P[(size_t)isl * c.nP + 6 * k];
  const float y = P[(size_t)isl * c.nP + 6 * k + 1];
  const float gx = __fsub_rn(x, c.x0b[isl]);
  const float gy = __fsub_rn(y, c.y0b[isl]);
  const float rx = rintf(gx);
  const float ry = rintf(gy);
  mb.dx = __fsub_rn(gx, rx);
  mb.dy = __fsub_rn(gy, ry);
  mb.ixt = (int)rx - c.T / 2;
  mb.iyt = (int)ry - c.T / 2;
  mb.wx0 = max(mb.ixt, 0);
  mb.wy0 = max(mb.iyt, 0);
  mb.bw = min(mb.ixt + c.T, c.B) - mb.wx0;
  mb.bh = min(mb.iyt + c.T, c.B) - mb.wy0;
  return mb;
}

__device__ __forceinline__ size_t stamp_slot(const ClassDev& c, int isl, int b,
                                             int k, int row) {
  return ((((size_t)isl * c.nb + b) * c.N + k) * c.R + row) *
         (size_t)(c.Sz * c.Sz);
}

__device__ inline void lanczos_taps(double d, float* L, float* dL) {
  double v[7], dv[7], s = 0.0, ds = 0.0;
  const double pi = 3.141592653589793;
  for (int t = 0; t < 7; ++t) {
    double x = (double)(t - 3) + d;
    double ax = fabs(x);
    if (ax < 1e-12) {
      v[t] = 1.0;
      dv[t] = 0.0;
    } else if (ax >= 3.0) {
      v[t] = 0.0;
      dv[t] = 0.0;
    } else {
      double px = pi * x;
      double s1, c1, s3, c3;
      sincos(px, &s1, &c1);
      sincos(px / 3.0, &s3, &c3);
      v[t] = 3.0 * s1 * s3 / (px * px);
      dv[t] = 3.0 * (pi * c1 * s3 + (pi / 3.0) * s1 * c3) / (px * px) -
              6.0 * s1 * s3 / (pi * pi * x * x * x);
    }
    s += v[t];
    ds += dv[t];
  }
  for (int t = 0; t < 7; ++t) {
    L[t] = (float)(v[t] / s);
    dL[t] = (float)((dv[t] * s - v[t] * ds) / (s * s));
  }
}

// polynomial term exponents, low order first
__device__ __forceinline__ void term_mn(int t, int& m, int& n) {
  int deg = 0, start = 0;
  while (start + deg + 1 <= t) {
    start += deg + 1;
    ++deg;
  }
  n = t - start;
  m = deg - n;
}

// Per-grid sparse forced photometry of one band (uph_sparse.cu): inputs,
// per-source work and the float64 system [A | I | b] in device memory.
struct SparseDev {
  int n, H, W, nterms, M, h, w, gx0, gy0, renorm, kmax, nparts;
  float reg;
  const float* coefs;      // (H, W, nterms)
  const float* os;         // x_origin, x_scale, y_origin, y_scale
  const float* px;
  const float* py;
  const float* data;       // (h, w)
  const float* invvar;
  const uint8_t* good;
  const int* nidx;         // (n, kmax)
  const uint8_t* nmask;
  const double* bn;        // background x_origin, x_scale, y_origin, y_scale
  float* wgrid;            // invvar where good, else 0
  float* stamps;           // (n, H, W)
  int* ixt;
  int* iyt;
  float* diag;
  float* twd;
  float* twb;              // (n, M)
  float* off;              // (n, kmax)
  double* part;            // (nparts, M*M + M)
  float* Af;               // (n + M)^2
  double* G;               // (n + M, 2 (n + M) + 1)
  int* prow;
  float* x;                // solution (n + M)
  float* var;              // diagonal of the inverse (n + M)
  // extended sources ("fft" backend): per-source type and shape (stype
  // null: all stars), the Sersic table, the unshifted galaxy stamps and
  // the Fourier work space (gal_ctas CTAs of gal_floats floats, pad fft_P)
  const int* stype;
  const float* lr;
  const float* e1;
  const float* e2;
  const float* sn;
  const double* tb_knots;
  const double* tb_amps;
  const double* tb_lv;
  const double* tb_core;
  int tb_n, tb_k;
  double tb_nmin, tb_nmax;
  int fft_P, gal_ctas;
  size_t gal_floats;
  float* gal;
  float* gws;
  // "direct" backend: EXP stamps from the exp_k-Gaussian mixture (amp, var)
  int direct, exp_k;
  const float* exp_mog;    // amp[exp_k] then var[exp_k]
};
size_t sparse_stamp_smem(int H, int W);
size_t sparse_gal_floats(int H, int W, int P);
int sparse_setup();
void launch_sparse_band(const SparseDev& d, cudaStream_t s);

// Device island decomposition (uph_islands.cu).
struct IslandDev {
  int n, ncx, ncy;
  int tries;               // unite attempts per coupled pair before giving up
  double x0, y0, cell;
  const double* x;
  const double* y;
  const double* r;
  const uint8_t* single;   // forced singletons (nullable)
  int* cid;                // (n) cell of each source
  int* count;              // (ncx * ncy)
  int* start;              // (ncx * ncy + 1)
  int* cursor;             // (ncx * ncy)
  int* bucket;             // (n) sources by cell
  int* parent;             // (n) union-find
  int* root;               // (n) minimum member index of the component
  int* err;
};
void launch_island_roots(const IslandDev& d, cudaStream_t s);

// Ellipse (logre, ee1, ee2) -> unit covariance and its Jacobian
// (sersic_mog.py:108-150, incl. the round-source nudge).
__device__ inline void cov_terms(double lr, double e1, double e2, float* cg,
                          float dc[3][3]) {
  double ex = exp(lr);
  double re = fmin(fmax(ex, 0.1), 1000.0);
  double dre = (ex > 0.1 && ex < 1000.0) ? re : 0.0;
  bool nudge = (e1 == 0.0) && (e2 == 0.0);
  double e1n = nudge ? 1e-4 : e1;
  double de1n = nudge ? 0.0 : 1.0;
  double ee = hypot(e1n, e2);
  double dee1 = e1n / ee * de1n, dee2 = e2 / ee;
  double ex2 = exp(-ee);
  double e = 1.0 - ex2;
  double den = 1.0 - e, dden = -1.0;
  if (!(den > 1e-4)) {
    den = 1e-4;
    dden = 0.0;
  }
  double ibr = (1.0 + e) / den;
  double dibr = (den - (1.0 + e) * dden) / (den * den);
  double ib = ibr, dib = dibr;
  if (!(ibr < 1000.0)) {
    ib = 1000.0;
    dib = 0.0;
  }
  double th = 0.5 * atan2(e2, e1n);
  double dth1 = -0.5 * e2 / (ee * ee) * de1n, dth2 = 0.5 * e1n / (ee * ee);
  double st, ct;
  sincos(th, &st, &ct);
  double s2 = 1.0 / (ib * ib);
  double r2 = re * re;
  cg[0] = (float)(r2 * (ct * ct * s2 + st * st));
  cg[1] = (float)(r2 * (st * st * s2 + ct * ct));
  cg[2] = (float)(r2 * ct * st * (1.0 - s2));
  double d_re[3] = {2 * re * (ct * ct * s2 + st * st),
                    2 * re * (st * st * s2 + ct * ct),
                    2 * re * ct * st * (1.0 - s2)};
  double ib3 = ib * ib * ib;
  double d_ib[3] = {r2 * ct * ct * (-2.0 / ib3), r2 * st * st * (-2.0 / ib3),
                    r2 * ct * st * (2.0 / ib3)};
  double d_th[3] = {2 * r2 * ct * st * (1.0 - s2),
                    -2 * r2 * ct * st * (1.0 - s2),
                    r2 * (ct * ct - st * st) * (1.0 - s2)};
  double dib_dee = dib * ex2;
  for (int q = 0; q < 3; ++q) {
    dc[0][q] = (float)(d_re[q] * dre);
    dc[1][q] = (float)(d_ib[q] * dib_dee * dee1 + d_th[q] * dth1);
    dc[2][q] = (float)(d_ib[q] * dib_dee * dee2 + d_th[q] * dth2);
  }
}

// 2 pi^2: the Gaussian Fourier exponent exp(-2 pi^2 k^T C k)
constexpr double UPH_TWO_PI2 = 19.739208802178716;

// Segment, interpolation weight and its derivative in n of the Sersic
// mixture table at index n (the piecewise-linear interpolant of
// sersic_mog.py:81-100); the index is clamped to the table's range, where
// the derivative is 0.
__device__ inline void sersic_segment(const double* knots, int nk, double nmin, double nmax,
                                      double n, int* seg, double* t, double* dt) {
  const bool inside = (n > nmin) && (n < nmax);
  const double nc = fmin(fmax(n, nmin), nmax);
  int lo = 0, hi = nk;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (knots[mid] <= nc) lo = mid + 1; else hi = mid;
  }
  const int s = max(0, min(lo - 1, nk - 2));
  const double n0 = knots[s], n1 = knots[s + 1];
  *seg = s;
  *t = (n1 > n0) ? (nc - n0) / (n1 - n0) : 0.0;
  *dt = (n1 > n0 && inside) ? 1.0 / (n1 - n0) : 0.0;
}

// ---- Shared-memory radix-2 FFTs for the Fourier-domain galaxy stamps ----
// In-place decimation-in-time FFTs of nl lines of length P = 2^logP stored
// contiguously in shared memory; sign -1 forward, +1 inverse (unnormalised);
// cw/sw hold cos and sin of 2 pi m / P.  The callers fill each line in
// bit-reversed order (fft_brev), so the transform starts at the butterflies.
// Two consecutive stages (half-lengths h and 2h) run as one pass: a thread
// takes the four elements j, j+h, j+2h, j+3h of a group of 4h and applies
// both stages' butterflies with the stages' own twiddles, which halves the
// barriers and shared-memory round trips; an odd last stage runs alone.
// Ends with a barrier.
__device__ inline int fft_brev(int k, int logP) {
  return (int)(__brev((unsigned)k) >> (32 - logP));
}

// Lines per pass when L lines go through a buffer of lb lines: the passes
// split L evenly (65 columns in buffers of 64 lines take 33 + 32, not 64 + 1).
__device__ inline int fft_pass_lines(int L, int lb) {
  const int np = (L + lb - 1) / lb;
  return (L + np - 1) / np;
}

__device__ inline void fft_bfly(float2& u, float2& v, float wr, float wi) {
  const float tr = wr * v.x - wi * v.y, ti = wr * v.y + wi * v.x;
  const float2 a = u;
  u = make_float2(a.x + tr, a.y + ti);
  v = make_float2(a.x - tr, a.y - ti);
}

__device__ inline void smem_fft_lines(float2* buf, int nl, int P, int logP, float sign,
                                      const float* cw, const float* sw) {
  const int tid = threadIdx.x, nth = blockDim.x;
  int h = 1;
  for (; 4 * h <= P; h <<= 2) {
    const int q = P >> 2;                      // four-element groups per line
    const int sA = P / (2 * h), sB = P / (4 * h);
    for (int e = tid; e < nl * q; e += nth) {
      const int line = e / q, b = e - line * q;
      const int grp = b / h, j = b - grp * h;
      const int i0 = (line << logP) + grp * 4 * h + j;
      float2 x0 = buf[i0], x1 = buf[i0 + h], x2 = buf[i0 + 2 * h], x3 = buf[i0 + 3 * h];
      const int mA = j * sA;
      fft_bfly(x0, x1, cw[mA], sign * sw[mA]);
      fft_bfly(x2, x3, cw[mA], sign * sw[mA]);
      const int mB0 = j * sB, mB1 = (j + h) * sB;
      fft_bfly(x0, x2, cw[mB0], sign * sw[mB0]);
      fft_bfly(x1, x3, cw[mB1], sign * sw[mB1]);
      buf[i0] = x0;
      buf[i0 + h] = x1;
      buf[i0 + 2 * h] = x2;
      buf[i0 + 3 * h] = x3;
    }
    __syncthreads();
  }
  if (2 * h == P) {
    const int hp = P >> 1, step = P / (2 * h);
    for (int e = tid; e < nl * hp; e += nth) {
      const int line = e / hp, b = e - line * hp;
      const int grp = b / h, j = b - grp * h;
      const int i0 = (line << logP) + grp * 2 * h + j;
      float2 u = buf[i0], v = buf[i0 + h];
      const int m = j * step;
      fft_bfly(u, v, cw[m], sign * sw[m]);
      buf[i0] = u;
      buf[i0 + h] = v;
    }
    __syncthreads();
  }
}

// Forward 2-D transform of an Hs x Ws real image zero-padded to P x P:
// X (P x Hf, Hf = P/2 + 1) from row transforms R (Hs x Hf) and column
// transforms; buf holds lb lines of P in shared memory.
__device__ inline void fft2_forward(const float* img, int Hs, int Ws, int P, int logP,
                                    float2* R, float2* X, float2* buf, int lb,
                                    const float* cw, const float* sw) {
  const int tid = threadIdx.x, nth = blockDim.x, Hf = P / 2 + 1;
  const int lr = fft_pass_lines(Hs, lb), lc = fft_pass_lines(Hf, lb);
  for (int i0 = 0; i0 < Hs; i0 += lr) {
    const int nl = min(lr, Hs - i0);
    for (int e = tid; e < nl * P; e += nth) {
      const int line = e >> logP, k = e & (P - 1);
      buf[(line << logP) + fft_brev(k, logP)] =
          make_float2(k < Ws ? img[(i0 + line) * Ws + k] : 0.f, 0.f);
    }
    __syncthreads();
    smem_fft_lines(buf, nl, P, logP, -1.f, cw, sw);
    for (int e = tid; e < nl * Hf; e += nth) {
      const int line = e / Hf, u = e - line * Hf;
      R[(size_t)(i0 + line) * Hf + u] = buf[(line << logP) + u];
    }
    __syncthreads();
  }
  for (int u0 = 0; u0 < Hf; u0 += lc) {
    const int nl = min(lc, Hf - u0);
    for (int e = tid; e < nl * P; e += nth) {
      const int k = e / nl, line = e - k * nl;
      buf[(line << logP) + fft_brev(k, logP)] =
          k < Hs ? R[(size_t)k * Hf + u0 + line] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    smem_fft_lines(buf, nl, P, logP, -1.f, cw, sw);
    for (int e = tid; e < nl * P; e += nth) {
      const int w = e / nl, line = e - w * nl;
      X[(size_t)w * Hf + u0 + line] = buf[(line << logP) + w];
    }
    __syncthreads();
  }
}

// Inverse column transforms of Q = Xb * fac (fac real, P x Hf; times the
// shape factor -2 pi^2 (d0 nu^2 + d1 nw^2 + 2 d2 nu nw) when dexpo), rows
// below Hs kept in C (Hs x Hf).
__device__ inline void fft2_inverse_cols(const float2* Xb, const float* fac, bool dexpo,
                                         float d0, float d1, float d2, int Hs, int P, int logP,
                                         float2* C, float2* buf, int lb, const float* cw,
                                         const float* sw) {
  const int tid = threadIdx.x, nth = blockDim.x, Hf = P / 2 + 1;
  const int lc = fft_pass_lines(Hf, lb);
  for (int u0 = 0; u0 < Hf; u0 += lc) {
    const int nl = min(lc, Hf - u0);
    for (int e = tid; e < nl * P; e += nth) {
      const int w = e / nl, line = e - w * nl, u = u0 + line;
      float f = fac[(size_t)w * Hf + u];
      if (dexpo) {
        const float nu = (float)u / (float)P;
        const float nw = (float)(w < P / 2 ? w : w - P) / (float)P;
        f *= -(float)UPH_TWO_PI2 * (d0 * nu * nu + d1 * nw * nw + 2.f * d2 * nu * nw);
      }
      const float2 x = Xb[(size_t)w * Hf + u];
      buf[(line << logP) + fft_brev(w, logP)] = make_float2(f * x.x, f * x.y);
    }
    __syncthreads();
    smem_fft_lines(buf, nl, P, logP, 1.f, cw, sw);
    for (int e = tid; e < nl * Hs; e += nth) {
      const int i = e / nl, line = e - i * nl;
      C[(size_t)i * Hf + u0 + line] = buf[(line << logP) + i];
    }
    __syncthreads();
  }
}

// Inverse row transforms (real output) of C (Hs x Hf, the half spectrum;
// the imaginary parts of the zero and Nyquist bins are dropped as a real
// inverse does), scaled by 1/P^2 and cropped to Hs x Ws, into out.
__device__ inline void fft2_inverse_rows(const float2* C, int Hs, int Ws, int P, int logP,
                                         float* out, float2* buf, int lb, const float* cw,
                                         const float* sw) {
  const int tid = threadIdx.x, nth = blockDim.x, Hf = P / 2 + 1;
  const float inv = 1.f / ((float)P * (float)P);
  const int lr = fft_pass_lines(Hs, lb);
  for (int i0 = 0; i0 < Hs; i0 += lr) {
    const int nl = min(lr, Hs - i0);
    for (int e = tid; e < nl * P; e += nth) {
      const int line = e >> logP, k = e & (P - 1);
      const float2* ci = C + (size_t)(i0 + line) * Hf;
      float2 v;
      if (k == 0) v = make_float2(ci[0].x, 0.f);
      else if (k == P / 2) v = make_float2(ci[Hf - 1].x, 0.f);
      else if (k < P / 2) v = ci[k];
      else v = make_float2(ci[P - k].x, -ci[P - k].y);
      buf[(line << logP) + fft_brev(k, logP)] = v;
    }
    __syncthreads();
    smem_fft_lines(buf, nl, P, logP, 1.f, cw, sw);
    for (int e = tid; e < nl * Ws; e += nth) {
      const int line = e / Ws, j = e - line * Ws;
      out[(i0 + line) * Ws + j] = buf[(line << logP) + j].x * inv;
    }
    __syncthreads();
  }
}

// Kernel launch wrappers (defined in the .cu units).
void launch_render(const ClassDev& c, const float* P, int phase,
                   cudaStream_t s);
int fft_pad_for(int T);
size_t gal_fft_floats(int T, int P);
int gal_fft_smem(int T, int P);
int gal_fft_setup();
size_t gal_direct_floats(int T);
void launch_star_stamps(int n, int H, int W, const float* coefs, int nt, const float* os,
                        const float* px, const float* py, float* out, int* ixt, int* iyt,
                        cudaStream_t s);
void launch_scene_sub_wave(float* stack, int Hp, int Wp, int pad, int T, const int* srcs,
                           int count, const float* stamps, const int* ixt, const int* iyt,
                           const float* flux, cudaStream_t s);
void launch_tile_bg_subtract(float* stack, int nb, int Hp, int Wp, int pad, int x0, int y0,
                             int w, int h, const float* coefs, int M, const double* norm,
                             int sms, cudaStream_t s);
int gal_direct_smem(int T);
void launch_gal_fft(const ClassDev& c, const float* P, int phase, cudaStream_t s);
void launch_gram_lin(const ClassDev& c, cudaStream_t s);
void launch_assemble(const ClassDev& c, cudaStream_t s);
void launch_gram_trial(const ClassDev& c, const float* P, int phase,
                       int final_mode, float* fout, float* cout, cudaStream_t s);
void launch_step(const ClassDev& c, int phase, int probe_j, float probe_lam,
                 int use_lam_final_scale, cudaStream_t s);
void launch_accept(const ClassDev& c, int phase, cudaStream_t s);
void launch_count_active(const ClassDev& c, cudaStream_t s);
void launch_diverged_compare(const ClassDev& c, uint8_t* out,
                             cudaStream_t s);
void launch_railed(const ClassDev& c, uint8_t* out, cudaStream_t s);
void launch_errors_begin(const ClassDev& c, cudaStream_t s);
void launch_final_errors(const ClassDev& c, cudaStream_t s);
void launch_flux_marg(const ClassDev& c, cudaStream_t s);
void launch_source_metrics(const ClassDev& c, cudaStream_t s);
void launch_copy_windows(const ClassDev& c, const float* fd, const float* fw, int fHp, int fWp,
                         const int* ox_f, const int* oy_f, cudaStream_t s);
void launch_addback(const ClassDev& c, const float* seed, const float* msf, cudaStream_t s);
void launch_residual_coadd(const ClassDev& c, cudaStream_t s);
void launch_reprof_set(const ClassDev& c, int n, int j, float dk, cudaStream_t s);
void launch_reprof_store(const ClassDev& c, int n, int j, cudaStream_t s);
void launch_errors_end(const ClassDev& c, cudaStream_t s);
size_t render_smem_bytes();
size_t gram_lin_smem_bytes(int Kmax);
size_t gram_trial_smem_bytes(int N);
size_t assemble_smem_bytes(int nLmax, int N);
size_t step_smem_bytes(int nLmax);
void launch_gram_tc(const ClassDev& c, cudaStream_t s);
size_t gram_tc_smem_bytes(int kmax);
int gram_tc_splits(int n_isl, int nb, int B, int sm_count);
int uph_kernel_setup();

// Compute-pipe peak kernels (uph_peaks.cu): FP32 and FP64 multiply-add and
// exp2f rates into out[0..2]; returns a cudaError_t.
int measure_peaks(cudaStream_t s, int sms, double* out);

// ---- Job-wide work queues of the LM loop -----------------------------------
// Each LM phase of a job runs as one persistent kernel per kernel kind over
// every chunk: its CTAs pull items from an atomic counter, an item being one
// unit of work (the CTA-sized piece the per-chunk kernels map to a block) of
// an active island.  The active islands of a phase are compacted on the
// device from a fixed longest-first order of every (chunk, island) of the
// job, with an exclusive prefix of units per kind, at the start of every
// iteration, so converged islands drop out of the queue on the device.
enum { QK_SETUP = 0, QK_RENDER, QK_GLIN, QK_GLINR, QK_GTC, QK_GTCR, QK_ASSEMBLE, QK_STEP,
       QK_TRIAL, QK_ACCEPT, QK_KINDS };

struct QueueList {
  const ClassDev* cls;   // (nch) chunk descriptors
  int2* act;             // (n_total) active (chunk, island) entries, longest first
  int* n_act;            // [1]
  int* pre;              // (QK_KINDS, stride) exclusive prefix of units per kind
  int stride;            // n_total + 1
  int* next;             // (QK_KINDS) item counters, zeroed by the build
  int cap[QK_KINDS];     // units per kind if every island of the list were
                         // active (the host caps the persistent grids by it)
  int per_cta;           // 1: one unit per CTA, grid = cap (CTAs past the
                         // active units exit at once); 0: persistent CTAs
};

// Block sets of a chunk's FP32 Gram (CTAs that share the 8 x 8 blocks of the
// upper triangle when there are more blocks than threads).
__host__ __device__ __forceinline__ int gram_lin_parts(int Kmax) {
  const int nbk = (Kmax + 7) / 8;
  const int nblk = nbk * (nbk + 1) / 2;
  return nblk <= 256 ? 1 : (nblk + 255) / 256;
}

// The per-chunk FP32 Gram kernel's grid y: block sets x pixel splits.
__host__ __device__ __forceinline__ int gram_lin_ydim(const ClassDev& c) {
  return gram_lin_parts(c.Kmax) * (c.gl_split > 1 ? c.gl_split : 1);
}

// Pixel splits of the FP32 Gram for a window of side B and Kmax rows: one
// CTA per 2048 window pixels of a large Gram, at most 8 (windows of 96 and
// 128 px hold the blends with the largest Grams and the fewest islands per
// class, whose Gram CTAs would otherwise run alone); no split for small
// Grams or windows.  Depends on the class only, so an island's Gram does not
// depend on how many islands its chunk holds.
__host__ __device__ __forceinline__ int gram_lin_splits(int B, int Kmax) {
  if (Kmax <= 32 || B * B < 4096) return 1;
  const int s = (B * B) / 2048;
  return s < 8 ? s : 8;
}

// Units of work per island of a chunk for each kernel kind: the blocks the
// per-chunk kernel gives one island.
__host__ __device__ __forceinline__ int queue_units(const ClassDev& c, int kind) {
  const bool tc = c.tc_min_rows < (1 << 30);
  switch (kind) {
    case QK_SETUP: return (c.nb * c.N + 3) / 4;   // four member records per CTA
    case QK_RENDER: return c.nb * c.N * c.ntile_side * c.ntile_side;
    case QK_GLIN: return c.nb * gram_lin_ydim(c);
    case QK_GLINR: return c.gl_split > 1 ? c.nb : 0;
    case QK_GTC: return tc ? c.nb * c.tc_split : 0;
    case QK_GTCR: return (tc && c.tc_split > 1) ? c.nb : 0;
    case QK_ASSEMBLE: return c.nb;
    case QK_TRIAL: return c.nb;
    default: return 1;   // step, accept
  }
}

// Entry of unit `it` in an exclusive prefix pre[0..n] (pre[0] = 0 <= it <
// pre[n]): the largest a with pre[a] <= it.  Warp-cooperative (called by all
// 32 lanes of one warp): each round compares 32 probes spread over the
// remaining range in one memory round trip and keeps the sub-range between
// the last probe at or below `it` and the next one.
__device__ __forceinline__ int queue_find(const int* pre, int n, int it) {
  const int lane = threadIdx.x & 31;
  int lo = 0, hi = n;                     // pre[lo] <= it < pre[hi]
  while (hi - lo > 32) {
    const long long span = hi - lo;       // >= 33: probes lo + span (j + 1) / 33 lie
    const int pos = lo + (int)(span * (lane + 1) / 33);   // in [lo + 1, hi - 1]
    const unsigned m = __ballot_sync(0xffffffffu, pre[pos] <= it);
    if (m) {
      const int k = 31 - __clz(m);
      const int nlo = lo + (int)(span * (k + 1) / 33);
      if (k < 31) hi = lo + (int)(span * (k + 2) / 33);
      lo = nlo;
    } else {
      hi = lo + (int)(span / 33);
    }
  }
  const int pos = lo + 1 + lane;
  const unsigned m = __ballot_sync(0xffffffffu, pos < hi && pre[pos] <= it);
  return m ? lo + 1 + (31 - __clz(m)) : lo;
}

// Persistent loop of a queue kernel: ranges of `grab` consecutive units from
// q.next until the kind's units run out (the first unit's entry found by
// warp 0, the next ones by stepping forward).  The chunk's descriptor is
// copied into shared memory when the chunk changes; body(c, island, unit)
// runs the per-chunk kernel's work for that unit with the whole CTA and
// returns true to stop this CTA (a bounded device wait expired).
template <class Body>
__device__ __forceinline__ void queue_run(const QueueList& q, int kind, int grab, Body body) {
  __shared__ ClassDev sc;
  __shared__ int s_base, s_a;
  const int n = *q.n_act;
  const int* pre = q.pre + (size_t)kind * q.stride;
  const int total = pre[n];
  int cur = -1;
  if (q.per_cta) {
    // one unit per CTA (grid-stride when the grid is smaller than the units)
    for (int it = blockIdx.x; it < total; it += gridDim.x) {
      if (threadIdx.x < 32) {
        const int a0 = queue_find(pre, n, it);
        if (threadIdx.x == 0) s_a = a0;
      }
      __syncthreads();
      const int a = s_a;
      const int ch = q.act[a].x;
      if (ch != cur) {
        const int* src = reinterpret_cast<const int*>(q.cls + ch);
        int* dst = reinterpret_cast<int*>(&sc);
        for (int i = threadIdx.x; i < (int)(sizeof(ClassDev) / sizeof(int)); i += blockDim.x)
          dst[i] = src[i];
        cur = ch;
      }
      __syncthreads();
      const bool stop = body(sc, q.act[a].y, it - pre[a]);
      __syncthreads();
      if (stop) return;
    }
    return;
  }
  for (;;) {
    if (threadIdx.x == 0) s_base = atomicAdd(q.next + kind, grab);
    __syncthreads();
    const int base = s_base;
    if (base >= total) break;
    if (threadIdx.x < 32) {
      const int a0 = queue_find(pre, n, base);
      if (threadIdx.x == 0) s_a = a0;
    }
    __syncthreads();
    int a = s_a;
    const int end = min(base + grab, total);
    for (int it = base; it < end; ++it) {
      while (pre[a + 1] <= it) ++a;         // the same values in every thread
      const int ch = q.act[a].x;
      if (ch != cur) {
        const int* src = reinterpret_cast<const int*>(q.cls + ch);
        int* dst = reinterpret_cast<int*>(&sc);
        for (int i = threadIdx.x; i < (int)(sizeof(ClassDev) / sizeof(int)); i += blockDim.x)
          dst[i] = src[i];
        cur = ch;
        __syncthreads();
      }
      const bool stop = body(sc, q.act[a].y, it - pre[a]);
      __syncthreads();
      if (stop) return;
    }
  }
}

// Launchers of the queue kernels (grid: resident CTAs on every SM).
void launch_q_setup(const QueueList& q, int phase, bool p_try, int sms, cudaStream_t s);
void launch_q_render(const QueueList& q, int phase, bool lin, bool p_try, size_t render_smem,
                     int sms, cudaStream_t s);
void launch_q_gram_lin(const QueueList& q, bool bg, bool reduce, size_t smem, int sms,
                       cudaStream_t s);
void launch_q_assemble(const QueueList& q, size_t smem, int sms, cudaStream_t s);
void launch_q_step(const QueueList& q, size_t smem, int sms, cudaStream_t s);
void launch_q_trial(const QueueList& q, bool bg, size_t smem, int sms, cudaStream_t s);
void launch_q_accept(const QueueList& q, int sms, cudaStream_t s);
void launch_q_gram_tc(const QueueList& q, size_t smem, bool reduce, int sms, cudaStream_t s);
void launch_q_build(const ClassDev* cls, const int2* order, int n_total, const QueueList& q,
                    int phase, cudaStream_t s);
void launch_q_count(const ClassDev* cls, const int2* order, int n_total, int* out,
                    cudaStream_t s);
size_t render_phase_smem(const ClassDev& c, int phase);

// Member stamp rendering: unit-flux model m_k and its analytic derivatives
// d m_k / d theta for the live parameters, on the part of the member's T x T
// stamp that falls inside the island window.
//
// One CTA = one 32x32 output tile of one member in one band of one island.
// The un-shifted stamp S (and its partials) is evaluated on the tile plus a
// 3-pixel Lanczos halo in shared memory, then the separable Lanczos-3 shift
// runs as an x pass and a y pass (fixed tap order, zero border at the stamp
// edge), exactly the reference's chain:
//   m   = corr_y(corr_x(S, Lx), Ly)                (lanczos.py:102-181)
//   dm/dx = corr_y(corr_x(S, dLx) + corr_x(S_x, Lx), Ly)
//   dm/dy = corr_y(corr_x(S, Lx), dLy) + corr_y(corr_x(S_y, Lx), Ly)
//   dm/dshape = corr_y(corr_x(S_shape, Lx), Ly)
// where dx = x - x0 - rint(x - x0) and d rint / dx = 0 (island_solver.py:441-458).
//
// S is either the pixelised polynomial PSF (render mode "reference",
// psf_polynomial.py:134-197) or the analytic Gaussian-mixture PSF convolved
// with the Sersic MoG galaxy (render mode "analytic").
#include "uph_internal.cuh"

namespace {

constexpr int NS = 7;            // S arrays: S, Sx, Sy, Slr, Se1, Se2, Su
constexpr int HP = UPH_HALO + 1; // padded halo pitch
constexpr int XP = UPH_TILE + 1;

struct GComp {
  float ia, ib, ic;          // inverse covariance
  float A, B, C, det;        // covariance xx, xy, yy
  float nrm, nx, ny, nu;     // weight * amplitude / (2 pi sqrt det) (+ d/dx, d/dy, d/dn)
  float v, dv;               // galaxy variance scale and d v / d n
  float dAx, dBx, dCx, dAy, dBy, dCy;
};

struct MemberSetup {
  float Lx[7], dLx[7], Ly[7], dLy[7];
  float beta[UPH_MAXNT], betax[UPH_MAXNT], betay[UPH_MAXNT];
  float dcov[3][3];          // d(cxx, cyy, cxy) / d(logre, ee1, ee2)
  float cg[3];               // unit galaxy covariance (cxx, cyy, cxy)
  float dndu;
  int ncomp;
  int is_gal;
  int need[NS];
  int live_row[6];           // stamp row of parameter j (0 = not live)
};

__device__ void lanczos_taps(double d, float* L, float* dL) {
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

__device__ double ipow(double x, int e) {
  double r = 1.0;
  for (int i = 0; i < e; ++i) r *= x;
  return r;
}

// Ellipse (logre, ee1, ee2) -> unit covariance and its Jacobian
// (sersic_mog.py:108-150, incl. the round-source nudge).
__device__ void cov_terms(double lr, double e1, double e2, float* cg,
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

__device__ void sersic_lookup(const ClassDev& c, double n, double* a,
                              double* v, double& core, double* da, double* dv,
                              double& dcore) {
  bool inside = (n > c.tb_nmin) && (n < c.tb_nmax);
  double nc = fmin(fmax(n, c.tb_nmin), c.tb_nmax);
  // searchsorted(side='right') - 1
  int lo = 0, hi = c.tb_n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (c.tb_knots[mid] <= nc) lo = mid + 1; else hi = mid;
  }
  int i = lo - 1;
  i = max(0, min(i, c.tb_n - 2));
  double n0 = c.tb_knots[i], n1 = c.tb_knots[i + 1];
  double t = 0.0, dt = 0.0;
  if (n1 > n0) {
    t = (nc - n0) / (n1 - n0);
    dt = inside ? 1.0 / (n1 - n0) : 0.0;
  }
  for (int g = 0; g < c.tb_k; ++g) {
    double a0 = c.tb_amps[i * c.tb_k + g], a1 = c.tb_amps[(i + 1) * c.tb_k + g];
    double l0 = c.tb_lv[i * c.tb_k + g], l1 = c.tb_lv[(i + 1) * c.tb_k + g];
    a[g] = (1 - t) * a0 + t * a1;
    v[g] = exp((1 - t) * l0 + t * l1);
    da[g] = dt * (a1 - a0);
    dv[g] = v[g] * dt * (l1 - l0);
  }
  core = (1 - t) * c.tb_core[i] + t * c.tb_core[i + 1];
  dcore = dt * (c.tb_core[i + 1] - c.tb_core[i]);
}

// Analytic-mode member setup: PSF components at (x, y) and the galaxy
// mixture, combined into Gaussian components (covariances add).
__device__ void setup_analytic(const ClassDev& c, int b, int isl, int k,
                               const float* P, MemberSetup& ms, GComp* comps,
                               bool lin) {
  const float* os = c.psf_os + 4 * b;
  double X = ((double)P[(size_t)isl * c.nP + 6 * k] - os[0]) / os[1];
  double Y = ((double)P[(size_t)isl * c.nP + 6 * k + 1] - os[2]) / os[3];
  double bt[UPH_MAXNT], bx[UPH_MAXNT], by[UPH_MAXNT];
  for (int t = 0; t < c.nt; ++t) {
    int m, n;
    term_mn(t, m, n);
    bt[t] = ipow(X, m) * ipow(Y, n);
    bx[t] = m > 0 ? m * ipow(X, m - 1) * ipow(Y, n) / os[1] : 0.0;
    by[t] = n > 0 ? n * ipow(X, m) * ipow(Y, n - 1) / os[3] : 0.0;
  }
  double w[UPH_MAXKPSF], wx[UPH_MAXKPSF], wy[UPH_MAXKPSF];
  double cq[UPH_MAXKPSF][3], cx[UPH_MAXKPSF][3], cy[UPH_MAXKPSF][3];
  double W = 0, Wx = 0, Wy = 0;
  for (int q = 0; q < c.kpsf; ++q) {
    double val[4] = {0, 0, 0, 0}, vx[4] = {0, 0, 0, 0}, vy[4] = {0, 0, 0, 0};
    for (int f = 0; f < 4; ++f) {
      const float* cf = c.mog + (((size_t)b * c.kpsf + q) * 4 + f) * c.nt;
      for (int t = 0; t < c.nt; ++t) {
        val[f] += cf[t] * bt[t];
        vx[f] += cf[t] * bx[t];
        vy[f] += cf[t] * by[t];
      }
    }
    double s = val[0], a1 = val[1], a2 = val[2];
    double s2 = s * s;
    cq[q][0] = s2 * (1 + a1);
    cq[q][1] = s2 * (1 - a1);
    cq[q][2] = s2 * a2;
    cx[q][0] = 2 * s * vx[0] * (1 + a1) + s2 * vx[1];
    cx[q][1] = 2 * s * vx[0] * (1 - a1) - s2 * vx[1];
    cx[q][2] = 2 * s * vx[0] * a2 + s2 * vx[2];
    cy[q][0] = 2 * s * vy[0] * (1 + a1) + s2 * vy[1];
    cy[q][1] = 2 * s * vy[0] * (1 - a1) - s2 * vy[1];
    cy[q][2] = 2 * s * vy[0] * a2 + s2 * vy[2];
    w[q] = val[3];
    wx[q] = vx[3];
    wy[q] = vy[3];
    W += val[3];
    Wx += vx[3];
    Wy += vy[3];
  }
  for (int q = 0; q < c.kpsf; ++q) {
    double wn = w[q] / W;
    double wnx = (wx[q] * W - w[q] * Wx) / (W * W);
    double wny = (wy[q] * W - w[q] * Wy) / (W * W);
    w[q] = wn;
    wx[q] = wnx;
    wy[q] = wny;
  }
  // galaxy mixture
  double ga[UPH_MAXGAL], gv[UPH_MAXGAL], gda[UPH_MAXGAL], gdv[UPH_MAXGAL];
  int ng = 0;
  ms.cg[0] = ms.cg[1] = ms.cg[2] = 0.f;
  ms.dndu = 0.f;
  if (ms.is_gal) {
    const float* pk = P + (size_t)isl * c.nP + 6 * k;
    double n, dndu = 0.0;
    if (c.free_n[isl * c.N + k]) {
      float u = pk[5];
      float nf = 0.29f + 6.01f / (1.0f + expf(-u));
      n = (double)nf;
      double eu = exp(-(double)u);
      dndu = 6.01 * eu / ((1.0 + eu) * (1.0 + eu));
    } else {
      n = (double)c.n_frozen[isl * c.N + k];
    }
    double a[UPH_MAXGAL], v[UPH_MAXGAL], da[UPH_MAXGAL], dv[UPH_MAXGAL];
    double core, dcore;
    sersic_lookup(c, n, a, v, core, da, dv, dcore);
    for (int g = 0; g < c.tb_k; ++g) {
      if (a[g] != 0.0 || da[g] != 0.0) {
        ga[ng] = a[g];
        gv[ng] = v[g];
        gda[ng] = da[g];
        gdv[ng] = dv[g];
        ++ng;
      }
    }
    if (core != 0.0 || dcore != 0.0) {
      ga[ng] = core;
      gv[ng] = 0.0;
      gda[ng] = dcore;
      gdv[ng] = 0.0;
      ++ng;
    }
    cov_terms((double)pk[2], (double)pk[3], (double)pk[4], ms.cg, ms.dcov);
    ms.dndu = (float)dndu;
  } else {
    ga[0] = 1.0;
    gv[0] = 0.0;
    gda[0] = 0.0;
    gdv[0] = 0.0;
    ng = 1;
  }
  int nc = 0;
  const double inv2pi = 0.15915494309189535;
  for (int q = 0; q < c.kpsf; ++q) {
    for (int g = 0; g < ng; ++g) {
      GComp& o = comps[nc++];
      double A = gv[g] * ms.cg[0] + cq[q][0];
      double C = gv[g] * ms.cg[1] + cq[q][1];
      double B = gv[g] * ms.cg[2] + cq[q][2];
      double det = A * C - B * B;
      double rs = inv2pi / sqrt(det);
      o.ia = (float)(C / det);
      o.ib = (float)(-B / det);
      o.ic = (float)(A / det);
      o.A = (float)A;
      o.B = (float)B;
      o.C = (float)C;
      o.det = (float)det;
      o.nrm = (float)(w[q] * ga[g] * rs);
      o.nx = (float)(wx[q] * ga[g] * rs);
      o.ny = (float)(wy[q] * ga[g] * rs);
      o.nu = (float)(w[q] * gda[g] * rs);
      o.v = (float)gv[g];
      o.dv = (float)gdv[g];
      o.dAx = (float)cx[q][0];
      o.dCx = (float)cx[q][1];
      o.dBx = (float)cx[q][2];
      o.dAy = (float)cy[q][0];
      o.dCy = (float)cy[q][1];
      o.dBy = (float)cy[q][2];
    }
  }
  ms.ncomp = nc;
}

__global__ void __launch_bounds__(256)
k_render(ClassDev c, const float* __restrict__ P, int phase) {
  extern __shared__ float smem[];
  __shared__ MemberSetup ms;
  __shared__ GComp comps[UPH_MAXKPSF * UPH_MAXGAL];
  __shared__ MemberBox mb;
  const int ntile = c.ntile_side * c.ntile_side;
  int t = blockIdx.x;
  const int tile = t % ntile;
  t /= ntile;
  const int k = t % c.N;
  t /= c.N;
  const int b = t % c.nb;
  const int isl = t / c.nb;
  if (isl >= c.n_isl) return;
  if (!isl_active(c.flags[isl], phase)) return;
  if (!c.mmask[isl * c.N + k]) return;
  const bool lin = (phase == PH_LIN);
  const int tid = threadIdx.x;

  if (tid == 0) {
    mb = member_box(c, isl, P, k);
    ms.is_gal = c.stype[isl * c.N + k] != 0;
    const uint8_t* kp = c.keep + ((size_t)isl * c.N + k) * 6;
    int row = 1;
    for (int j = 0; j < 6; ++j) {
      bool live = lin && kp[j] && (j < 2 || ms.is_gal);
      ms.live_row[j] = live ? row++ : 0;
    }
    for (int s = 0; s < NS; ++s) ms.need[s] = 0;
    ms.need[0] = 1;
    ms.need[1] = ms.live_row[0] && c.psf_varies;
    ms.need[2] = ms.live_row[1] && c.psf_varies;
    for (int s = 0; s < 3; ++s) ms.need[3 + s] = ms.live_row[2 + s] != 0;
    ms.need[6] = ms.live_row[5] != 0;
    lanczos_taps((double)mb.dx, ms.Lx, ms.dLx);
    lanczos_taps((double)mb.dy, ms.Ly, ms.dLy);
    if (c.mode == 0) {
      const float* os = c.psf_os + 4 * b;
      const float x = P[(size_t)isl * c.nP + 6 * k];
      const float y = P[(size_t)isl * c.nP + 6 * k + 1];
      const float X = __fdiv_rn(__fsub_rn(x, os[0]), os[1]);
      const float Y = __fdiv_rn(__fsub_rn(y, os[2]), os[3]);
      const float ix = __fdiv_rn(1.0f, os[1]);
      const float iy = __fdiv_rn(1.0f, os[3]);
      for (int tt = 0; tt < c.nt; ++tt) {
        int m, n;
        term_mn(tt, m, n);
        float xm = 1.f, yn = 1.f, xm1 = 1.f, yn1 = 1.f;
        for (int i = 0; i < m; ++i) xm *= X;
        for (int i = 0; i < n; ++i) yn *= Y;
        for (int i = 0; i + 1 < m; ++i) xm1 *= X;
        for (int i = 0; i + 1 < n; ++i) yn1 *= Y;
        ms.beta[tt] = xm * yn;
        ms.betax[tt] = m > 0 ? (float)m * xm1 * yn * ix : 0.f;
        ms.betay[tt] = n > 0 ? (float)n * xm * yn1 * iy : 0.f;
      }
    } else {
      setup_analytic(c, b, isl, k, P, ms, comps, lin);
    }
  }
  __syncthreads();
  if (mb.bw <= 0 || mb.bh <= 0) return;
  const int ty = tile / c.ntile_side, tx = tile % c.ntile_side;
  const int oy0 = mb.wy0 + UPH_TILE * ty, ox0 = mb.wx0 + UPH_TILE * tx;
  if (oy0 >= mb.wy0 + mb.bh || ox0 >= mb.wx0 + mb.bw) return;
  const int oh = min(UPH_TILE, mb.wy0 + mb.bh - oy0);
  const int ow = min(UPH_TILE, mb.wx0 + mb.bw - ox0);
  const int si0 = oy0 - mb.iyt, sj0 = ox0 - mb.ixt;  // stamp coords of tile
  const int hr = oh + 6, hc = ow + 6;
  float* S = smem;                           // NS * UPH_HALO * HP
  float* X = smem + NS * UPH_HALO * HP;      // NS * UPH_HALO * XP
  const int T = c.T, c0 = c.T / 2;

  // ---- un-shifted stamp (and partials) on the halo region ----
  for (int e = tid; e < hr * hc; e += blockDim.x) {
    const int r = e / hc, cc = e % hc;
    const int si = si0 - 3 + r, sj = sj0 - 3 + cc;
    float v[NS] = {0, 0, 0, 0, 0, 0, 0};
    if (si >= 0 && si < T && sj >= 0 && sj < T) {
      if (c.mode == 0) {
        const float* cf = c.psf_coefs + (((size_t)b * T + si) * T + sj) * c.nt;
        float s0 = 0.f, sx = 0.f, sy = 0.f;
        for (int tt = 0; tt < c.nt; ++tt) {
          const float cv = cf[tt];
          s0 = fmaf(cv, ms.beta[tt], s0);
          sx = fmaf(cv, ms.betax[tt], sx);
          sy = fmaf(cv, ms.betay[tt], sy);
        }
        v[0] = s0;
        v[1] = sx;
        v[2] = sy;
      } else {
        const float xo = (float)(sj - c0), yo = (float)(si - c0);
        float s0 = 0.f, sx = 0.f, sy = 0.f, gA = 0.f, gB = 0.f, gC = 0.f,
              u1 = 0.f, u2 = 0.f;
        for (int q = 0; q < ms.ncomp; ++q) {
          const GComp& o = comps[q];
          const float Q = fmaf(o.ia * xo, xo, fmaf(2.f * o.ib * xo, yo, o.ic * yo * yo));
          const float ex = expf(-0.5f * Q);
          const float nw = o.nrm * ex;
          s0 += nw;
          if (lin) {
            const float i2d = 0.5f / o.det;
            const float dA = (Q * o.C - yo * yo - o.C) * i2d;
            const float dC = (Q * o.A - xo * xo - o.A) * i2d;
            const float dB = (xo * yo - o.B * Q + o.B) * (2.f * i2d);
            if (ms.need[1]) sx += o.nx * ex + nw * (dA * o.dAx + dC * o.dCx + dB * o.dBx);
            if (ms.need[2]) sy += o.ny * ex + nw * (dA * o.dAy + dC * o.dCy + dB * o.dBy);
            if (ms.is_gal) {
              const float nv = nw * o.v;
              gA = fmaf(nv, dA, gA);
              gC = fmaf(nv, dC, gC);
              gB = fmaf(nv, dB, gB);
              u1 = fmaf(o.nu, ex, u1);
              u2 += nw * o.dv * (dA * ms.cg[0] + dC * ms.cg[1] + dB * ms.cg[2]);
            }
          }
        }
        v[0] = s0;
        v[1] = sx;
        v[2] = sy;
        for (int s = 0; s < 3; ++s)
          v[3 + s] = gA * ms.dcov[s][0] + gC * ms.dcov[s][1] + gB * ms.dcov[s][2];
        v[6] = ms.dndu * (u1 + u2);
      }
    }
    for (int s = 0; s < NS; ++s)
      if (ms.need[s]) S[(s * UPH_HALO + r) * HP + cc] = v[s];
  }
  __syncthreads();

  // ---- x pass: X0 = cx(S,L), X1 = cx(S,dL) + cx(Sx,L), X2 = cx(Sy,L),
  //      X3..5 = cx(S_shape,L), X6 = cx(Su,L) ----
  const bool dox = ms.live_row[0] != 0;
  for (int e = tid; e < hr * ow; e += blockDim.x) {
    const int r = e / ow, cc = e % ow;
    const float* s0 = S + (0 * UPH_HALO + r) * HP + cc;
    float a0 = ms.Lx[0] * s0[0];
    for (int q = 1; q < 7; ++q) a0 = fmaf(ms.Lx[q], s0[q], a0);
    X[(0 * UPH_HALO + r) * XP + cc] = a0;
    if (dox) {
      float a1 = ms.dLx[0] * s0[0];
      for (int q = 1; q < 7; ++q) a1 = fmaf(ms.dLx[q], s0[q], a1);
      if (ms.need[1]) {
        const float* s1 = S + (1 * UPH_HALO + r) * HP + cc;
        float b1 = ms.Lx[0] * s1[0];
        for (int q = 1; q < 7; ++q) b1 = fmaf(ms.Lx[q], s1[q], b1);
        a1 += b1;
      }
      X[(1 * UPH_HALO + r) * XP + cc] = a1;
    }
    for (int s = 2; s < NS; ++s) {
      if (!ms.need[s]) continue;
      const float* sp = S + (s * UPH_HALO + r) * HP + cc;
      float a = ms.Lx[0] * sp[0];
      for (int q = 1; q < 7; ++q) a = fmaf(ms.Lx[q], sp[q], a);
      X[(s * UPH_HALO + r) * XP + cc] = a;
    }
  }
  __syncthreads();

  // ---- y pass and store ----
  const int Sz = c.Sz;
  for (int e = tid; e < oh * ow; e += blockDim.x) {
    const int rr = e / ow, cc = e % ow;
    const int wy = oy0 + rr, wx = ox0 + cc;
    const size_t off = (size_t)(wy - mb.wy0) * Sz + (wx - mb.wx0);
    const float* x0 = X + (0 * UPH_HALO + rr) * XP + cc;
    float m = ms.Ly[0] * x0[0];
    for (int q = 1; q < 7; ++q) m = fmaf(ms.Ly[q], x0[q * XP], m);
    c.stamps[stamp_slot(c, isl, b, k, 0) + off] = m;
    if (!lin) continue;
    if (ms.live_row[0]) {
      const float* x1 = X + (1 * UPH_HALO + rr) * XP + cc;
      float d = ms.Ly[0] * x1[0];
      for (int q = 1; q < 7; ++q) d = fmaf(ms.Ly[q], x1[q * XP], d);
      c.stamps[stamp_slot(c, isl, b, k, ms.live_row[0]) + off] = d;
    }
    if (ms.live_row[1]) {
      float d = ms.dLy[0] * x0[0];
      for (int q = 1; q < 7; ++q) d = fmaf(ms.dLy[q], x0[q * XP], d);
      if (ms.need[2]) {
        const float* x2 = X + (2 * UPH_HALO + rr) * XP + cc;
        float d2 = ms.Ly[0] * x2[0];
        for (int q = 1; q < 7; ++q) d2 = fmaf(ms.Ly[q], x2[q * XP], d2);
        d += d2;
      }
      c.stamps[stamp_slot(c, isl, b, k, ms.live_row[1]) + off] = d;
    }
    for (int j = 2; j < 6; ++j) {
      if (!ms.live_row[j]) continue;
      const int s = j + 1;  // S arrays 3..6 hold lr, e1, e2, u
      const float* xs = X + (s * UPH_HALO + rr) * XP + cc;
      float d = ms.Ly[0] * xs[0];
      for (int q = 1; q < 7; ++q) d = fmaf(ms.Ly[q], xs[q * XP], d);
      c.stamps[stamp_slot(c, isl, b, k, ms.live_row[j]) + off] = d;
    }
  }
}

}  // namespace

size_t render_smem_bytes() {
  return sizeof(float) * (size_t)NS * UPH_HALO * (HP + XP);
}

void launch_render(const ClassDev& c, const float* P, int phase,
                   cudaStream_t s) {
  const long long nblk = (long long)c.n_isl * c.nb * c.N * c.ntile_side * c.ntile_side;
  if (nblk <= 0) return;
  k_render<<<(unsigned)nblk, 256, render_smem_bytes(), s>>>(c, P, phase);
}

int uph_render_setup() {
  return (int)cudaFuncSetAttribute(k_render,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)render_smem_bytes());
}

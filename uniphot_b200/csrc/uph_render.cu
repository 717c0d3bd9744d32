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
#include <algorithm>

#include "uph_internal.cuh"

namespace {

constexpr int NS = 7;            // S arrays: S, Sx, Sy, Slr, Se1, Se2, Su
constexpr int HP = UPH_HALO + 1; // padded halo pitch

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
  int support_half;          // S is zero beyond this offset from the centre
  int nact;                  // components active on this tile
  uint8_t act[UPH_MAXKPSF * UPH_MAXGAL];
};

// Pruning threshold: a Gaussian term whose Mahalanobis distance Q exceeds
// this everywhere on a tile contributes < exp(-23) ~ 1e-10 of its norm there
// (its derivative rows at most a factor ~Q more), far below the float32
// resolution of the pixels it would touch relative to the member's peak.
constexpr float QCUT = 46.f;

// Per-tile record of one active analytic component: the exponent
// coefficients (Q' = qa x^2 + qb x y + qc y^2, value = nrm 2^Q') and, for the
// linearisation, one quadratic form per derivative row so that
//   row_o = sum_comp 2^Q' (a_o x^2 + b_o x y + c_o y^2 + d_o).
// Rows o = 0..5 are S arrays 1..6 (x, y, log r_e, e1, e2, Sersic n): the
// covariance derivatives dQ/dA, dQ/dC, dQ/dB of the exponential are quadratic
// forms, and the member's d(cov)/d(shape) and d n / d u are folded in.
constexpr int MAXCOMP = UPH_MAXKPSF * UPH_MAXGAL;
constexpr float KEXP = -0.72134752044448170f;   // -1 / (2 ln 2)

template <int NOUT>
__device__ __forceinline__ void mog_pair(const float4* __restrict__ rec, int na,
                                         float x2a, float xya, float y2a,
                                         float x2b, float xyb, float y2b,
                                         float* va, float* vb) {
  float s0a = 0.f, s0b = 0.f;
  float aa[NOUT > 0 ? NOUT : 1], ab[NOUT > 0 ? NOUT : 1];
#pragma unroll
  for (int o = 0; o < NOUT; ++o) aa[o] = ab[o] = 0.f;
  for (int a = 0; a < na; ++a) {
    const float4 q = rec[a * (NOUT + 1)];
    const float ea = exp2f(fmaf(q.x, x2a, fmaf(q.y, xya, q.z * y2a)));
    const float eb = exp2f(fmaf(q.x, x2b, fmaf(q.y, xyb, q.z * y2b)));
    s0a = fmaf(q.w, ea, s0a);
    s0b = fmaf(q.w, eb, s0b);
#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
      const float4 k = rec[a * (NOUT + 1) + 1 + o];
      aa[o] = fmaf(ea, fmaf(k.x, x2a, fmaf(k.y, xya, fmaf(k.z, y2a, k.w))), aa[o]);
      ab[o] = fmaf(eb, fmaf(k.x, x2b, fmaf(k.y, xyb, fmaf(k.z, y2b, k.w))), ab[o]);
    }
  }
  va[0] = s0a;
  vb[0] = s0b;
#pragma unroll
  for (int o = 0; o < NOUT; ++o) {
    va[1 + o] = aa[o];
    vb[1 + o] = ab[o];
  }
}

// Minimum over the rectangle [x0,x1] x [y0,y1] of
// Q = ia x^2 + 2 ib x y + ic y^2 (positive definite).
__device__ float qmin_box(float ia, float ib, float ic, float x0, float x1,
                          float y0, float y1) {
  if (x0 <= 0.f && x1 >= 0.f && y0 <= 0.f && y1 >= 0.f) return 0.f;
  float best = INFINITY;
  const float xs[2] = {x0, x1}, ys[2] = {y0, y1};
  for (int e = 0; e < 2; ++e) {
    const float xe = xs[e];
    const float y = fminf(fmaxf(-ib * xe / ic, y0), y1);
    best = fminf(best, ia * xe * xe + 2.f * ib * xe * y + ic * y * y);
    const float ye = ys[e];
    const float x = fminf(fmaxf(-ib * ye / ia, x0), x1);
    best = fminf(best, ia * x * x + 2.f * ib * x * ye + ic * ye * ye);
  }
  return best;
}

__device__ double ipow(double x, int e) {
  double r = 1.0;
  for (int i = 0; i < e; ++i) r *= x;
  return r;
}

// Per-member scratch of the parallel setup (analytic mode).
struct PsfComp {
  double w, wx, wy;          // raw weight and its d/dx, d/dy
  double cov[3], cx[3], cy[3];
};
struct GalComp {
  double a, v, da, dv;
};
struct SetupScratch {
  PsfComp pq[UPH_MAXKPSF];
  GalComp gg[UPH_MAXGAL];
  int ng;
  int seg;                   // Sersic table segment
  double t, dt;              // interpolation weight and d t / d n
  double W, Wx, Wy;          // weight sums
};

// PSF component q at the member position (one thread per component).
__device__ void psf_component(const ClassDev& c, int b, double X, double Y,
                              double ixs, double iys, int q, PsfComp& o) {
  double val[4] = {0, 0, 0, 0}, vx[4] = {0, 0, 0, 0}, vy[4] = {0, 0, 0, 0};
  for (int t = 0; t < c.nt; ++t) {
    int m, n;
    term_mn(t, m, n);
    const double bt = ipow(X, m) * ipow(Y, n);
    const double bx = m > 0 ? m * ipow(X, m - 1) * ipow(Y, n) * ixs : 0.0;
    const double by = n > 0 ? n * ipow(X, m) * ipow(Y, n - 1) * iys : 0.0;
    for (int f = 0; f < 4; ++f) {
      const double cf = c.mog[(((size_t)b * c.kpsf + q) * 4 + f) * c.nt + t];
      val[f] += cf * bt;
      vx[f] += cf * bx;
      vy[f] += cf * by;
    }
  }
  const double s = val[0], a1 = val[1], a2 = val[2], s2 = s * s;
  o.cov[0] = s2 * (1 + a1);
  o.cov[1] = s2 * (1 - a1);
  o.cov[2] = s2 * a2;
  o.cx[0] = 2 * s * vx[0] * (1 + a1) + s2 * vx[1];
  o.cx[1] = 2 * s * vx[0] * (1 - a1) - s2 * vx[1];
  o.cx[2] = 2 * s * vx[0] * a2 + s2 * vx[2];
  o.cy[0] = 2 * s * vy[0] * (1 + a1) + s2 * vy[1];
  o.cy[1] = 2 * s * vy[0] * (1 - a1) - s2 * vy[1];
  o.cy[2] = 2 * s * vy[0] * a2 + s2 * vy[2];
  o.w = val[3];
  o.wx = vx[3];
  o.wy = vy[3];
}

// Per (island, band, member) setup at parameters P: Lanczos taps, PSF basis
// (reference mode) or the combined Gaussian components (analytic mode),
// written once to the member record that every render tile of the member
// reads.
__device__ __forceinline__ void member_setup_warp(const ClassDev& c,
                                                  const float* __restrict__ P, int phase,
                                                  int bx, SetupScratch& sc, int& is_gal,
                                                  int& ncomp) {
  const int k = bx % c.N;
  const int b = (bx / c.N) % c.nb;
  const int isl = bx / (c.N * c.nb);
  if (isl >= c.n_isl) return;
  if (!isl_active(c.flags[isl], phase)) return;
  if (!c.mmask[isl * c.N + k]) return;
  const int lane = threadIdx.x & 31;
  MemberRecord* rec = c.mrec + ((size_t)isl * c.nb + b) * c.N + k;
  const float px = P[(size_t)isl * c.nP + 6 * k];
  const float py = P[(size_t)isl * c.nP + 6 * k + 1];
  if (lane == 0) {
    is_gal = c.has_gal && c.stype[isl * c.N + k] != 0;
    for (int a = 0; a < 3; ++a) {
      rec->cg[a] = 0.f;
      for (int q = 0; q < 3; ++q) rec->dcov[a][q] = 0.f;
    }
    rec->dndu = 0.f;
    rec->ncomp = 0;
    rec->ngal = 0;
    if (is_gal) {
      const float* pk = P + (size_t)isl * c.nP + 6 * k;
      double n;
      if (c.free_n[isl * c.N + k]) {
        const float u = pk[5];
        n = (double)(0.29f + 6.01f / (1.0f + expf(-u)));
        const double eu = exp(-(double)u);
        rec->dndu = (float)(6.01 * eu / ((1.0 + eu) * (1.0 + eu)));
      } else {
        n = (double)c.n_frozen[isl * c.N + k];
      }
      sersic_segment(c.tb_knots, c.tb_n, c.tb_nmin, c.tb_nmax, n, &sc.seg, &sc.t, &sc.dt);
      cov_terms((double)pk[2], (double)pk[3], (double)pk[4], rec->cg, rec->dcov);
    }
  } else if (lane == 1) {
    const float gx = __fsub_rn(px, c.x0b[isl]);
    lanczos_taps((double)__fsub_rn(gx, rintf(gx)), rec->Lx, rec->dLx);
  } else if (lane == 2) {
    const float gy = __fsub_rn(py, c.y0b[isl]);
    lanczos_taps((double)__fsub_rn(gy, rintf(gy)), rec->Ly, rec->dLy);
  } else if (lane >= 11 && lane < 11 + UPH_MAXNT && c.mode == 0) {
    const int tt = lane - 11;
    if (tt < c.nt) {
      const float* os = c.psf_os + 4 * b;
      const float X = __fdiv_rn(__fsub_rn(px, os[0]), os[1]);
      const float Y = __fdiv_rn(__fsub_rn(py, os[2]), os[3]);
      const float ix = __fdiv_rn(1.0f, os[1]);
      const float iy = __fdiv_rn(1.0f, os[3]);
      int m, n;
      term_mn(tt, m, n);
      float xm = 1.f, yn = 1.f, xm1 = 1.f, yn1 = 1.f;
      for (int i = 0; i < m; ++i) xm *= X;
      for (int i = 0; i < n; ++i) yn *= Y;
      for (int i = 0; i + 1 < m; ++i) xm1 *= X;
      for (int i = 0; i + 1 < n; ++i) yn1 *= Y;
      rec->beta[tt] = xm * yn;
      rec->betax[tt] = m > 0 ? (float)m * xm1 * yn * ix : 0.f;
      rec->betay[tt] = n > 0 ? (float)n * xm * yn1 * iy : 0.f;
    }
  } else if (lane >= 3 && lane < 3 + UPH_MAXKPSF && c.mode == 1) {
    const int q = lane - 3;
    if (q < c.kpsf) {
      const float* os = c.psf_os + 4 * b;
      const double X = ((double)px - os[0]) / os[1];
      const double Y = ((double)py - os[2]) / os[3];
      psf_component(c, b, X, Y, 1.0 / os[1], 1.0 / os[3], q, sc.pq[q]);
    }
  }
  __syncwarp();
  if (c.mode != 1) {
    // reference mode: the galaxy's Sersic mixture for the Fourier-domain
    // convolution (sersic_mog.py:81-100), core apart
    if (!is_gal) return;
    const int g = lane;
    if (g < c.tb_k) {
      const int seg = sc.seg;
      const double t = sc.t, dt = sc.dt;
      const double a0 = c.tb_amps[seg * c.tb_k + g], a1 = c.tb_amps[(seg + 1) * c.tb_k + g];
      const double l0 = c.tb_lv[seg * c.tb_k + g], l1 = c.tb_lv[(seg + 1) * c.tb_k + g];
      const double v = exp((1 - t) * l0 + t * l1);
      rec->ga[g] = (1 - t) * a0 + t * a1;
      rec->gv[g] = v;
      rec->gda[g] = dt * (a1 - a0);
      rec->gdv[g] = v * dt * (l1 - l0);
    } else if (g == c.tb_k) {
      const int seg = sc.seg;
      rec->gcore = (1 - sc.t) * c.tb_core[seg] + sc.t * c.tb_core[seg + 1];
      rec->gdcore = sc.dt * (c.tb_core[seg + 1] - c.tb_core[seg]);
      rec->ngal = c.tb_k;
    }
    return;
  }
  if (lane == 0) {
    double W = 0, Wx = 0, Wy = 0;
    for (int q = 0; q < c.kpsf; ++q) {
      W += sc.pq[q].w;
      Wx += sc.pq[q].wx;
      Wy += sc.pq[q].wy;
    }
    sc.W = W;
    sc.Wx = Wx;
    sc.Wy = Wy;
  } else if (lane >= 16 && lane < 16 + UPH_MAXGAL && is_gal) {
    const int g = lane - 16;
    const int seg = sc.seg;
    const double t = sc.t, dt = sc.dt;
    GalComp& o = sc.gg[g];
    if (g < c.tb_k) {
      const double a0 = c.tb_amps[seg * c.tb_k + g], a1 = c.tb_amps[(seg + 1) * c.tb_k + g];
      const double l0 = c.tb_lv[seg * c.tb_k + g], l1 = c.tb_lv[(seg + 1) * c.tb_k + g];
      o.a = (1 - t) * a0 + t * a1;
      o.v = exp((1 - t) * l0 + t * l1);
      o.da = dt * (a1 - a0);
      o.dv = o.v * dt * (l1 - l0);
    } else if (g == c.tb_k) {          // delta core: zero-variance component
      o.a = (1 - t) * c.tb_core[seg] + t * c.tb_core[seg + 1];
      o.v = 0.0;
      o.da = dt * (c.tb_core[seg + 1] - c.tb_core[seg]);
      o.dv = 0.0;
    }
  }
  __syncwarp();
  if (lane == 0) {
    // compact the galaxy components that contribute (non-zero amplitude or
    // amplitude derivative); a star is a single unit delta
    int ng = 0;
    if (is_gal) {
      for (int g = 0; g <= c.tb_k; ++g)
        if (sc.gg[g].a != 0.0 || sc.gg[g].da != 0.0) sc.gg[ng++] = sc.gg[g];
    } else {
      sc.gg[0].a = 1.0;
      sc.gg[0].v = 0.0;
      sc.gg[0].da = 0.0;
      sc.gg[0].dv = 0.0;
      ng = 1;
    }
    sc.ng = ng;
    ncomp = c.kpsf * ng;
    rec->ncomp = ncomp;
  }
  __syncwarp();
  const float* cg = rec->cg;
  for (int e = lane; e < ncomp; e += 32) {
    const int q = e / sc.ng, g = e - (e / sc.ng) * sc.ng;
    const PsfComp& pq = sc.pq[q];
    const GalComp& gq = sc.gg[g];
    const double W = sc.W;
    const double wn = pq.w / W;
    const double wnx = (pq.wx * W - pq.w * sc.Wx) / (W * W);
    const double wny = (pq.wy * W - pq.w * sc.Wy) / (W * W);
    const double A = gq.v * cg[0] + pq.cov[0];
    const double C = gq.v * cg[1] + pq.cov[1];
    const double Bc = gq.v * cg[2] + pq.cov[2];
    const double det = A * C - Bc * Bc;
    const double rs = 0.15915494309189535 / sqrt(det);
    GComp o;
    o.ia = (float)(C / det);
    o.ib = (float)(-Bc / det);
    o.ic = (float)(A / det);
    o.A = (float)A;
    o.B = (float)Bc;
    o.C = (float)C;
    o.det = (float)(0.5 / det);
    o.nrm = (float)(wn * gq.a * rs);
    o.nx = (float)(wnx * gq.a * rs);
    o.ny = (float)(wny * gq.a * rs);
    o.nu = (float)(wn * gq.da * rs);
    o.v = (float)gq.v;
    o.dv = (float)gq.dv;
    o.dAx = (float)pq.cx[0];
    o.dCx = (float)pq.cx[1];
    o.dBx = (float)pq.cx[2];
    o.dAy = (float)pq.cy[0];
    o.dCy = (float)pq.cy[1];
    o.dBy = (float)pq.cy[2];
    rec->comps[e] = o;
  }
}

// One warp per member record, four records per CTA (warp-level syncs only:
// the warps of a CTA are independent).
constexpr int SETUP_WARPS = 4;
// CTAs per SM the star-only linearisation render is held to (32 registers)
#ifndef RENDER_LIN_STAR_CTAS
#define RENDER_LIN_STAR_CTAS 8
#endif

__device__ __forceinline__ void member_setup_body(const ClassDev& c,
                                                  const float* __restrict__ P, int phase,
                                                  int rec0, int nrec) {
  __shared__ SetupScratch sc[SETUP_WARPS];
  __shared__ int is_gal[SETUP_WARPS], ncomp[SETUP_WARPS];
  const int w = threadIdx.x >> 5;
  if (w < nrec) member_setup_warp(c, P, phase, rec0 + w, sc[w], is_gal[w], ncomp[w]);
}

__global__ void __launch_bounds__(32 * SETUP_WARPS)
k_member_setup(ClassDev c, const float* __restrict__ P, int phase) {
  const long long nrec = (long long)c.n_isl * c.nb * c.N;
  const long long r0 = (long long)blockIdx.x * SETUP_WARPS;
  member_setup_body(c, P, phase, (int)r0, (int)std::min<long long>(SETUP_WARPS, nrec - r0));
}

template <bool LIN, bool GAL = true>
__device__ __forceinline__ void render_body(const ClassDev& c, const float* __restrict__ P,
                                            int phase, int bx) {
  // LIN: linearisation render (model and derivative rows); the trial and
  // probe renders (model row only) are a separate instantiation that needs
  // far fewer registers, hence more CTAs per SM.  GAL = false: the chunk
  // holds no galaxy (c.has_gal == 0), and the galaxy paths are not compiled
  // in (the star paths run the same operations in either instantiation).
  extern __shared__ float smem[];
  __shared__ MemberSetup ms;
  __shared__ float4 trec[MAXCOMP * (LIN ? (GAL ? 7 : 3) : 1)];   // per-tile component records
  __shared__ MemberBox mb;
  const int ntile = c.ntile_side * c.ntile_side;
  int t = bx;
  const int tile = t % ntile;
  t /= ntile;
  const int k = t % c.N;
  t /= c.N;
  const int b = t % c.nb;
  const int isl = t / c.nb;
  if (isl >= c.n_isl) return;
  if (!isl_active(c.flags[isl], phase)) return;
  if (!c.mmask[isl * c.N + k]) return;
  constexpr bool lin = LIN;
  const int tid = threadIdx.x;

  const MemberRecord* rec = c.mrec + ((size_t)isl * c.nb + b) * c.N + k;
  if (tid == 0) {
    mb = member_box(c, isl, P, k);
    ms.is_gal = GAL && c.has_gal && c.stype[isl * c.N + k] != 0;
    ms.support_half = ms.is_gal ? c.T / 2 : c.native / 2;
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
    ms.ncomp = rec->ncomp;
    ms.dndu = rec->dndu;
    for (int a = 0; a < 3; ++a) {
      ms.cg[a] = rec->cg[a];
      for (int q = 0; q < 3; ++q) ms.dcov[a][q] = rec->dcov[a][q];
    }
  }
  if (tid < 7) {
    ms.Lx[tid] = rec->Lx[tid];
    ms.dLx[tid] = rec->dLx[tid];
    ms.Ly[tid] = rec->Ly[tid];
    ms.dLy[tid] = rec->dLy[tid];
  }
  if (c.mode == 0) {
    for (int tt = tid; tt < c.nt; tt += blockDim.x) {
      ms.beta[tt] = rec->beta[tt];
      ms.betax[tt] = rec->betax[tt];
      ms.betay[tt] = rec->betay[tt];
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
  float* S = smem;   // nsa * UPH_HALO * HP; the x pass overwrites it in place
  const int T = c.T, c0 = c.T / 2;
  const int hs = ms.support_half;
  // halo rectangle intersected with the support box (offsets from centre)
  const int ylo = max(si0 - 3, max(0, c0 - hs)) - c0;
  const int yhi = min(si0 + oh + 2, min(T - 1, c0 + hs)) - c0;
  const int xlo = max(sj0 - 3, max(0, c0 - hs)) - c0;
  const int xhi = min(sj0 + ow + 2, min(T - 1, c0 + hs)) - c0;
  bool empty = (ylo > yhi) || (xlo > xhi);
  if (!empty && c.mode == 1) {
    if (tid == 0) ms.nact = 0;
    __syncthreads();
    for (int q = tid; q < ms.ncomp; q += blockDim.x) {
      const GComp& o = rec->comps[q];
      ms.act[q] = qmin_box(o.ia, o.ib, o.ic, (float)xlo, (float)xhi, (float)ylo,
                           (float)yhi) <= QCUT;
    }
    __syncthreads();
    if (tid == 0) {
      int na = 0;
      for (int q = 0; q < ms.ncomp; ++q)
        if (ms.act[q]) ms.act[na++] = (uint8_t)q;
      ms.nact = na;
    }
    __syncthreads();
    empty = (ms.nact == 0);
  }
  // analytic records: 0 derivative rows (trial), 2 (star: x, y) or 6
  // (galaxies: x, y, three shape rows, and the Sersic-index row only when
  // the index is live)
  int nout = 0;
  const bool is_gal = GAL && ms.is_gal;
  if (lin) nout = is_gal ? (ms.need[6] ? 6 : 5) : ((ms.need[1] || ms.need[2]) ? 2 : 0);
  if (tid == 0 && c.work) {
    // algorithmic work of this tile: the stamp rows written; on the tile's
    // pixels inside the member's support, per Gaussian term that reaches the
    // tile (analytic) one exponential and 4 + 4 nout FP32 multiply-adds, or
    // (pixelised PSF) the polynomial per needed S array; then 7 + 7
    // multiply-adds per shifted S array and pixel for the Lanczos passes
    int rows = 1;
    if (lin)
      for (int j = 0; j < 6; ++j) rows += ms.live_row[j] != 0;
    unsigned long long flops = 0, exps = 0;
    if (!empty) {
      const int sy = min(si0 + oh, c0 + hs + 1) - max(si0, c0 - hs);
      const int sx = min(sj0 + ow, c0 + hs + 1) - max(sj0, c0 - hs);
      const unsigned long long sup = (unsigned long long)max(sy, 0) * max(sx, 0);
      int nsarr = 0;
      for (int q = 0; q < NS; ++q) nsarr += (q == 0 || ms.need[q]) ? 1 : 0;
      if (c.mode == 1) {
        exps = sup * (unsigned long long)ms.nact;
        flops = exps * 2ull * (4 + 4 * nout);
      } else if (!is_gal) {
        flops = sup * 2ull * c.nt * (unsigned long long)nsarr;
      }
      // shifted arrays: S and its partials, plus the tap derivatives of the
      // position rows
      const int nshift = nsarr + (ms.live_row[0] ? 1 : 0) + (ms.live_row[1] ? 1 : 0);
      flops += 28ull * (unsigned long long)(oh * ow) * nshift;
    }
    work_add(c, WK_RENDER, 4ull * (unsigned long long)(oh * ow * rows), flops, exps);
  }
  if (!empty && c.mode == 1) {
    for (int a = tid; a < ms.nact; a += blockDim.x) {
      const GComp& o = rec->comps[ms.act[a]];
      float4* r = trec + a * (nout + 1);
      r[0] = make_float4(KEXP * o.ia, 2.f * KEXP * o.ib, KEXP * o.ic, o.nrm);
      if (nout == 0) continue;
      const float i2d = o.det;   // holds 0.5 / det
      // dA, dC, dB of the covariance-derivative chain as quadratic forms
      const float4 PA = make_float4(i2d * o.C * o.ia, i2d * 2.f * o.C * o.ib,
                                    i2d * (o.C * o.ic - 1.f), -i2d * o.C);
      const float4 PC = make_float4(i2d * (o.A * o.ia - 1.f), i2d * 2.f * o.A * o.ib,
                                    i2d * o.A * o.ic, -i2d * o.A);
      const float t2 = 2.f * i2d;
      const float4 PB = make_float4(-t2 * o.B * o.ia, t2 * (1.f - 2.f * o.B * o.ib),
                                    -t2 * o.B * o.ic, t2 * o.B);
      auto comb = [&](float wa, float wc, float wb, float s, float add) {
        return make_float4(s * (wa * PA.x + wc * PC.x + wb * PB.x),
                           s * (wa * PA.y + wc * PC.y + wb * PB.y),
                           s * (wa * PA.z + wc * PC.z + wb * PB.z),
                           s * (wa * PA.w + wc * PC.w + wb * PB.w) + add);
      };
      r[1] = comb(o.dAx, o.dCx, o.dBx, o.nrm, o.nx);
      r[2] = comb(o.dAy, o.dCy, o.dBy, o.nrm, o.ny);
      if (GAL && nout >= 5) {
        const float nv = o.nrm * o.v;
        for (int q = 0; q < 3; ++q)
          r[3 + q] = comb(ms.dcov[q][0], ms.dcov[q][1], ms.dcov[q][2], nv, 0.f);
      }
      if (GAL && nout == 6) {
        const float4 u = comb(ms.cg[0], ms.cg[1], ms.cg[2], o.nrm * o.dv, o.nu);
        r[6] = make_float4(ms.dndu * u.x, ms.dndu * u.y, ms.dndu * u.z, ms.dndu * u.w);
      }
    }
    __syncthreads();
  }
  if (empty) {
    // every value on this tile is zero: write the zeros and stop
    for (int e = tid; e < oh * ow; e += blockDim.x) {
      const int rr = e / ow, cc = e % ow;
      const size_t off = (size_t)(oy0 + rr - mb.wy0) * c.Sz + (ox0 + cc - mb.wx0);
      c.stamps[stamp_slot(c, isl, b, k, 0) + off] = 0.f;
      if (lin)
        for (int j = 0; j < 6; ++j)
          if (ms.live_row[j]) c.stamps[stamp_slot(c, isl, b, k, ms.live_row[j]) + off] = 0.f;
    }
    return;
  }

  // ---- un-shifted stamp (and partials) on the halo region ----
  const int nh = hr * hc;
  if (c.mode == 0 && is_gal) {
    // reference-mode galaxy: the unshifted rows from the Fourier-domain
    // convolution (k_gal_fft)
    const float* gs = c.gstamp + (((size_t)isl * c.nb + b) * c.N + k) * 7 * (size_t)(T * T);
    for (int e = tid; e < nh; e += blockDim.x) {
      const int r = e / hc, cc = e % hc;
      const int si = si0 - 3 + r, sj = sj0 - 3 + cc;
      const bool ok = si >= 0 && si < T && sj >= 0 && sj < T;
      const size_t o = (size_t)si * T + sj;
      for (int q = 0; q < NS; ++q)
        if (q == 0 || ms.need[q])
          S[(q * UPH_HALO + r) * HP + cc] = ok ? gs[(size_t)q * T * T + o] : 0.f;
    }
  } else if (c.mode == 0) {
    for (int e = tid; e < nh; e += blockDim.x) {
      const int r = e / hc, cc = e % hc;
      const int si = si0 - 3 + r, sj = sj0 - 3 + cc;
      float v0 = 0.f, v1 = 0.f, v2 = 0.f;
      if (si >= 0 && si < T && sj >= 0 && sj < T && abs(si - c0) <= hs &&
          abs(sj - c0) <= hs) {
        const float* cf = c.psf_coefs + (((size_t)b * T + si) * T + sj) * c.nt;
        for (int tt = 0; tt < c.nt; ++tt) {
          const float cv = cf[tt];
          v0 = fmaf(cv, ms.beta[tt], v0);
          v1 = fmaf(cv, ms.betax[tt], v1);
          v2 = fmaf(cv, ms.betay[tt], v2);
        }
      }
      S[(0 * UPH_HALO + r) * HP + cc] = v0;
      if (ms.need[1]) S[(1 * UPH_HALO + r) * HP + cc] = v1;
      if (ms.need[2]) S[(2 * UPH_HALO + r) * HP + cc] = v2;
    }
  } else {
    // halo pixels outside the member's support (and outside the stamp) are
    // zero: clear them, then evaluate only the support rectangle
    // [ylo, yhi] x [xlo, xhi] (offsets from the stamp centre), two pixels
    // per thread sharing every component record
    const int ry0 = ylo + c0 - (si0 - 3), rx0 = xlo + c0 - (sj0 - 3);
    const int rh = yhi - ylo + 1, rw = xhi - xlo + 1;
    const int nr = rh * rw;
    for (int e = tid; e < nh; e += blockDim.x) {
      const int r = e / hc, cc = e - r * hc;
      if (r >= ry0 && r < ry0 + rh && cc >= rx0 && cc < rx0 + rw) continue;
      S[(0 * UPH_HALO + r) * HP + cc] = 0.f;
      for (int q = 1; q <= nout; ++q)
        if (ms.need[q]) S[(q * UPH_HALO + r) * HP + cc] = 0.f;
    }
    const int step = 2 * blockDim.x;
    for (int e0 = tid; e0 < nr; e0 += step) {
      const int e1 = e0 + blockDim.x;
      float x2[2], xy[2], y2[2];
      int rr[2], cs[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int e = min(h ? e1 : e0, nr - 1);
        const int ry = e / rw, rx = e - ry * rw;
        rr[h] = ry0 + ry;
        cs[h] = rx0 + rx;
        const float xo = (float)(xlo + rx), yo = (float)(ylo + ry);
        x2[h] = xo * xo;
        xy[h] = xo * yo;
        y2[h] = yo * yo;
      }
      float va[NS], vb[NS];
      if (GAL && nout == 6)
        mog_pair<6>(trec, ms.nact, x2[0], xy[0], y2[0], x2[1], xy[1], y2[1], va, vb);
      else if (GAL && nout == 5)
        mog_pair<5>(trec, ms.nact, x2[0], xy[0], y2[0], x2[1], xy[1], y2[1], va, vb);
      else if (nout == 2)
        mog_pair<2>(trec, ms.nact, x2[0], xy[0], y2[0], x2[1], xy[1], y2[1], va, vb);
      else
        mog_pair<0>(trec, ms.nact, x2[0], xy[0], y2[0], x2[1], xy[1], y2[1], va, vb);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if ((h ? e1 : e0) >= nr) continue;
        const float* v = h ? vb : va;
        const int r = rr[h], cc = cs[h];
        S[(0 * UPH_HALO + r) * HP + cc] = v[0];
        for (int q = 1; q <= nout; ++q)
          if (ms.need[q]) S[(q * UPH_HALO + r) * HP + cc] = v[q];
      }
    }
  }
  __syncthreads();

  // ---- x pass, in place: X0 = cx(S,L), X1 = cx(S,dL) + cx(Sx,L),
  //      X2 = cx(Sy,L), X3..5 = cx(S_shape,L), X6 = cx(Su,L).  One warp per
  //      halo row (lane = output column): a row's outputs depend only on that
  //      row, so the warp reads all of it, syncs, then overwrites it ----
  {
    const bool dox = ms.live_row[0] != 0;
    const int lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    for (int r = warp; r < hr; r += nw) {
      float xv[NS];
      const int cc = lane;
      if (cc < ow) {
        const float* s0 = S + (0 * UPH_HALO + r) * HP + cc;
        float a0 = ms.Lx[0] * s0[0];
        for (int q = 1; q < 7; ++q) a0 = fmaf(ms.Lx[q], s0[q], a0);
        xv[0] = a0;
        if (dox) {
          float a1 = ms.dLx[0] * s0[0];
          for (int q = 1; q < 7; ++q) a1 = fmaf(ms.dLx[q], s0[q], a1);
          if (ms.need[1]) {
            const float* s1 = S + (1 * UPH_HALO + r) * HP + cc;
            float b1 = ms.Lx[0] * s1[0];
            for (int q = 1; q < 7; ++q) b1 = fmaf(ms.Lx[q], s1[q], b1);
            a1 += b1;
          }
          xv[1] = a1;
        }
#pragma unroll
        for (int sa = 2; sa < (GAL ? NS : 3); ++sa) {
          if (!ms.need[sa]) continue;
          const float* sp = S + (sa * UPH_HALO + r) * HP + cc;
          float a = ms.Lx[0] * sp[0];
          for (int q = 1; q < 7; ++q) a = fmaf(ms.Lx[q], sp[q], a);
          xv[sa] = a;
        }
      }
      __syncwarp();
      if (cc < ow) {
        S[(0 * UPH_HALO + r) * HP + cc] = xv[0];
        if (dox) S[(1 * UPH_HALO + r) * HP + cc] = xv[1];
#pragma unroll
        for (int sa = 2; sa < (GAL ? NS : 3); ++sa)
          if (ms.need[sa]) S[(sa * UPH_HALO + r) * HP + cc] = xv[sa];
      }
      __syncwarp();
    }
  }
  __syncthreads();

  // ---- y pass and store ----
  const int Sz = c.Sz;
  for (int e = tid; e < oh * ow; e += blockDim.x) {
    const int rr = e / ow, cc = e % ow;
    const int wy = oy0 + rr, wx = ox0 + cc;
    const size_t off = (size_t)(wy - mb.wy0) * Sz + (wx - mb.wx0);
    const float* x0 = S + (0 * UPH_HALO + rr) * HP + cc;
    float m = ms.Ly[0] * x0[0];
    for (int q = 1; q < 7; ++q) m = fmaf(ms.Ly[q], x0[q * HP], m);
    c.stamps[stamp_slot(c, isl, b, k, 0) + off] = m;
    if (!lin) continue;
    if (ms.live_row[0]) {
      const float* x1 = S + (1 * UPH_HALO + rr) * HP + cc;
      float d = ms.Ly[0] * x1[0];
      for (int q = 1; q < 7; ++q) d = fmaf(ms.Ly[q], x1[q * HP], d);
      c.stamps[stamp_slot(c, isl, b, k, ms.live_row[0]) + off] = d;
    }
    if (ms.live_row[1]) {
      float d = ms.dLy[0] * x0[0];
      for (int q = 1; q < 7; ++q) d = fmaf(ms.dLy[q], x0[q * HP], d);
      if (ms.need[2]) {
        const float* x2 = S + (2 * UPH_HALO + rr) * HP + cc;
        float d2 = ms.Ly[0] * x2[0];
        for (int q = 1; q < 7; ++q) d2 = fmaf(ms.Ly[q], x2[q * HP], d2);
        d += d2;
      }
      c.stamps[stamp_slot(c, isl, b, k, ms.live_row[1]) + off] = d;
    }
    for (int j = 2; j < (GAL ? 6 : 2); ++j) {
      if (!ms.live_row[j]) continue;
      const int s = j + 1;  // S arrays 3..6 hold lr, e1, e2, u
      const float* xs = S + (s * UPH_HALO + rr) * HP + cc;
      float d = ms.Ly[0] * xs[0];
      for (int q = 1; q < 7; ++q) d = fmaf(ms.Ly[q], xs[q * HP], d);
      c.stamps[stamp_slot(c, isl, b, k, ms.live_row[j]) + off] = d;
    }
  }
}

// The linearisation render at the compiler's own register choice (61, four
// CTAs per SM, the shared-memory limit too); the trial render (model row
// only) held to 32 registers for eight CTAs per SM (a 20-byte spill; the
// solve measured faster at each step from four to eight CTAs).
__global__ void __launch_bounds__(256) k_render_lin(ClassDev c, const float* __restrict__ P,
                                                    int phase) {
  render_body<true>(c, P, phase, blockIdx.x);
}

// The linearisation render of chunks without galaxies: the galaxy paths
// compiled out, three stamp arrays, and an occupancy bound.
__global__ void __launch_bounds__(256, RENDER_LIN_STAR_CTAS) k_render_lin_star(
    ClassDev c, const float* __restrict__ P, int phase) {
  render_body<true, false>(c, P, phase, blockIdx.x);
}

__global__ void __launch_bounds__(256, 8) k_render_trial(ClassDev c,
                                                         const float* __restrict__ P,
                                                         int phase) {
  render_body<false>(c, P, phase, blockIdx.x);
}

// Queue kernels of the LM loop: the member set-up and the render of every
// active island of the job (P = the chunk's p, or p_try for the trial point).
__global__ void __launch_bounds__(128) kq_member_setup(QueueList q, int phase, int p_try) {
  queue_run(q, QK_SETUP, 8, [&](const ClassDev& c, int isl, int u) {
    // unit u: the island's records 4u .. 4u + 3
    const int nr = c.nb * c.N;
    member_setup_body(c, p_try ? c.p_try : c.p, phase, isl * nr + SETUP_WARPS * u,
                      min(SETUP_WARPS, nr - SETUP_WARPS * u));
    return false;
  });
}

// (three resident CTAs per SM, as the per-chunk linearisation render's
// shared memory allows: the descriptor fields then stay in shared memory
// instead of registers)
template <bool LIN>
__global__ void __launch_bounds__(256, 3) kq_render(QueueList q, int phase, int p_try) {
  queue_run(q, QK_RENDER, 4, [&](const ClassDev& c, int isl, int u) {
    render_body<LIN>(c, p_try ? c.p_try : c.p, phase,
                     isl * c.nb * c.N * c.ntile_side * c.ntile_side + u);
    return false;
  });
}

}  // namespace

// Resident CTAs of kernel f on every SM at `smem` dynamic bytes (at least
// one per SM).
template <class F>
static unsigned queue_grid(F f, int threads, size_t smem, int sms, int cap, int per_cta) {
  if (cap <= 0) return 1;
  if (per_cta) return (unsigned)cap;
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, f, threads, smem) != cudaSuccess ||
      per < 1)
    per = 1;
  return (unsigned)std::max(1, std::min(per * sms, cap));
}

void launch_q_setup(const QueueList& q, int phase, bool p_try, int sms, cudaStream_t s) {
  kq_member_setup<<<queue_grid(kq_member_setup, 128, 0, sms, q.cap[QK_SETUP], q.per_cta), 128, 0, s>>>(
      q, phase, p_try);
}

void launch_q_render(const QueueList& q, int phase, bool lin, bool p_try, size_t render_smem,
                     int sms, cudaStream_t s) {
  if (lin)
    kq_render<true><<<queue_grid(kq_render<true>, 256, render_smem, sms, q.cap[QK_RENDER], q.per_cta), 256,
                      render_smem, s>>>(q, phase, p_try);
  else
    kq_render<false><<<queue_grid(kq_render<false>, 256, render_smem, sms, q.cap[QK_RENDER], q.per_cta),
                       256, render_smem, s>>>(q, phase, p_try);
}

size_t render_smem_bytes() {
  return sizeof(float) * (size_t)NS * UPH_HALO * HP;
}

// Shared arrays a launch needs: every S/X slot index used by the phase is
// below this count (trial renders use S only; star classes S, Sx, Sy).
static int render_arrays(const ClassDev& c, int phase) {
  if (phase != PH_LIN) return 1;
  return c.has_gal ? NS : 3;
}

size_t render_phase_smem(const ClassDev& c, int phase) {
  return sizeof(float) * (size_t)render_arrays(c, phase) * UPH_HALO * HP;
}

void launch_render(const ClassDev& c, const float* P, int phase,
                   cudaStream_t s) {
  const long long nblk = (long long)c.n_isl * c.nb * c.N * c.ntile_side * c.ntile_side;
  if (nblk <= 0) return;
  const int nsa = render_arrays(c, phase);
  const size_t bytes = sizeof(float) * (size_t)nsa * UPH_HALO * HP;
  const long long nrec = (long long)c.n_isl * c.nb * c.N;
  k_member_setup<<<(unsigned)((nrec + SETUP_WARPS - 1) / SETUP_WARPS), 32 * SETUP_WARPS, 0, s>>>(
      c, P, phase);
  if (c.mode == 0 && c.gstamp) launch_gal_fft(c, P, phase, s);
  if (phase == PH_LIN && !c.has_gal)
    k_render_lin_star<<<(unsigned)nblk, 256, bytes, s>>>(c, P, phase);
  else if (phase == PH_LIN)
    k_render_lin<<<(unsigned)nblk, 256, bytes, s>>>(c, P, phase);
  else
    k_render_trial<<<(unsigned)nblk, 256, bytes, s>>>(c, P, phase);
}

int uph_render_setup() {
  cudaError_t e = cudaFuncSetAttribute(k_render_lin,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)render_smem_bytes());
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(kq_render<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)render_smem_bytes());
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(kq_render<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)render_smem_bytes());
  if (e != cudaSuccess) return (int)e;
  return (int)cudaFuncSetAttribute(k_render_trial,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)render_smem_bytes());
}

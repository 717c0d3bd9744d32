// Pixel passes and small dense algebra of the VarPro-LM step.
//
// k_gram_lin   -- weighted Gram G = Z W Z^T of the rows
//                 Z = [dm/dtheta (nL) ; m (nr) ; data (1)] over the island
//                 window of one band (FP32 CUDA cores, fixed-order
//                 deterministic reduction).
// k_assemble   -- from G: the f64 VarPro flux solve and the exact
//                 Golub-Pereyra Gauss-Newton blocks
//                   J_i = -W^1/2 (f_k D_i + M^T c_i),
//                   c_i = A64^-1 (e_k s_i - f_k u_i),
//                   s_i = D_i^T W (d - M^T f),  u_i = M W D_i,
//                 i.e. H_b = J J^T and g_b = J r without materialising J
//                 (the reference pushes tangents through jax.linearize,
//                 island_solver.py:812-865).
// k_gram_trial -- trial chi2: flux solve on [m; data] then the whitened
//                 residual pass r = sqrt(w)(d - sum_k f_k m_k)
//                 (island_solver.py:570-605, 668-684); also final fluxes and
//                 sqrt(diag inv A64) (island_solver.py:1467-1482).
// k_step       -- band sum, keep mask, damping, f64 LU solve, clips, box
//                 bounds (island_solver.py:921-967).
// k_accept     -- accept/reject, lambda update, three convergence prongs
//                 (island_solver.py:968-1002).
#include <algorithm>

#include "uph_internal.cuh"

namespace {

constexpr int NT = 256;

__device__ __forceinline__ void decode_upper(int idx, int nbk, int& bi,
                                             int& bj) {
  int row = 0;
  while (idx >= nbk - row) {
    idx -= nbk - row;
    ++row;
  }
  bi = row;
  bj = row + idx;
}

// Shared pixel loop: accumulates the Gram of K rows (row descriptors in
// rk/rs, member boxes in box) over the B x B window of band b, writing the
// full K x K result to out (pitch ld).  Used by both Gram kernels.
struct RowSrc {
  const int16_t* rk;
  const int16_t* rs;
  int K;
  const float* fc = nullptr;   // residual form: linear solution (stride-NL layout)
  int nr = 0;                  // member model rows
  int nbg = 0;                 // background rows after them
  int N = 0;                   // slot of background coefficient j in fc: N + j
};

// Value of Gram row r at window pixel (wy, wx), already scaled by sqrt(w).
// The last row is the data, or in residual form (fc set) the residual
// d - sum_k fc_k m_k, summed in member order as the trial pass does.
template <bool BG>
__device__ __forceinline__ float row_value(const ClassDev& c, int isl, int b,
                                           const RowSrc& rows, const int4* box,
                                           int r, int wy, int wx, float sw,
                                           const float* dbase) {
  const int rs = rows.rs[r];
  if (BG && rs <= -2) return bg_basis(-2 - rs, wy, wx, c.B) * sw;
  if (rs < 0) {
    const float d = dbase[(size_t)wy * c.Wp + wx];
    if (!rows.fc) return d * sw;
    float model = 0.f;
    for (int k = 0; k < rows.nr; ++k) {
      const int4 bx = box[k];
      const int ly = wy - bx.y, lx = wx - bx.x;
      if (ly >= 0 && ly < bx.w && lx >= 0 && lx < bx.z)
        model = fmaf(rows.fc[k], c.stamps[stamp_slot(c, isl, b, k, 0) + (size_t)ly * c.Sz + lx],
                     model);
    }
    if (BG)
      for (int j = 0; j < rows.nbg; ++j)
        model = fmaf(rows.fc[rows.N + j], bg_basis(j, wy, wx, c.B), model);
    return sw * (d - model);
  }
  const int k = rows.rk[r];
  const int4 bx = box[k];
  const int ly = wy - bx.y, lx = wx - bx.x;
  if (ly >= 0 && ly < bx.w && lx >= 0 && lx < bx.z)
    return c.stamps[stamp_slot(c, isl, b, k, rs) + (size_t)ly * c.Sz + lx] * sw;
  return 0.f;
}

// Small-K path (K <= 8): every thread accumulates the packed upper triangle
// of its own pixels in registers; warp-shuffle + fixed-order block reduction.
template <bool BG>
__device__ void gram_window_small(const ClassDev& c, int isl, int b,
                                  const RowSrc& rows, const int4* box,
                                  float* out, int ld, float* sm) {
  const int tid = threadIdx.x;
  const int K = rows.K;
  const int B = c.B;
  const int npix = B * B;
  const size_t plane = (size_t)c.Hp * c.Wp;
  const float* dbase = c.dstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
  const float* wbase = c.wstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
  float acc[36];
#pragma unroll
  for (int e = 0; e < 36; ++e) acc[e] = 0.f;
  for (int pix = tid; pix < npix; pix += NT) {
    const int wy = pix / B, wx = pix - (pix / B) * B;
    const float sw = sqrtf(wbase[(size_t)wy * c.Wp + wx]);
    float z[8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
      z[r] = (r < K) ? row_value<BG>(c, isl, b, rows, box, r, wy, wx, sw, dbase) : 0.f;
    int e = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = i; j < 8; ++j) {
        acc[e] = fmaf(z[i], z[j], acc[e]);
        ++e;
      }
  }
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int e = 0; e < 36; ++e) {
    float v = acc[e];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    acc[e] = v;
  }
  if (lane == 0)
    for (int e = 0; e < 36; ++e) sm[warp * 36 + e] = acc[e];
  __syncthreads();
  if (tid < 36) {
    float t = 0.f;
    for (int w = 0; w < NT / 32; ++w) t += sm[w * 36 + tid];
    int i = 0, rem = tid;
    while (rem >= 8 - i) {
      rem -= 8 - i;
      ++i;
    }
    const int j = i + rem;
    if (i < K && j < K) {
      out[i * ld + j] = t;
      out[j * ld + i] = t;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;"
               :
               : "r"(d), "l"(src), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// Pixel-tile geometry of the tiled Gram path for K rows.
__host__ __device__ __forceinline__ int gram_tile_pixels(int K) {
  return (K <= 32) ? 128 : (K <= 96 ? 64 : 32);
}

// Stage pixels [pix0, pix0 + TP) of rows 0..K-1 UNWEIGHTED (stamp values,
// data; zero outside a member's box) into Z (pitch LD) and the raw weights
// into Wt, by 4-byte cp.async (one commit group).  Rows K..nrows-1 are not
// touched: the caller zeroes them once.
template <bool BG>
__device__ __forceinline__ void stage_rows(const ClassDev& c, int isl, int b,
                                           const RowSrc& rows, const int4* box,
                                           float* Z, float* Wt, int pix0, int TP,
                                           int lgTP, int LD, int nrows) {
  const int tid = threadIdx.x;
  const int K = rows.K, B = c.B, npix = B * B;
  const float invB = 1.0f / (float)B;
  const size_t plane = (size_t)c.Hp * c.Wp;
  const float* dbase = c.dstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
  const float* wbase = c.wstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
  for (int e = tid; e < K * TP; e += blockDim.x) {
    const int r = e >> lgTP, q = e & (TP - 1);
    const int pix = pix0 + q;
    const float* src = dbase;
    bool ok = false;
    if (pix < npix) {
      const int wy = (int)(((float)pix + 0.5f) * invB);
      const int wx = pix - wy * B;
      const int rs = rows.rs[r];
      if (BG && rs <= -2) {
        // background basis: computed, not copied
        Z[r * LD + q] = bg_basis(-2 - rs, wy, wx, B);
        continue;
      } else if (rs < 0) {
        src = dbase + (size_t)wy * c.Wp + wx;
        ok = true;
      } else {
        const int k = rows.rk[r];
        const int4 bx = box[k];
        const int ly = wy - bx.y, lx = wx - bx.x;
        if (ly >= 0 && ly < bx.w && lx >= 0 && lx < bx.z) {
          src = c.stamps + stamp_slot(c, isl, b, k, rs) + (size_t)ly * c.Sz + lx;
          ok = true;
        }
      }
    }
    cp_async4(Z + r * LD + q, src, ok);
  }
  for (int q = tid; q < TP; q += blockDim.x) {
    const int pix = pix0 + q;
    const float* src = wbase;
    bool ok = false;
    if (pix < npix) {
      const int wy = (int)(((float)pix + 0.5f) * invB);
      src = wbase + (size_t)wy * c.Wp + (pix - wy * B);
      ok = true;
    }
    cp_async4(Wt + q, src, ok);
  }
  cp_async_commit();
}

__host__ __device__ __forceinline__ int log2_tile(int TP) {
  return (TP == 128) ? 7 : (TP == 64 ? 6 : 5);
}

// Dynamic shared floats the staged tiles of K rows use: two tiles of
// ceil8(K) rows x (TP + 1), two weight rows, the cross-warp partials.
__host__ __device__ __forceinline__ int tile_floats(int K) {
  const int nrows = ((K + 7) / 8) * 8;
  const int TP = gram_tile_pixels(K);
  return 2 * nrows * (TP + 1) + 2 * TP + (NT / 32) * 64;
}

__device__ __forceinline__ unsigned dynamic_smem_bytes() {
  unsigned v;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(v));
  return v;
}

// Tiled path (K > 8): the rows are staged UNWEIGHTED -- stamp values, data
// (zero outside a member's box) and the raw weights -- by 4-byte cp.async
// into double-buffered shared tiles, so the copies of tile t + 1 are in
// flight while tile t is consumed; the weight enters the product
// (sum_pix w z_i z_j).  In residual form the last row is rebuilt from the
// staged model rows once a tile has landed (d - sum_k fc_k m_k in member
// order, the trial pass's order).  Each thread accumulates one 8 x 8 block
// of the upper triangle over its share of the pixels; the s threads sharing
// a block are s consecutive lanes (s a power of two), reduced by shuffles in
// a fixed order, and through a small shared buffer when s > 32.
// sp / nsp: this CTA's share of the window's pixel tiles (contiguous, in
// order), for a Gram split over nsp CTAs whose partial Grams are summed
// afterwards; the small path (K <= 8) runs whole in split 0.  SMALL: the
// caller guarantees K <= 8, and the tiled path (its 8 x 8 register blocks)
// is not compiled in, so the kernel keeps few registers.
template <bool BG, bool SMALL = false>
__device__ void gram_window(const ClassDev& c, int isl, int b, RowSrc rows,
                            const int4* box, float* out, int ld, int part,
                            float* sm, int sp = 0, int nsp = 1) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int K = rows.K;
  if (SMALL || K <= 8) {
    if (part == 0 && sp == 0) gram_window_small<BG>(c, isl, b, rows, box, out, ld, sm);
    return;
  }
  if (sizeof(float) * (size_t)tile_floats(K) > dynamic_smem_bytes()) {
    // launched with too little shared memory for these tiles: report, skip
    if (threadIdx.x == 0 && c.err) atomicExch(c.err, 2);
    return;
  }
  const int nbk = (K + 7) / 8;
  const int nblk = nbk * (nbk + 1) / 2;
  int s, my, split;
  if (nblk <= NT) {
    s = 1;
    while (2 * s * nblk <= NT) s *= 2;
    my = tid / s;
    split = tid - my * s;
    if (my >= nblk) my = -1;
  } else {
    s = 1;
    my = part * NT + tid;
    split = 0;
    if (my >= nblk) my = -1;
  }
  int bi = 0, bj = 0;
  if (my >= 0) decode_upper(my, nbk, bi, bj);
  const int TP = gram_tile_pixels(K);
  const int lgTP = log2_tile(TP);
  const int LD = TP + 1;
  const int nrows = nbk * 8;
  // buffers: Z0 Z1 (nrows x LD each), W0 W1 (TP each), red ((NT / 32) x 64)
  float* red = sm + 2 * nrows * LD + 2 * TP;
  const int npix = c.B * c.B;
  const int nlin = rows.nr + rows.nbg;
  const int m0 = K - 1 - nlin;      // first linear row (residual form)
  auto stage = [&](int pix0, int bufi) {
    stage_rows<BG>(c, isl, b, rows, box, sm + bufi * nrows * LD,
               sm + 2 * nrows * LD + bufi * TP, pix0, TP, lgTP, LD, nrows);
  };

  float acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
  const int ntall = (npix + TP - 1) / TP;
  const int tps = (ntall + nsp - 1) / nsp;        // tiles per split
  const int t0 = sp * tps;
  const int ntile = min(ntall, t0 + tps);
  // padding rows K..nrows-1 of both tiles stay zero for the whole pass
  for (int e = tid; e < (nrows - K) * LD; e += NT) {
    sm[K * LD + e] = 0.f;
    sm[nrows * LD + K * LD + e] = 0.f;
  }
  __syncthreads();
  if (t0 < ntile) stage(t0 * TP, 0);
  for (int t = t0; t < ntile; ++t) {
    const int cur = (t - t0) & 1;
    cp_async_wait_all();
    __syncthreads();
    float* Z = sm + cur * nrows * LD;
    const float* Wt = sm + 2 * nrows * LD + cur * TP;
    if (rows.fc) {
      // residual row from the staged model rows
      for (int q = tid; q < TP; q += NT) {
        float model = 0.f;
        for (int k = 0; k < rows.nr; ++k) model = fmaf(rows.fc[k], Z[(m0 + k) * LD + q], model);
        if (BG)
          for (int j = 0; j < rows.nbg; ++j)
            model = fmaf(rows.fc[rows.N + j], Z[(m0 + rows.nr + j) * LD + q], model);
        Z[(K - 1) * LD + q] = Z[(K - 1) * LD + q] - model;
      }
      __syncthreads();
    }
    if (t + 1 < ntile) stage((t + 1) * TP, cur ^ 1);
    if (my >= 0) {
      const float* za = Z + bi * 8 * LD;
      const float* zb = Z + bj * 8 * LD;
      for (int q = split; q < TP; q += s) {
        const float w = Wt[q];
        float a[8], bb[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          a[i] = za[i * LD + q];
          bb[i] = zb[i * LD + q] * w;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], bb[j], acc[i][j]);
      }
    }
  }
  // fixed-order reduction over the s pixel splits of each block
  const int sw = s < 32 ? s : 32;
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      float v = acc[i][j];
      for (int o = 1; o < sw; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      acc[i][j] = v;
    }
  if (s > 32) {
    // one partial per warp; warps of a block are consecutive
    __syncthreads();
    if (lane == 0) {
#pragma unroll
      for (int e = 0; e < 64; ++e) red[warp * 64 + e] = acc[e >> 3][e & 7];
    }
    __syncthreads();
    if (my >= 0 && split == 0) {
      const int w0 = (my * s) >> 5, nw = s >> 5;
#pragma unroll
      for (int e = 0; e < 64; ++e) {
        float t = red[w0 * 64 + e];
        for (int w = 1; w < nw; ++w) t += red[(w0 + w) * 64 + e];
        acc[e >> 3][e & 7] = t;
      }
    }
  }
  if (my >= 0 && split == 0) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int gi = bi * 8 + i;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int gj = bj * 8 + j;
        if (gi < K && gj < K) {
          out[gi * ld + gj] = acc[i][j];
          out[gj * ld + gi] = acc[i][j];
        }
      }
    }
  }
  __syncthreads();
}

__device__ void load_boxes(const ClassDev& c, int isl, const float* P,
                           int4* box) {
  for (int k = threadIdx.x; k < c.N; k += blockDim.x) {
    MemberBox mb = member_box(c, isl, P, k);
    box[k] = make_int4(mb.wx0, mb.wy0, mb.bw, mb.bh);
  }
}

template <bool BG, bool SMALL = false>
__device__ __forceinline__ void gram_lin_body(const ClassDev& c, int bx, int by) {
  extern __shared__ float sm[];
  __shared__ int4 box[UPH_MAXN];
  const int isl = bx / c.nb, b = bx % c.nb;
  if (isl >= c.n_isl || !isl_active(c.flags[isl], PH_LIN)) return;
  const int nr = c.isl_nr[isl];
  const int K = gram_K(c, isl);
  if (tc_island(c, isl, K)) return;  // the tensor-core Gram handles this island
  // by = block set + parts x pixel split
  const int parts = gram_lin_parts(c.Kmax);
  const int part = by % parts, sp = by / parts;
  const int nsp = c.gl_split > 1 ? c.gl_split : 1;
  const int nbk = (K + 7) / 8;
  const int nblk = nbk * (nbk + 1) / 2;
  if (part * NT >= max(nblk, 1) && part > 0) return;
  if (nblk <= NT && part > 0) return;
  load_boxes(c, isl, c.p, box);
  __syncthreads();
  if (threadIdx.x == 0 && by == 0)
    gram_work(c, WK_GRAM, c.row_k + (size_t)isl * c.Kmax, c.row_s + (size_t)isl * c.Kmax,
              K, box);
  // the mixed form forms every Gram in residual form (k_assemble matches)
  RowSrc rows{c.row_k + (size_t)isl * c.Kmax, c.row_s + (size_t)isl * c.Kmax, K,
              c.fcur ? c.fcur + ((size_t)isl * c.nb + b) * c.NL : nullptr, nr, c.nbg, c.N};
  const size_t mat = (size_t)c.Kmax * c.Kmax;
  float* out = nsp > 1 ? c.glpart + (size_t)sp * c.n_isl * c.nb * mat
                       : c.gram;
  gram_window<BG, SMALL>(c, isl, b, rows, box, out + ((size_t)isl * c.nb + b) * mat,
                         c.Kmax, part, sm, sp, nsp);
}

// Sum of the gl_split partial FP32 Grams of an (island, band), in split order
// (deterministic), into the chunk's Gram; a Gram of K <= 8 rows was formed
// whole by split 0.
__device__ __forceinline__ void gram_lin_reduce_body(const ClassDev& c, int bx) {
  const int isl = bx / c.nb, b = bx % c.nb;
  if (isl >= c.n_isl || !isl_active(c.flags[isl], PH_LIN)) return;
  const int K = gram_K(c, isl);
  if (tc_island(c, isl, K)) return;
  const size_t mat = (size_t)c.Kmax * c.Kmax;
  const size_t stride = (size_t)c.n_isl * c.nb * mat;
  const float* src = c.glpart + ((size_t)isl * c.nb + b) * mat;
  float* dst = c.gram + ((size_t)isl * c.nb + b) * mat;
  const int nsp = K <= 8 ? 1 : c.gl_split;
  for (int e = threadIdx.x; e < K * K; e += NT) {
    const int r = e / K, q = e - (e / K) * K;
    const size_t o = (size_t)r * c.Kmax + q;
    float t = src[o];
    for (int sp = 1; sp < nsp; ++sp) t += src[sp * stride + o];
    dst[o] = t;
  }
}

__global__ void __launch_bounds__(NT) k_gram_lin_reduce(ClassDev c) {
  gram_lin_reduce_body(c, blockIdx.x);
}

template <bool BG>
__global__ void __launch_bounds__(NT) k_gram_lin(ClassDev c) {
  gram_lin_body<BG>(c, blockIdx.x, blockIdx.y);
}

// Chunks whose Grams all have at most 8 rows (most singleton classes): the
// same work without the tiled path's registers (79 instead of 128: three
// CTAs per SM instead of two).
template <bool BG>
__global__ void __launch_bounds__(NT) k_gram_lin_small(ClassDev c) {
  gram_lin_body<BG, true>(c, blockIdx.x, blockIdx.y);
}

// Gauss-Jordan elimination with partial pivoting on M (n x ncol, pitch ld):
// turns the left n x n block into the identity; the remaining columns hold
// A^-1 [rhs].  All threads of the block participate.
//
// With diag (the matrix's original diagonal), cond and perm (n ints of
// shared scratch for the row order) non-null, thread 0
// also writes a conditioning indicator of the diagonally scaled matrix
// D^-1/2 A D^-1/2: the spread max/min of the pivots in that scaling (each
// pivot |M[p][col]| divided by sqrt(diag[row of p] diag[col])), 1 for a
// diagonal matrix and 1 / (1 - rho^2) for two members of correlation rho.
__device__ void gauss_jordan(double* M, int n, int ncol, int ld, double* fac,
                             int* piv, const double* diag = nullptr,
                             float* cond = nullptr, int* perm = nullptr) {
  const int tid = threadIdx.x;
  double rmin = INFINITY, rmax = 0.0;
  if (!perm) cond = nullptr;   // the indicator needs the caller's row-order scratch
  if (tid == 0 && cond)
    for (int r = 0; r < n; ++r) perm[r] = r;
  for (int col = 0; col < n; ++col) {
    if (tid == 0) {
      int p = col;
      double best = fabs(M[col * ld + col]);
      for (int r = col + 1; r < n; ++r) {
        double v = fabs(M[r * ld + col]);
        if (v > best) {
          best = v;
          p = r;
        }
      }
      *piv = p;
      if (cond) {
        const double sc = sqrt(fabs(diag[perm[p]] * diag[col]));
        const double rr = sc > 0.0 ? best / sc : 0.0;
        rmin = fmin(rmin, rr);
        rmax = fmax(rmax, rr);
        const int t = perm[p];
        perm[p] = perm[col];
        perm[col] = t;
      }
    }
    __syncthreads();
    const int p = *piv;
    if (p != col)
      for (int j = tid; j < ncol; j += blockDim.x) {
        double t = M[col * ld + j];
        M[col * ld + j] = M[p * ld + j];
        M[p * ld + j] = t;
      }
    __syncthreads();
    const double inv = 1.0 / M[col * ld + col];
    __syncthreads();
    for (int j = tid; j < ncol; j += blockDim.x) M[col * ld + j] *= inv;
    for (int r = tid; r < n; r += blockDim.x) fac[r] = M[r * ld + col];
    __syncthreads();
    for (int e = tid; e < n * ncol; e += blockDim.x) {
      const int r = e / ncol, j = e - (e / ncol) * ncol;
      if (r != col) M[r * ld + j] -= fac[r] * M[col * ld + j];
    }
    __syncthreads();
  }
  if (tid == 0 && cond) *cond = rmin > 0.0 ? (float)(rmax / rmin) : INFINITY;
}

__device__ __forceinline__ void assemble_body(const ClassDev& c, int bx) {
  extern __shared__ double dsm[];
  __shared__ double fac[UPH_MAXLIN];
  __shared__ double ridge[UPH_MAXLIN];
  __shared__ int piv;
  const int isl = bx / c.nb, b = bx % c.nb;
  if (isl >= c.n_isl || !isl_active(c.flags[isl], PH_LIN)) return;
  const int tid = threadIdx.x;
  const int nL = c.isl_nL[isl], nr = c.isl_nr[isl];
  const int nl = nr + c.nbg;   // linear rows: member models, then background
  const int K = gram_K(c, isl);
  const float* G = c.gram + ((size_t)isl * c.nb + b) * c.Kmax * c.Kmax;
  const int ldg = c.Kmax;
  const int16_t* rk = c.row_k + (size_t)isl * c.Kmax;
  float* Hb = c.Hb + ((size_t)isl * c.nb + b) * c.nLmax * c.nLmax;
  float* gb = c.gb + ((size_t)isl * c.nb + b) * c.nLmax;
  const int ncol = 2 * nl + 1;
  const int lda = ncol;
  constexpr int LS = UPH_MAXLIN;           // row stride of the nL x nl blocks
  double* Aug = dsm;                       // nl x (2 nl + 1)
  double* DM = Aug + LS * (2 * LS + 1);    // nL x nl
  double* Cm = DM + (size_t)c.nLmax * LS;  // nL x nl
  double* Wm = Cm + (size_t)c.nLmax * LS;  // nL x nl
  double* vec = Wm + (size_t)c.nLmax * LS; // f64[nl], a[nl], q[nl]
  double* f64v = vec;
  double* av = vec + LS;
  double* qv = av + LS;
  if (nL == 0) {
    return;
  }
  const int m0 = nL;  // first linear row
  const int dr = nL + nl;
  // Residual form (tensor-core Gram): the last Gram row is r = d - M^T fc
  // with fc the fluxes solved at the same parameters, so G holds M W r and
  // D W r instead of M W d and D W d.  Every quantity below is rewritten in
  // terms of the small differences fc - f, which avoids the cancellation of
  // D W d - D W M^T f at high signal to noise:
  //   f = fc + (A + reg I)^-1 (M W r - reg fc),
  //   D W (d - M^T x) = D W r + D W M^T (fc - x),
  //   M W d - A x     = M W r + A (fc - x).
  if (tid == 0)
    work_add(c, WK_ASSEMBLE, 4ull * (unsigned long long)(K * K + nL * nL + nL), 0);
  const bool resid = c.fcur != nullptr;   // mixed form: every Gram in residual form
  const float* fcb = resid ? c.fcur + ((size_t)isl * c.nb + b) * c.NL : nullptr;
  // linear slot l in the stride-NL arrays: members at l, background j at N + j
  auto fcl = [&](int l) -> double { return (double)fcb[l < nr ? l : c.N + (l - nr)]; };
  // ridge: reg on members (island_solver.py:570-590), reg * |diag| on the
  // background rows (forced_phot_sparse.py:474-489)
  for (int l = tid; l < nl; l += NT)
    ridge[l] = l < nr ? (double)c.reg
                      : (double)c.reg * fmax(fabs((double)G[(m0 + l) * ldg + m0 + l]), 1e-30);
  __syncthreads();
  for (int e = tid; e < nl * ncol; e += NT) {
    const int r = e / ncol, j = e - (e / ncol) * ncol;
    double v;
    if (j < nl) {
      v = (double)G[(m0 + r) * ldg + m0 + j];
      if (j == r) v += ridge[r];
    } else if (j < 2 * nl) {
      v = (j - nl == r) ? 1.0 : 0.0;
    } else {
      v = (double)G[(m0 + r) * ldg + dr];
      if (resid) v -= ridge[r] * fcl(r);
    }
    Aug[r * lda + j] = v;
  }
  for (int e = tid; e < nL * nl; e += NT) {
    const int i = e / nl, l = e - (e / nl) * nl;
    DM[i * LS + l] = (double)G[i * ldg + m0 + l];
  }
  __syncthreads();
  gauss_jordan(Aug, nl, ncol, lda, fac, &piv);
  // f64 fluxes and their float32 copy (the model uses f32 fluxes)
  for (int l = tid; l < nl; l += NT) {
    f64v[l] = Aug[l * lda + 2 * nl] + (resid ? fcl(l) : 0.0);
    av[l] = (double)(float)f64v[l];
  }
  __syncthreads();
  // q = b - A a  (A without ridge)
  for (int l = tid; l < nl; l += NT) {
    double t = (double)G[(m0 + l) * ldg + dr];
    if (resid)
      for (int m = 0; m < nl; ++m)
        t += (double)G[(m0 + l) * ldg + m0 + m] * (fcl(m) - av[m]);
    else
      for (int m = 0; m < nl; ++m) t -= (double)G[(m0 + l) * ldg + m0 + m] * av[m];
    qv[l] = t;
  }
  // c_i = Ainv (e_k s_i - f_k u_i), rounded to f32
  for (int i = tid; i < nL; i += NT) {
    const int k = rk[i];
    double si = (double)G[i * ldg + dr];
    if (resid)
      for (int m = 0; m < nl; ++m) si += DM[i * LS + m] * (fcl(m) - f64v[m]);
    else
      for (int m = 0; m < nl; ++m) si -= DM[i * LS + m] * f64v[m];
    const double fk = f64v[k];
    for (int l = 0; l < nl; ++l) {
      double t = Aug[l * lda + nl + k] * si;
      double u = 0.0;
      for (int m = 0; m < nl; ++m) u += Aug[l * lda + nl + m] * DM[i * LS + m];
      t -= fk * u;
      Cm[i * LS + l] = (double)(float)t;
    }
  }
  __syncthreads();
  if (c.cjac) {
    // the flux sensitivities of this band, for the marginalised flux error
    float* cj = c.cjac + ((size_t)isl * c.nb + b) * c.nLmax * UPH_MAXLIN;
    for (int e = tid; e < nL * nl; e += NT) {
      const int j = e / nl, l = e - (e / nl) * nl;
      cj[(size_t)j * UPH_MAXLIN + l] = (float)Cm[j * LS + l];
    }
  }
  // W_j = A c_j + a_j DM_j
  for (int e = tid; e < nL * nl; e += NT) {
    const int j = e / nl, l = e - (e / nl) * nl;
    double t = av[rk[j]] * DM[j * LS + l];
    for (int m = 0; m < nl; ++m) t += (double)G[(m0 + l) * ldg + m0 + m] * Cm[j * LS + m];
    Wm[j * LS + l] = t;
  }
  __syncthreads();
  // H_ij = a_i (a_j DD_ij + DM_i . c_j) + c_i . W_j
  const int npair = nL * (nL + 1) / 2;
  for (int e = tid; e < npair; e += NT) {
    int i = 0, rem = e;
    while (rem >= nL - i) {
      rem -= nL - i;
      ++i;
    }
    const int j = i + rem;
    const double ai = av[rk[i]], aj = av[rk[j]];
    double t1 = aj * (double)G[i * ldg + j];
    double t2 = 0.0;
    for (int l = 0; l < nl; ++l) {
      t1 += DM[i * LS + l] * Cm[j * LS + l];
      t2 += Cm[i * LS + l] * Wm[j * LS + l];
    }
    const float h = (float)(ai * t1 + t2);
    Hb[i * c.nLmax + j] = h;
    Hb[j * c.nLmax + i] = h;
  }
  // g_i = -(a_i (Dd_i - DM_i . a) + c_i . q)
  for (int i = tid; i < nL; i += NT) {
    double t = (double)G[i * ldg + dr];
    if (resid)
      for (int m = 0; m < nl; ++m) t += DM[i * LS + m] * (fcl(m) - av[m]);
    else
      for (int m = 0; m < nl; ++m) t -= DM[i * LS + m] * av[m];
    double u = 0.0;
    for (int l = 0; l < nl; ++l) u += Cm[i * LS + l] * qv[l];
    gb[i] = (float)(-(av[rk[i]] * t + u));
  }
}

__global__ void __launch_bounds__(NT) k_assemble(ClassDev c) { assemble_body(c, blockIdx.x); }

template <bool BG>
__device__ __forceinline__ void gram_trial_body(const ClassDev& c, const float* __restrict__ P,
                                                int phase, int final_mode,
                                                float* __restrict__ fout,
                                                float* __restrict__ cout, int bx) {
  extern __shared__ float sm[];
  __shared__ int4 box[UPH_MAXN];
  __shared__ int16_t rk[UPH_MAXLIN + 1], rs[UPH_MAXLIN + 1];
  __shared__ double Aug[UPH_MAXLIN * (2 * UPH_MAXLIN + 1)];
  __shared__ double fac[UPH_MAXLIN];
  __shared__ double dg[UPH_MAXLIN];
  __shared__ float gmm[(UPH_MAXLIN + 1) * (UPH_MAXLIN + 1)];
  __shared__ float fl32[UPH_MAXLIN];
  __shared__ int permsh[UPH_MAXLIN];
  __shared__ double red[NT];
  __shared__ int redi[NT];
  __shared__ int piv;
  const int isl = bx / c.nb, b = bx % c.nb;
  if (isl >= c.n_isl || !isl_active(c.flags[isl], phase)) return;
  const int tid = threadIdx.x;
  const int nr = c.isl_nr[isl];
  const int nl = nr + c.nbg;   // linear rows: member models, then background
  const int K = nl + 1;
  load_boxes(c, isl, P, box);
  for (int r = tid; r < K; r += NT) {
    rk[r] = (int16_t)(r < nr ? r : 0);
    rs[r] = (int16_t)(r < nr ? 0 : (r < nl ? -2 - (r - nr) : -1));
  }
  __syncthreads();
  if (tid == 0 && c.work) {
    unsigned long long px = 0;
    for (int k = 0; k < nr; ++k)
      px += (unsigned long long)max(box[k].z, 0) * (unsigned long long)max(box[k].w, 0);
    work_add(c, WK_TRIAL, 4ull * (px + 2ull * c.B * c.B) + 8ull, 0);
  }
  RowSrc rows{rk, rs, K};
  gram_window<BG>(c, isl, b, rows, box, gmm, K, 0, sm);
  __syncthreads();
  const int ncol = 2 * nl + 1;
  // ridge: reg on members (island_solver.py:570-590), reg * |diag| on the
  // background rows (forced_phot_sparse.py:474-489); dg holds the diagonal
  // Aug receives, read from the finished Gram (not from Aug, which other
  // threads are still filling)
  for (int r = tid; r < nl; r += NT) {
    const double a = (double)gmm[r * K + r];
    dg[r] = a + (r < nr ? (double)c.reg : (double)c.reg * fmax(fabs(a), 1e-30));
  }
  __syncthreads();
  for (int e = tid; e < nl * ncol; e += NT) {
    const int r = e / ncol, j = e - (e / ncol) * ncol;
    double v;
    if (j < nl) {
      v = (j == r) ? dg[r] : (double)gmm[r * K + j];
    } else if (j < 2 * nl) {
      v = (j - nl == r) ? 1.0 : 0.0;
    } else {
      v = (double)gmm[r * K + nl];
    }
    Aug[r * ncol + j] = v;
  }
  __syncthreads();
  gauss_jordan(Aug, nl, ncol, ncol, fac, &piv, dg,
               cout ? cout + (size_t)isl * c.nb + b : nullptr, permsh);
  for (int l = tid; l < nl; l += NT) fl32[l] = (float)Aug[l * ncol + 2 * nl];
  if (fout) {
    // stride-NL layout: members at k, background coefficient j at N + j
    float* fo = fout + ((size_t)isl * c.nb + b) * c.NL;
    for (int k = tid; k < c.NL; k += NT) {
      const int l = k < c.N ? (k < nr ? k : -1) : nr + (k - c.N);
      fo[k] = l >= 0 ? (float)Aug[l * ncol + 2 * nl] : 0.f;
    }
  }
  __syncthreads();
  // residual pass
  const int B = c.B, Sz = c.Sz;
  const size_t plane = (size_t)c.Hp * c.Wp;
  const float* dbase = c.dstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
  const float* wbase = c.wstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
  double acc = 0.0;
  int good = 0;
  for (int pix = tid; pix < B * B; pix += NT) {
    const int wy = pix / B, wx = pix - (pix / B) * B;
    const float w = wbase[(size_t)wy * c.Wp + wx];
    const float d = dbase[(size_t)wy * c.Wp + wx];
    float model = 0.f;
    for (int k = 0; k < nr; ++k) {
      const int4 bx = box[k];
      const int ly = wy - bx.y, lx = wx - bx.x;
      if (ly >= 0 && ly < bx.w && lx >= 0 && lx < bx.z)
        model = fmaf(fl32[k], c.stamps[stamp_slot(c, isl, b, k, 0) + (size_t)ly * Sz + lx], model);
    }
    if (BG)
      for (int j = 0; j < c.nbg; ++j) model = fmaf(fl32[nr + j], bg_basis(j, wy, wx, B), model);
    const float r = sqrtf(w) * (d - model);
    acc += (double)r * (double)r;
    good += (w > 0.f);
  }
  red[tid] = acc;
  redi[tid] = good;
  __syncthreads();
  for (int st = NT / 2; st > 0; st >>= 1) {
    if (tid < st) {
      red[tid] += red[tid + st];
      redi[tid] += redi[tid + st];
    }
    __syncthreads();
  }
  if (tid == 0) c.chi2b[(size_t)isl * c.nb + b] = red[0];
  if (final_mode) {
    float* fo = c.flux + ((size_t)isl * c.nb + b) * c.N;
    float* eo = c.ferr + ((size_t)isl * c.nb + b) * c.N;
    for (int k = tid; k < c.N; k += NT) {
      if (k < nr) {
        fo[k] = fl32[k];
        eo[k] = (float)sqrt(fmax(Aug[k * ncol + nl + k], 1e-30));
      } else {
        fo[k] = 0.f;
        eo[k] = 1.0f;  // padded slot: unit diagonal
      }
    }
    if (c.nbg)
      for (int j = tid; j < c.nbg; j += NT) {
        const int l = nr + j;
        c.bgout[((size_t)isl * c.nb + b) * UPH_MAXBG + j] = fl32[l];
        c.bgerr[((size_t)isl * c.nb + b) * UPH_MAXBG + j] =
            (float)sqrt(fmax(Aug[l * ncol + nl + l], 1e-30));
      }
    if (tid == 0) c.ngood[(size_t)isl * c.nb + b] = redi[0];
  }
}

template <bool BG>
__global__ void __launch_bounds__(NT)
k_gram_trial(ClassDev c, const float* __restrict__ P, int phase,
             int final_mode, float* __restrict__ fout, float* __restrict__ cout) {
  gram_trial_body<BG>(c, P, phase, final_mode, fout, cout, blockIdx.x);
}

// LU with partial pivoting of the n x (n+1) augmented system in M (pitch
// n+1); the solution overwrites column n.
__device__ void lu_solve(double* M, int n, int* piv, double* x) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nw = blockDim.x >> 5;
  const int ld = n + 1;
  for (int col = 0; col < n; ++col) {
    // pivot: the first row (in row order) of largest |M[r][col]|, r >= col
    if (warp == 0) {
      double best = -1.0;
      int p = col;
      for (int r = col + lane; r < n; r += 32) {
        const double v = fabs(M[r * ld + col]);
        if (v > best) {
          best = v;
          p = r;
        }
      }
      for (int off = 16; off > 0; off >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, off);
        const int op = __shfl_down_sync(0xffffffffu, p, off);
        if (ob > best || (ob == best && op < p)) {
          best = ob;
          p = op;
        }
      }
      if (lane == 0) *piv = p;
    }
    __syncthreads();
    const int p = *piv;
    if (p != col)
      for (int j = col + tid; j < ld; j += blockDim.x) {
        double t = M[col * ld + j];
        M[col * ld + j] = M[p * ld + j];
        M[p * ld + j] = t;
      }
    __syncthreads();
    // eliminate below the pivot: one row per warp, columns across lanes
    const double pv = M[col * ld + col];
    for (int r = col + 1 + warp; r < n; r += nw) {
      const double f = M[r * ld + col] / pv;
      for (int j = col + 1 + lane; j < ld; j += 32) M[r * ld + j] -= f * M[col * ld + j];
    }
    __syncthreads();
  }
  // back substitution, column oriented: x_r is final once the rows below
  // have been folded into the right-hand side
  for (int r = n - 1; r >= 0; --r) {
    const double xr = M[r * ld + n] / M[r * ld + r];
    if (tid == 0) x[r] = xr;
    for (int i = tid; i < r; i += blockDim.x) M[i * ld + n] -= M[i * ld + r] * xr;
    __syncthreads();
  }
  for (int i = tid; i < n; i += blockDim.x) M[i * ld + n] = x[i];
  __syncthreads();
}

// Trust-region radius update (island_solver.py:154-163): Nocedal & Wright
// Alg. 4.1 gain-ratio thresholds, shrink and expand factors; a step counts
// as reaching the boundary at 99% of the radius.
constexpr double TR_ETA_LO = 0.25, TR_ETA_HI = 0.75;
constexpr double TR_SHRINK = 0.25, TR_EXPAND = 2.0, TR_AT_BOUNDARY = 0.99;

// Sum of one double per thread over the block, in a fixed order (warp
// butterflies, then the warps' partials in warp order); every thread gets
// the total.  red holds NT / 32 doubles.
__device__ double block_sum_d(double v, double* red) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < NT / 32; ++w) t += red[w];
  return t;
}

// Masked, ridged normal matrix entry Hm[i][j] of the live rows (float, the
// same arithmetic as the matrix handed to the solve): kept rows take H,
// frozen rows a unit diagonal; the diagonal adds the prior 1/sigma^2 and
// 1e-8.
__device__ __forceinline__ float hm_entry(const ClassDev& c, const float* H, int ldH,
                                          const uint8_t* kp, const int16_t* rp,
                                          const float* pinv, int i, int j) {
  float h;
  if (kp[i] && kp[j]) h = H[i * ldH + j]; else h = (i == j) ? 1.f : 0.f;
  if (i != j) return h;
  if (c.has_priors) {
    const float pi2 = kp[i] ? __fmul_rn(pinv[rp[i]], pinv[rp[i]]) : 0.f;
    h = __fadd_rn(h, pi2);
  }
  return __fadd_rn(h, 1e-8f);
}

// Gradient entry of live row i with the prior pull (float).
__device__ __forceinline__ float gm_entry(const ClassDev& c, const float* g,
                                          const uint8_t* kp, const int16_t* rp,
                                          const float* p, const float* pm,
                                          const float* pinv, int i) {
  float gi = kp[i] ? g[i] : 0.f;
  if (c.has_priors && kp[i]) {
    const int pp = rp[i];
    gi = __fadd_rn(gi, __fmul_rn(__fmul_rn(pinv[pp], pinv[pp]), __fsub_rn(p[pp], pm[pp])));
  }
  return gi;
}

// Trust-region scaled dogleg (island_solver.py:1021-1078) for one island,
// after the LU solve left x = Hm^-1 g in column nL of M.  With the Marquardt
// scaling D = sqrt(diag Hm): the Gauss-Newton step s_gn = -D x, the Cauchy
// point s_c = -alpha D^-1 g along the scaled gradient, and the dogleg to the
// radius Dr (carried in lam; 0 seeds it with |s_gn|).  Writes p_try =
// box-clip(p + D^-1 s) and, for k_accept, the predicted chi2 gain of the
// realised step, Dr, the radius cap |D (upper - lower)| and whether the
// step reached the boundary.  Parameters outside the live set have unit
// diagonal and zero gradient: their scaled step is 0 and D = 1.
__device__ void step_dogleg(const ClassDev& c, int isl, int nL, const double* M,
                            const uint8_t* kp, const float* H, const float* g,
                            double* dsc, double* gh, double* sgn, double* red,
                            int16_t* qlive) {
  const int tid = threadIdx.x;
  const int nP = c.nP;
  const int ldH = c.nLmax;
  const int ld = nL + 1;
  const int16_t* rp = c.row_p + (size_t)isl * c.Kmax;
  const float* p = c.p + (size_t)isl * nP;
  const float* pm = c.prior_mean + (size_t)isl * nP;
  const float* pinv = c.prior_inv + (size_t)isl * nP;
  const float* lo = c.lower + (size_t)isl * nP;
  const float* hi = c.upper + (size_t)isl * nP;
  float* out = c.p_try + (size_t)isl * nP;
  for (int q = tid; q < nP; q += NT) qlive[q] = -1;
  __syncthreads();
  double a = 0.0, b = 0.0;
  for (int i = tid; i < nL; i += NT) {
    qlive[rp[i]] = (int16_t)i;
    const double d = sqrt(fmax((double)hm_entry(c, H, ldH, kp, rp, pinv, i, i), 1e-12));
    const double gi = (double)gm_entry(c, g, kp, rp, p, pm, pinv, i);
    dsc[i] = d;
    gh[i] = gi / d;
    sgn[i] = d * -M[i * ld + nL];
    a += sgn[i] * sgn[i];
    b += gh[i] * gh[i];
  }
  const double n_gn = sqrt(block_sum_d(a, red));
  const double gg = block_sum_d(b, red);
  double Dr = (double)c.lam[isl];
  if (Dr <= 0.0) Dr = fmax(n_gn, 1e-6);
  // gh . (D^-1 Hm D^-1) gh
  a = 0.0;
  for (int i = tid; i < nL; i += NT) {
    double t = 0.0;
    for (int j = 0; j < nL; ++j)
      t += (double)hm_entry(c, H, ldH, kp, rp, pinv, i, j) * (gh[j] / dsc[j]);
    a += gh[i] * (t / dsc[i]);
  }
  const double ghHgh = block_sum_d(a, red);
  const double alpha = ghHgh > 0.0 ? gg / fmax(ghHgh, 1e-30) : 1.0;
  double ss = 0.0, sd = 0.0, dd = 0.0;
  for (int i = tid; i < nL; i += NT) {
    const double sc = -alpha * gh[i];
    const double df = sgn[i] - sc;
    ss += sc * sc;
    sd += sc * df;
    dd += df * df;
  }
  ss = block_sum_d(ss, red);
  sd = block_sum_d(sd, red);
  dd = block_sum_d(dd, red);
  const double n_c = sqrt(ss);
  const double bb = 2.0 * sd;
  const double cc = ss - Dr * Dr;
  const double disc = fmax(bb * bb - 4.0 * dd * cc, 0.0);
  const double t_bl = fmin(fmax((-bb + sqrt(disc)) / fmax(2.0 * dd, 1e-30), 0.0), 1.0);
  const int leg = (n_gn <= Dr) ? 0 : (n_c >= Dr ? 1 : 2);
  const double cscale = (n_c > 0.0) ? Dr / fmax(n_c, 1e-30) : 1.0;
  for (int q = tid; q < nP; q += NT) out[q] = p[q];
  __syncthreads();
  a = 0.0;
  for (int i = tid; i < nL; i += NT) {
    const double sc = -alpha * gh[i];
    const double si = leg == 0 ? sgn[i] : (leg == 1 ? cscale * sc : sc + t_bl * (sgn[i] - sc));
    a += si * si;
    const float d = kp[i] ? (float)(si / dsc[i]) : 0.f;
    out[rp[i]] = __fadd_rn(p[rp[i]], d);
  }
  const double s_norm = sqrt(block_sum_d(a, red));   // (synchronises)
  for (int q = tid; q < nP; q += NT) out[q] = fminf(fmaxf(out[q], lo[q]), hi[q]);
  __syncthreads();
  // predicted gain of the realised step d = p_try - p (float differences):
  // -(g.d + d.Hm.d / 2); parameters outside the live set have unit Hm
  for (int i = tid; i < nL; i += NT) sgn[i] = (double)__fsub_rn(out[rp[i]], p[rp[i]]);
  __syncthreads();
  a = 0.0;
  b = 0.0;
  for (int i = tid; i < nL; i += NT) {
    double t = 0.0;
    for (int j = 0; j < nL; ++j) t += (double)hm_entry(c, H, ldH, kp, rp, pinv, i, j) * sgn[j];
    a += (double)gm_entry(c, g, kp, rp, p, pm, pinv, i) * sgn[i] + 0.5 * sgn[i] * t;
  }
  for (int q = tid; q < nP; q += NT) {
    const int i = qlive[q];
    const double span = (double)__fsub_rn(hi[q], lo[q]);
    const double dq = i >= 0 ? dsc[i] * span : span;
    b += dq * dq;
    if (i < 0) {
      const double d = (double)__fsub_rn(out[q], p[q]);
      a += 0.5 * d * d;
    }
  }
  const double pred = -block_sum_d(a, red);
  const double dmax = sqrt(block_sum_d(b, red));
  if (tid == 0) {
    double* t = c.trs + (size_t)isl * 4;
    t[0] = pred;
    t[1] = Dr;
    t[2] = dmax;
    t[3] = (s_norm >= TR_AT_BOUNDARY * Dr) ? 1.0 : 0.0;
  }
}

// probe_mode: 0 normal step, 1 diverged probe j (lam_final * 10^(j-4)),
// 2 plateau probe (lam = probe_lam).  With c.tr a normal step is the
// trust-region dogleg (island_solver.py:1004-1078); the probes stay damped
// steps at lam, as the reference's probes are.
__device__ __forceinline__ void step_body(const ClassDev& c, int phase, int probe_mode,
                                          int probe_j, float probe_lam, int bx) {
  extern __shared__ double lsm[];
  __shared__ int piv;
  __shared__ double fac[UPH_MAXLIVE];
  __shared__ float delta[UPH_MAXLIVE];
  __shared__ uint8_t kp[UPH_MAXLIVE];
  __shared__ double tr_a[UPH_MAXLIVE], tr_b[UPH_MAXLIVE], tr_c[UPH_MAXLIVE];
  __shared__ double red[NT / 32];
  __shared__ int16_t qlive[6 * UPH_MAXN];
  const int isl = bx;
  if (isl >= c.n_isl) return;
  const uint8_t fl = c.flags[isl];
  if (!isl_active(fl, phase)) return;
  const int tid = threadIdx.x;
  const int nL = c.isl_nL[isl];
  const int nP = c.nP;
  const int ldH = c.nLmax;
  float* H = c.H + (size_t)isl * ldH * ldH;
  float* g = c.g + (size_t)isl * ldH;
  const int16_t* rp = c.row_p + (size_t)isl * c.Kmax;
  if (tid == 0 && c.work) {
    const unsigned long long hl = (unsigned long long)(nL * nL + nL);
    const bool sum = probe_mode == 0 && (fl & FL_NEEDLIN);
    work_add(c, WK_STEP, 4ull * ((sum ? c.nb + 1 : 1) * hl + 2ull * nP),
             (unsigned long long)(2.0 * nL * nL * nL / 3.0));
  }
  if (probe_mode == 0 && (fl & FL_NEEDLIN)) {
    for (int e = tid; e < nL * nL; e += NT) {
      const int i = e / nL, j = e - (e / nL) * nL;
      float t = 0.f;
      for (int b = 0; b < c.nb; ++b)
        t += c.Hb[((size_t)isl * c.nb + b) * ldH * ldH + i * ldH + j];
      H[i * ldH + j] = t;
    }
    for (int i = tid; i < nL; i += NT) {
      float t = 0.f;
      for (int b = 0; b < c.nb; ++b) t += c.gb[((size_t)isl * c.nb + b) * ldH + i];
      g[i] = t;
    }
    __syncthreads();
    if (tid == 0) c.flags[isl] = fl & ~FL_NEEDLIN;
  }
  float lam;
  int nst_eff = c.nst[isl];
  if (probe_mode == 1) {
    const float sc = (float)pow(10.0, (double)(probe_j - 4));
    lam = c.lam[isl] * sc;
    nst_eff = c.nst[isl] - 4 + probe_j;
  } else if (probe_mode == 2) {
    lam = probe_lam;
  } else {
    lam = c.lam[isl];
  }
  const float* p = c.p + (size_t)isl * nP;
  const float* pm = c.prior_mean + (size_t)isl * nP;
  const float* pinv = c.prior_inv + (size_t)isl * nP;
  for (int i = tid; i < nL; i += NT) {
    const int pp = rp[i];
    bool k = true;
    if (c.un_freeze > 0 && (pp % 6) == 5 && !(nst_eff < c.un_freeze)) k = false;
    kp[i] = k;
  }
  __syncthreads();
  const bool trs = c.tr && probe_mode == 0;
  const bool use_smem = (nL <= UPH_LU_SMEM_N);
  double* M = use_smem ? lsm : (c.lu + (size_t)isl * c.nLmax * (c.nLmax + 1));
  const int ld = nL + 1;
  for (int e = tid; e < nL * ld; e += NT) {
    const int i = e / ld, j = e - (e / ld) * ld;
    double v;
    if (j < nL) {
      float h;
      if (kp[i] && kp[j]) h = H[i * ldH + j]; else h = (i == j) ? 1.f : 0.f;
      if (i == j) {
        float hd = trs ? h : __fadd_rn(h, __fmul_rn(lam, h));
        if (c.has_priors) {
          const int pp = rp[i];
          const float pi2 = kp[i] ? __fmul_rn(pinv[pp], pinv[pp]) : 0.f;
          hd = __fadd_rn(hd, pi2);
        }
        hd = __fadd_rn(hd, 1e-8f);
        v = (double)hd;
      } else {
        v = (double)h;
      }
    } else {
      float gi = kp[i] ? g[i] : 0.f;
      if (c.has_priors && kp[i]) {
        const int pp = rp[i];
        gi = __fadd_rn(gi, __fmul_rn(__fmul_rn(pinv[pp], pinv[pp]),
                                     __fsub_rn(p[pp], pm[pp])));
      }
      v = (double)gi;
    }
    M[i * ld + j] = v;
  }
  __syncthreads();
  if (nL > 0) lu_solve(M, nL, &piv, fac);
  if (trs) {
    step_dogleg(c, isl, nL, M, kp, H, g, tr_a, tr_b, tr_c, red, qlive);
    return;
  }
  for (int i = tid; i < nL; i += NT) {
    const int pp = rp[i];
    float d = -(float)M[i * ld + nL];
    if (!kp[i]) d = 0.f;
    const int j = pp % 6;
    const float cl = (j < 2) ? c.pos_step_max : (j < 5 ? 0.15f : 0.5f);
    d = fminf(fmaxf(d, -cl), cl);
    delta[i] = d;
  }
  __syncthreads();
  float* out = (probe_mode == 1)
                   ? c.probe_p + ((size_t)isl * 4 + probe_j) * nP
                   : c.p_try + (size_t)isl * nP;
  const float* lo = c.lower + (size_t)isl * nP;
  const float* hi = c.upper + (size_t)isl * nP;
  for (int q = tid; q < nP; q += NT) out[q] = p[q];
  __syncthreads();
  for (int i = tid; i < nL; i += NT) out[rp[i]] = __fadd_rn(p[rp[i]], delta[i]);
  __syncthreads();
  for (int q = tid; q < nP; q += NT) out[q] = fminf(fmaxf(out[q], lo[q]), hi[q]);
}

__global__ void __launch_bounds__(NT)
k_step(ClassDev c, int phase, int probe_mode, int probe_j, float probe_lam) {
  step_body(c, phase, probe_mode, probe_j, probe_lam, blockIdx.x);
}

__device__ __forceinline__ void accept_one(const ClassDev& c, int phase, int isl) {
  if (isl >= c.n_isl) return;
  const uint8_t fl = c.flags[isl];
  if (!isl_active(fl, phase)) return;
  const int nP = c.nP;
  const float* pt = c.p_try + (size_t)isl * nP;
  work_add(c, WK_ACCEPT, 8ull * c.nb + 8ull * nP, 0);
  // chi2 of p_try: float32 band accumulation (legacy), and for dlnp the
  // float64 accumulation of the same band sums (island_solver.py:741-758)
  float chi2_try = 0.f;
  double chi2_64 = 0.0;
  for (int b = 0; b < c.nb; ++b) {
    const double cb = c.chi2b[(size_t)isl * c.nb + b];
    chi2_try = __fadd_rn(chi2_try, (float)cb);
    chi2_64 += cb;
  }
  if (c.has_priors) {
    float pen = 0.f;
    double pen64 = 0.0;
    const float* pm = c.prior_mean + (size_t)isl * nP;
    const float* pinv = c.prior_inv + (size_t)isl * nP;
    for (int q = 0; q < nP; ++q) {
      const int k = q / 6;
      if (!(c.keep[(size_t)isl * nP + q] && c.mmask[isl * c.N + k])) continue;
      const float t = __fmul_rn(pinv[q], __fsub_rn(pt[q], pm[q]));
      const float t2 = __fmul_rn(t, t);
      pen = __fadd_rn(pen, t2);
      pen64 += (double)t2;
    }
    chi2_try = __fadd_rn(chi2_try, pen);
    chi2_64 += pen64;
  }
  if (phase == PH_ALL) {
    c.chi2[isl] = chi2_try;
    if (c.dlnp) c.chi2d[isl] = chi2_64;
    return;
  }
  if (phase == PH_PROBE) {
    const float d = __fsub_rn(chi2_try, c.chi2[isl]);
    c.probe_best[isl] = fminf(c.probe_best[isl], d);
    return;
  }
  float* p = c.p + (size_t)isl * nP;
  const float chi2 = c.chi2[isl];
  const float lam = c.lam[isl];
  const bool accept = c.dlnp ? (chi2_64 < c.chi2d[isl]) : (chi2_try < chi2);
  float lam_new;
  if (c.tr) {
    // radius update from the gain ratio of the realised step
    // (island_solver.py:1079-1092; Nocedal & Wright Alg. 4.1 constants)
    const double* t = c.trs + (size_t)isl * 4;
    const double pred = t[0], Dr = t[1], dmax = t[2];
    const double actual = (double)__fsub_rn(chi2, chi2_try);
    const double rho = actual / (pred > 0.0 ? pred : 1e-30);
    const double dn = (rho < TR_ETA_LO)
                          ? Dr * TR_SHRINK
                          : ((rho > TR_ETA_HI && t[3] != 0.0) ? fmin(Dr * TR_EXPAND, dmax) : Dr);
    lam_new = (float)dn;
  } else {
    lam_new = accept ? fmaxf(__fmul_rn(lam, 0.1f), 1e-9f) : fminf(__fmul_rn(lam, 10.0f), 1e6f);
  }
  const float dchi2 = __fsub_rn(chi2, chi2_try);
  float pos_step = 0.f, shape_step = 0.f;
  if (accept) {
    for (int k = 0; k < c.N; ++k) {
      const float mm = c.mmask[isl * c.N + k] ? 1.f : 0.f;
      const float sx = __fsub_rn(pt[6 * k], p[6 * k]);
      const float sy = __fsub_rn(pt[6 * k + 1], p[6 * k + 1]);
      pos_step = fmaxf(pos_step, mm * hypotf(sx, sy));
      for (int j = 2; j < 6; ++j)
        shape_step = fmaxf(shape_step, mm * fabsf(__fsub_rn(pt[6 * k + j], p[6 * k + j])));
    }
  }
  // dlnp (island_solver.py:1283-1292): absolute sub-quantum ftol, and the
  // step prong only on sub-quantum steps
  const bool sub_q = c.dlnp && (c.chi2d[isl] - chi2_64 < (double)c.quantum);
  const bool small = c.dlnp ? (accept && sub_q)
                            : (accept && (dchi2 < __fmul_rn(c.ftol_rel, fmaxf(chi2, 1.0f))));
  int consec = c.consec[isl];
  consec = small ? consec + 1 : (accept ? 0 : consec);
  const bool step_small = accept && (pos_step < c.step_tol) && (shape_step < 0.01f) &&
                          (!c.dlnp || sub_q);
  int nrej = accept ? 0 : c.nrej[isl] + 1;
  if (c.changed) {
    // "changed" counting (island_solver.py:1180-1192): the reject counts
    // only when its proposal differs from the previous rejected one (exact
    // comparison); identical-proposal runs of 4 set the diverged flag
    int ns = c.n_same[isl];
    float* pr = c.prej + (size_t)isl * nP;
    bool same = ns > 0;
    for (int q = 0; q < nP && same; ++q) same = pt[q] == pr[q];
    ns = accept ? 0 : (same ? ns + 1 : 1);
    if (!accept)
      for (int q = 0; q < nP; ++q) pr[q] = pt[q];
    nrej = accept ? 0 : (same ? c.nrej[isl] : c.nrej[isl] + 1);
    c.n_same[isl] = ns;
    if (ns >= 4) c.div_live[isl] = 1;
  }
  bool stall_now = nrej >= 4;
  if (c.dlnp && !accept) {
    // terminal reject-exits: tested at the lam cap, or a no-move proposal
    bool no_move = true;
    for (int q = 0; q < nP && no_move; ++q) no_move = pt[q] == p[q];
    if (lam >= 1e6f || no_move) stall_now = true;
  }
  const bool conv = (consec >= 2) || step_small || stall_now;
  uint8_t nf = fl;
  if (accept) {
    for (int q = 0; q < nP; ++q) p[q] = pt[q];
    if (c.fcur) {
      const size_t o = (size_t)isl * c.nb * c.NL;
      for (int e = 0; e < c.nb * c.NL; ++e) c.fcur[o + e] = c.ftry[o + e];
      for (int b = 0; b < c.nb; ++b)
        c.acond_cur[(size_t)isl * c.nb + b] = c.acond_try[(size_t)isl * c.nb + b];
    }
    c.chi2[isl] = chi2_try;
    if (c.dlnp) c.chi2d[isl] = chi2_64;
    nf |= FL_NEEDLIN;
  }
  if (conv) nf |= FL_CONV;
  if (stall_now) nf |= FL_STALL; else nf &= ~FL_STALL;
  c.flags[isl] = nf;
  c.lam[isl] = lam_new;
  c.consec[isl] = consec;
  c.nrej[isl] = nrej;
  c.nst[isl] = c.nst[isl] + 1;
}

__global__ void k_accept(ClassDev c, int phase) {
  accept_one(c, phase, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---- queue kernels of the LM loop (one launch per kind for the job) ----

// BG: every chunk of the job solves the planar background jointly (the
// host launches the variant that matches the job)
template <bool BG>
__global__ void __launch_bounds__(NT) kq_gram_lin(QueueList q) {
  queue_run(q, QK_GLIN, 1, [&](const ClassDev& c, int isl, int u) {
    const int ydim = gram_lin_ydim(c);
    gram_lin_body<BG>(c, isl * c.nb + u / ydim, u % ydim);
    return false;
  });
}

__global__ void __launch_bounds__(NT) kq_gram_lin_reduce(QueueList q) {
  queue_run(q, QK_GLINR, 1, [&](const ClassDev& c, int isl, int u) {
    gram_lin_reduce_body(c, isl * c.nb + u);
    return false;
  });
}

__global__ void __launch_bounds__(NT) kq_assemble(QueueList q) {
  queue_run(q, QK_ASSEMBLE, 1, [&](const ClassDev& c, int isl, int u) {
    assemble_body(c, isl * c.nb + u);
    return false;
  });
}

// the LM step of every island still iterating (PH_TRIAL: not converged)
__global__ void __launch_bounds__(NT) kq_step(QueueList q) {
  queue_run(q, QK_STEP, 1, [&](const ClassDev& c, int isl, int u) {
    step_body(c, PH_TRIAL, 0, 0, 0.f, isl);
    return false;
  });
}

// the trial chi2 at p_try (fluxes and conditioning of the trial point kept
// for the mixed form)
template <bool BG>
__global__ void __launch_bounds__(NT) kq_gram_trial(QueueList q) {
  queue_run(q, QK_TRIAL, 1, [&](const ClassDev& c, int isl, int u) {
    gram_trial_body<BG>(c, c.p_try, PH_TRIAL, 0, c.ftry, c.acond_try, isl * c.nb + u);
    return false;
  });
}

// accept / reject of every active island, one thread per island
__global__ void kq_accept(QueueList q) {
  const int n = *q.n_act;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
    const int2 e = q.act[a];
    accept_one(q.cls[e.x], PH_TRIAL, e.y);
  }
}

// Exclusive scan of v over the CTA (blockDim.x = QB_THREADS); *total gets the
// CTA's sum.  wsum: 32 ints of shared scratch.
constexpr int QB_THREADS = 1024;
__device__ int block_excl_scan(int v, int* wsum, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = wsum[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    wsum[lane] = w;
  }
  __syncthreads();
  const int ex = x - v + (warp ? wsum[warp - 1] : 0);
  *total = wsum[31];
  __syncthreads();
  return ex;
}

// Compacts the job's (chunk, island) order to the islands active in `phase`
// (order kept: longest first) and writes, per kernel kind, the exclusive
// prefix of units over the active entries; zeroes the item counters.  One
// CTA of QB_THREADS threads.
__global__ void __launch_bounds__(QB_THREADS)
k_queue_build(const ClassDev* __restrict__ cls, const int2* __restrict__ order, int n_total,
              QueueList q, int phase) {
  __shared__ int wsum[32];
  int run_n = 0;
  int run[QK_KINDS];
#pragma unroll
  for (int k = 0; k < QK_KINDS; ++k) run[k] = 0;
  for (int base = 0; base < n_total; base += QB_THREADS) {
    const int i = base + threadIdx.x;
    int2 e = make_int2(0, 0);
    bool act = false;
    if (i < n_total) {
      e = order[i];
      act = isl_active(cls[e.x].flags[e.y], phase);
    }
    int tot;
    const int pos = block_excl_scan(act ? 1 : 0, wsum, &tot);
    if (act) q.act[run_n + pos] = e;
#pragma unroll
    for (int k = 0; k < QK_KINDS; ++k) {
      const int u = act ? queue_units(cls[e.x], k) : 0;
      int tk;
      const int ex = block_excl_scan(u, wsum, &tk);
      if (act) q.pre[(size_t)k * q.stride + run_n + pos] = run[k] + ex;
      run[k] += tk;
    }
    run_n += tot;
  }
  if (threadIdx.x == 0) {
    *q.n_act = run_n;
    for (int k = 0; k < QK_KINDS; ++k) {
      q.pre[(size_t)k * q.stride + run_n] = run[k];
      q.next[k] = 0;
    }
  }
}

// Islands of the job still iterating (not converged), into *out.
__global__ void k_queue_count(const ClassDev* __restrict__ cls, const int2* __restrict__ order,
                              int n_total, int* out) {
  __shared__ int red[NT];
  int cnt = 0;
  for (int i = threadIdx.x; i < n_total; i += NT) {
    const int2 e = order[i];
    cnt += (cls[e.x].flags[e.y] & FL_CONV) ? 0 : 1;
  }
  red[threadIdx.x] = cnt;
  __syncthreads();
  for (int st = NT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// Islands of the chunk still iterating into n_active[0], stalled islands
// (the post-loop probes' subjects) into n_active[1].
__global__ void k_count_active(ClassDev c) {
  __shared__ int s[NT], z[NT];
  int t = 0, u = 0;
  for (int i = threadIdx.x; i < c.n_isl; i += NT) {
    t += !(c.flags[i] & FL_CONV);
    u += (c.flags[i] & FL_STALL) ? 1 : 0;
  }
  s[threadIdx.x] = t;
  z[threadIdx.x] = u;
  __syncthreads();
  for (int st = NT / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) {
      s[threadIdx.x] += s[threadIdx.x + st];
      z[threadIdx.x] += z[threadIdx.x + st];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    c.n_active[0] = s[0];
    c.n_active[1] = z[0];
  }
}

__global__ void k_diverged_compare(ClassDev c, uint8_t* out) {
  const int isl = blockIdx.x * blockDim.x + threadIdx.x;
  if (isl >= c.n_isl) return;
  if (!(c.flags[isl] & FL_PROBE)) {
    out[isl] = 0;
    return;
  }
  const float* q = c.probe_p + (size_t)isl * 4 * c.nP;
  bool same = true;
  for (int j = 1; j < 4; ++j)
    for (int e = 0; e < c.nP; ++e) same = same && (q[j * c.nP + e] == q[e]);
  out[isl] = same;
}

// Bound-pinned disclosure of the trust-region step (island_solver.py:
// 1717-1728): some kept member parameter sits at its lower or upper bound.
__global__ void k_railed(ClassDev c, uint8_t* out) {
  const int isl = blockIdx.x * blockDim.x + threadIdx.x;
  if (isl >= c.n_isl) return;
  const size_t o = (size_t)isl * c.nP;
  bool r = false;
  for (int q = 0; q < c.nP; ++q) {
    if (!(c.keep[o + q] && c.mmask[(size_t)isl * c.N + q / 6])) continue;
    const float v = c.p[o + q];
    r = r || (v <= c.lower[o + q]) || (v >= c.upper[o + q]);
  }
  out[isl] = r ? 1 : 0;
}

// Relinearisation at the final parameters for the covariance: every
// island's flags are saved, then set so that the linearisation kernels
// (render, Gram, assembly) run on it; k_errors_end puts them back.
__global__ void k_errors_begin(ClassDev c) {
  const int isl = blockIdx.x * blockDim.x + threadIdx.x;
  if (isl >= c.n_isl) return;
  const uint8_t fl = c.flags[isl];
  c.flsave[isl] = fl;
  c.flags[isl] = (uint8_t)(FL_NEEDLIN | (fl & FL_REAL));
}

__global__ void k_errors_end(ClassDev c) {
  const int isl = blockIdx.x * blockDim.x + threadIdx.x;
  if (isl >= c.n_isl) return;
  c.flags[isl] = c.flsave[isl];
}

// Marginal covariance of the nonlinear parameters (island_solver.py:
// 1484-1547) for one island: H = sum over bands of the per-band Gauss-Newton
// blocks (float, band order as the step), the static keep mask (every live
// row; no annealing), plus the prior diagonal, inverted in float64 by
// Gauss-Jordan on [Hm | I].  Rows outside the live set are unit rows of the
// full matrix, so their variance is 1 and their covariances 0.  Output per
// member: var(x, y, logre, ee1, ee2, u), cov(ee1, ee2), then the prior
// fractions pinv^2 / (H_kk + pinv^2) on the data diagonal (0 where that sum
// is 0, NaN for every slot without priors).
__global__ void __launch_bounds__(NT) k_final_errors(ClassDev c) {
  __shared__ double fac[UPH_MAXLIVE];
  __shared__ float hdiag[UPH_MAXLIVE];
  __shared__ int16_t qlive[6 * UPH_MAXN];
  __shared__ int piv;
  const int isl = blockIdx.x;
  if (isl >= c.n_isl) return;
  const int tid = threadIdx.x;
  const int nL = c.isl_nL[isl];
  const int nP = c.nP;
  const int ldH = c.nLmax;
  const int ld = 2 * c.nLmax;
  const int16_t* rp = c.row_p + (size_t)isl * c.Kmax;
  const float* pinv = c.prior_inv + (size_t)isl * nP;
  double* A = c.ews + (size_t)isl * c.nLmax * ld;
  for (int q = tid; q < nP; q += NT) qlive[q] = -1;
  __syncthreads();
  for (int i = tid; i < nL; i += NT) qlive[rp[i]] = (int16_t)i;
  for (int e = tid; e < nL * nL; e += NT) {
    const int i = e / nL, j = e - (e / nL) * nL;
    float h = 0.f;
    for (int b = 0; b < c.nb; ++b)
      h += c.Hb[((size_t)isl * c.nb + b) * ldH * ldH + i * ldH + j];
    if (i == j) {
      hdiag[i] = h;
      if (c.has_priors) h = __fadd_rn(h, __fmul_rn(pinv[rp[i]], pinv[rp[i]]));
    }
    A[i * ld + j] = (double)h;
    A[i * ld + nL + j] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  if (nL > 0) gauss_jordan(A, nL, 2 * nL, ld, fac, &piv);
  float* out = c.perr + (size_t)isl * c.N * 13;
  for (int e = tid; e < c.N * 13; e += NT) {
    const int k = e / 13, col = e - (e / 13) * 13;
    float v;
    if (col < 6) {
      const int i = qlive[6 * k + col];
      v = i >= 0 ? (float)A[i * ld + nL + i] : 1.f;
    } else if (col == 6) {
      const int i3 = qlive[6 * k + 3], i4 = qlive[6 * k + 4];
      v = (i3 >= 0 && i4 >= 0) ? (float)A[i3 * ld + nL + i4] : 0.f;
    } else if (!c.has_priors) {
      v = NAN;
    } else {
      const int i = qlive[6 * k + col - 7];
      const float pd = i >= 0 ? __fmul_rn(pinv[6 * k + col - 7], pinv[6 * k + col - 7]) : 0.f;
      const float den = __fadd_rn(i >= 0 ? hdiag[i] : 0.f, pd);
      v = den > 0.f ? __fdiv_rn(pd, den) : 0.f;
    }
    out[e] = v;
  }
}

// Shape-marginalised flux-variance increment (island_solver.py:1549-1613)
// for one island, after k_final_errors left Sigma = Hm^-1 in the right half
// of its work space: per band b and extended member k,
// dv = sum_ij J_ki Sigma_ij J_kj over the live parameters of extended
// members, J_ki = d f_k / d theta_i from the relinearisation's assembly.
// One warp per member; lanes over i with a fixed-order shuffle reduction.
__global__ void __launch_bounds__(NT) k_flux_marg(ClassDev c) {
  __shared__ uint8_t marg[UPH_MAXLIVE];
  const int isl = blockIdx.x;
  if (isl >= c.n_isl) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nL = c.isl_nL[isl], nr = c.isl_nr[isl];
  const int ld = 2 * c.nLmax;
  const int16_t* rp = c.row_p + (size_t)isl * c.Kmax;
  const double* A = c.ews + (size_t)isl * c.nLmax * ld;
  for (int i = tid; i < nL; i += NT) marg[i] = c.stype[(size_t)isl * c.N + rp[i] / 6] != 0;
  __syncthreads();
  for (int e = warp; e < c.nb * c.N; e += NT / 32) {
    const int b = e / c.N, k = e - (e / c.N) * c.N;
    float* out = c.femarg + ((size_t)isl * c.nb + b) * c.N + k;
    const bool ext = k < nr && c.stype[(size_t)isl * c.N + k] != 0;
    if (!ext) {
      if (lane == 0) *out = 0.f;
      continue;
    }
    const float* J = c.cjac + ((size_t)isl * c.nb + b) * c.nLmax * UPH_MAXLIN;
    double acc = 0.0;
    for (int i = lane; i < nL; i += 32) {
      if (!marg[i]) continue;
      double t = 0.0;
      for (int j = 0; j < nL; ++j)
        if (marg[j]) t += A[i * ld + nL + j] * (double)J[(size_t)j * UPH_MAXLIN + k];
      acc += (double)J[(size_t)i * UPH_MAXLIN + k] * t;
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) *out = (float)fmax(acc, 0.0);
  }
}

// Source-metric moments of one (island, band) at the final parameters
// (island_solver.py:1639-1715), from the final pass's model rows and
// fluxes: per member k over its stamp box, sum m, sum own^2, sum
// (members' model - own) own, sum m [w == 0], sum m w (d - model)^2, with
// own = f_k m and the model including the background plane when it is
// solved.  Double accumulation, fixed-order block reduction.
template <bool BG>
__global__ void __launch_bounds__(NT) k_source_metrics(ClassDev c) {
  __shared__ int4 box[UPH_MAXN];
  __shared__ float fl[UPH_MAXLIN];
  __shared__ double red[5][NT / 32];
  const int isl = blockIdx.x / c.nb, b = blockIdx.x % c.nb;
  if (isl >= c.n_isl) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nr = c.isl_nr[isl];
  const int B = c.B, Sz = c.Sz;
  load_boxes(c, isl, c.p, box);
  for (int k = tid; k < nr; k += NT) fl[k] = c.flux[((size_t)isl * c.nb + b) * c.N + k];
  if (BG)
    for (int j = tid; j < c.nbg; j += NT)
      fl[nr + j] = c.bgout[((size_t)isl * c.nb + b) * UPH_MAXBG + j];
  __syncthreads();
  const size_t plane = (size_t)c.Hp * c.Wp;
  const float* dbase = c.dstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
  const float* wbase = c.wstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
  double* out = c.smom + ((size_t)isl * c.nb + b) * c.N * 5;
  for (int k = 0; k < c.N; ++k) {
    double a[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const int4 bk = k < nr ? box[k] : make_int4(0, 0, 0, 0);
    const int npx = max(bk.z, 0) * max(bk.w, 0);
    for (int e = tid; e < npx; e += NT) {
      const int ly = e / bk.z, lx = e - (e / bk.z) * bk.z;
      const int wy = bk.y + ly, wx = bk.x + lx;
      const float m = c.stamps[stamp_slot(c, isl, b, k, 0) + (size_t)ly * Sz + lx];
      float model = 0.f;
      for (int l = 0; l < nr; ++l) {
        const int4 bx = box[l];
        const int yy = wy - bx.y, xx = wx - bx.x;
        if (yy >= 0 && yy < bx.w && xx >= 0 && xx < bx.z)
          model = fmaf(fl[l], c.stamps[stamp_slot(c, isl, b, l, 0) + (size_t)yy * Sz + xx], model);
      }
      float full = model;
      if (BG)
        for (int j = 0; j < c.nbg; ++j) full = fmaf(fl[nr + j], bg_basis(j, wy, wx, B), full);
      const float w = wbase[(size_t)wy * c.Wp + wx];
      const float d = dbase[(size_t)wy * c.Wp + wx];
      const float own = fl[k] * m;
      const float r = d - full;
      a[0] += (double)m;
      a[1] += (double)own * (double)own;
      a[2] += (double)(model - own) * (double)own;
      a[3] += (w == 0.f) ? (double)m : 0.0;
      a[4] += (double)m * (double)w * (double)r * (double)r;
    }
    for (int q = 0; q < 5; ++q) {
      double v = a[q];
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if (lane == 0) red[q][warp] = v;
    }
    __syncthreads();
    if (tid < 5) {
      double t = 0.0;
      for (int w = 0; w < NT / 32; ++w) t += red[tid][w];
      out[k * 5 + tid] = t;
    }
    __syncthreads();
  }
}

// Band combination of the source metrics (island_solver.py:1691-1715), in
// float32 as the reference: fin = clip(sum m, 0, 1) weights fracflux and
// fracmasked; fracin and rchisq are ratios of band sums; the window flux
// f * sum m per band.  Padded slots: NaN (rchisq, fracin, window flux), 0.
__global__ void k_metrics_combine(ClassDev c) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= c.n_isl * c.N) return;
  const int isl = e / c.N, k = e - (e / c.N) * c.N;
  const bool mm = c.mmask[(size_t)isl * c.N + k] != 0;
  float ffn = 0.f, ffd = 0.f, finn = 0.f, find = 0.f, fmn = 0.f, fmd = 0.f, rcn = 0.f, rcd = 0.f;
  for (int b = 0; b < c.nb; ++b) {
    const double* m = c.smom + (((size_t)isl * c.nb + b) * c.N + k) * 5;
    const float sm = (float)m[0], bot = (float)m[1], top = (float)m[2];
    const float fin = fminf(fmaxf(sm, 0.f), 1.f);
    const float ratio = bot > 0.f ? __fdiv_rn(top, bot) : 0.f;
    const float fm = fminf(fmaxf((float)m[3], 0.f), 1.f);
    ffn = __fadd_rn(ffn, __fmul_rn(fin, ratio));
    ffd = __fadd_rn(ffd, fin);
    finn = __fadd_rn(finn, fabsf(sm));
    find = __fadd_rn(find, 1.f);
    fmn = __fadd_rn(fmn, __fmul_rn(fin, fm));
    fmd = __fadd_rn(fmd, fin);
    rcn = __fadd_rn(rcn, fabsf((float)m[4]));
    rcd = __fadd_rn(rcd, fabsf(sm));
    const float f = c.flux[((size_t)isl * c.nb + b) * c.N + k];
    c.swin[((size_t)isl * c.nb + b) * c.N + k] = mm ? __fmul_rn(f, sm) : NAN;
  }
  float* o = c.smet + ((size_t)isl * c.N + k) * 4;
  o[0] = (mm && rcd > 0.f) ? __fdiv_rn(rcn, rcd) : NAN;
  o[1] = (mm && ffd > 0.f) ? __fdiv_rn(ffn, ffd) : 0.f;
  o[2] = (mm && find > 0.f) ? __fdiv_rn(finn, find) : NAN;
  o[3] = (mm && fmd > 0.f) ? __fdiv_rn(fmn, fmd) : 0.f;
}

// Band-coadded residual of one island at the final parameters
// (island_solver.py:1615-1637): per window pixel, sum over bands in band
// order of w (d - model) and of w (float32), the model being the final
// pass's fluxes times its model rows (and the plane when it is solved).
template <bool BG>
__global__ void __launch_bounds__(NT) k_residual_coadd(ClassDev c) {
  __shared__ int4 box[UPH_MAXN];
  __shared__ float fl[UPH_MAXLIN];
  const int isl = blockIdx.x;
  if (isl >= c.n_isl) return;
  const int tid = threadIdx.x;
  const int nr = c.isl_nr[isl];
  const int B = c.B, Sz = c.Sz;
  const size_t plane = (size_t)c.Hp * c.Wp;
  load_boxes(c, isl, c.p, box);
  float* R = c.resid + (size_t)isl * B * B;
  float* W = c.resid_w + (size_t)isl * B * B;
  for (int pix = tid; pix < B * B; pix += NT) {
    R[pix] = 0.f;
    W[pix] = 0.f;
  }
  for (int b = 0; b < c.nb; ++b) {
    __syncthreads();
    for (int k = tid; k < nr; k += NT) fl[k] = c.flux[((size_t)isl * c.nb + b) * c.N + k];
    if (BG)
      for (int j = tid; j < c.nbg; j += NT)
        fl[nr + j] = c.bgout[((size_t)isl * c.nb + b) * UPH_MAXBG + j];
    __syncthreads();
    const float* dbase = c.dstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
    const float* wbase = c.wstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
    for (int pix = tid; pix < B * B; pix += NT) {
      const int wy = pix / B, wx = pix - (pix / B) * B;
      float model = 0.f;
      for (int k = 0; k < nr; ++k) {
        const int4 bx = box[k];
        const int ly = wy - bx.y, lx = wx - bx.x;
        if (ly >= 0 && ly < bx.w && lx >= 0 && lx < bx.z)
          model = fmaf(fl[k], c.stamps[stamp_slot(c, isl, b, k, 0) + (size_t)ly * Sz + lx], model);
      }
      if (BG)
        for (int j = 0; j < c.nbg; ++j) model = fmaf(fl[nr + j], bg_basis(j, wy, wx, B), model);
      const float w = wbase[(size_t)wy * c.Wp + wx];
      const float d = dbase[(size_t)wy * c.Wp + wx];
      R[pix] = __fadd_rn(R[pix], __fmul_rn(w, __fsub_rn(d, model)));
      W[pix] = __fadd_rn(W[pix], w);
    }
  }
}

// Re profile (island_solver.py:1779-1792), one scan point: p_try = p with
// member n's log-radius moved by dk (float add), for the islands where slot
// n holds an extended member; the others are left out of the probe phase
// and their profile entry is 0 (their model does not depend on it).
__global__ void k_reprof_set(ClassDev c, int n, int j, float dk) {
  const int isl = blockIdx.x;
  if (isl >= c.n_isl) return;
  const int nP = c.nP;
  const bool ext = n < c.isl_nr[isl] && c.stype[(size_t)isl * c.N + n] != 0;
  const float* p = c.p + (size_t)isl * nP;
  float* pt = c.p_try + (size_t)isl * nP;
  for (int q = threadIdx.x; q < nP; q += blockDim.x)
    pt[q] = (q == 6 * n + 2 && ext) ? __fadd_rn(p[q], dk) : p[q];
  if (threadIdx.x == 0) {
    c.flags[isl] = ext ? (uint8_t)(FL_PROBE | FL_REAL) : (uint8_t)FL_REAL;
    if (!ext) c.reprof[((size_t)isl * c.N + n) * 12 + j] = 0.f;
  }
}

// chi2 of p_try (float32 band accumulation plus the prior penalty, as the
// step's accept) minus the chi2 at p, for the probed islands.
__global__ void k_reprof_store(ClassDev c, int n, int j) {
  const int isl = blockIdx.x * blockDim.x + threadIdx.x;
  if (isl >= c.n_isl || !(c.flags[isl] & FL_PROBE)) return;
  const int nP = c.nP;
  const float* pt = c.p_try + (size_t)isl * nP;
  float chi2 = 0.f;
  for (int b = 0; b < c.nb; ++b) chi2 = __fadd_rn(chi2, (float)c.chi2b[(size_t)isl * c.nb + b]);
  if (c.has_priors) {
    float pen = 0.f;
    const float* pm = c.prior_mean + (size_t)isl * nP;
    const float* pinv = c.prior_inv + (size_t)isl * nP;
    for (int q = 0; q < nP; ++q) {
      if (!(c.keep[(size_t)isl * nP + q] && c.mmask[isl * c.N + q / 6])) continue;
      const float t = __fmul_rn(pinv[q], __fsub_rn(pt[q], pm[q]));
      pen = __fadd_rn(pen, __fmul_rn(t, t));
    }
    chi2 = __fadd_rn(chi2, pen);
  }
  c.reprof[((size_t)isl * c.N + n) * 12 + j] = __fsub_rn(chi2, c.chi2[isl]);
}

// Scene subtract: each island's windows copied out of the field stacks
// into the chunk's private stacks (island isl at rows isl*B.. of a B-wide
// stack per band), so the add-back below changes no other island's data.
__global__ void k_copy_windows(ClassDev c, const float* __restrict__ fd,
                               const float* __restrict__ fw, int fHp, int fWp,
                               const int* __restrict__ ox_f, const int* __restrict__ oy_f) {
  const int isl = blockIdx.x / c.nb, b = blockIdx.x % c.nb;
  if (isl >= c.n_isl) return;
  const int B = c.B;
  const size_t fplane = (size_t)fHp * fWp, plane = (size_t)c.Hp * c.Wp;
  const float* sd = fd + b * fplane + (size_t)oy_f[isl] * fWp + ox_f[isl];
  const float* sw = fw + b * fplane + (size_t)oy_f[isl] * fWp + ox_f[isl];
  float* dd = const_cast<float*>(c.dstack) + b * plane + (size_t)isl * B * B;
  float* dw = const_cast<float*>(c.wstack) + b * plane + (size_t)isl * B * B;
  for (int pix = threadIdx.x; pix < B * B; pix += blockDim.x) {
    const int y = pix / B, x = pix - (pix / B) * B;
    dd[pix] = sd[(size_t)y * fWp + x];
    dw[pix] = sw[(size_t)y * fWp + x];
  }
}

// Scene subtract add-back (island_solver.py:1795-1818): window data +=
// sum_k member_s1_flux[k, b] m_k, the model rows of the render at the seed
// parameters, members in slot order.
__global__ void __launch_bounds__(NT) k_addback(ClassDev c, const float* __restrict__ seed,
                                                const float* __restrict__ msf) {
  __shared__ int4 box[UPH_MAXN];
  __shared__ float fl[UPH_MAXN];
  const int isl = blockIdx.x / c.nb, b = blockIdx.x % c.nb;
  if (isl >= c.n_isl) return;
  const int tid = threadIdx.x, nr = c.isl_nr[isl], B = c.B, Sz = c.Sz;
  load_boxes(c, isl, seed, box);
  for (int k = tid; k < nr; k += NT) fl[k] = msf[((size_t)isl * c.N + k) * c.nb + b];
  __syncthreads();
  float* dd = const_cast<float*>(c.dstack) + b * (size_t)c.Hp * c.Wp + (size_t)isl * B * B;
  for (int pix = tid; pix < B * B; pix += NT) {
    const int wy = pix / B, wx = pix - (pix / B) * B;
    float model = 0.f;
    for (int k = 0; k < nr; ++k) {
      const int4 bx = box[k];
      const int ly = wy - bx.y, lx = wx - bx.x;
      if (ly >= 0 && ly < bx.w && lx >= 0 && lx < bx.z)
        model = fmaf(fl[k], c.stamps[stamp_slot(c, isl, b, k, 0) + (size_t)ly * Sz + lx], model);
    }
    dd[pix] = __fadd_rn(dd[pix], model);
  }
}

__global__ void k_set_probe(ClassDev c) {
  const int isl = blockIdx.x * blockDim.x + threadIdx.x;
  if (isl >= c.n_isl) return;
  const uint8_t fl = c.flags[isl];
  c.flags[isl] = (fl & FL_STALL) ? (fl | FL_PROBE) : (fl & ~FL_PROBE);
}

}  // namespace

__global__ void k_fill_float(float* p, float v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

void launch_fill_float(float* p, float v, int n, cudaStream_t s) {
  if (n > 0) k_fill_float<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p, v, n);
}

void launch_railed(const ClassDev& c, uint8_t* out, cudaStream_t s) {
  k_railed<<<(unsigned)((c.n_isl + 127) / 128), 128, 0, s>>>(c, out);
}

void launch_errors_begin(const ClassDev& c, cudaStream_t s) {
  k_errors_begin<<<(unsigned)((c.n_isl + 127) / 128), 128, 0, s>>>(c);
}

void launch_errors_end(const ClassDev& c, cudaStream_t s) {
  k_errors_end<<<(unsigned)((c.n_isl + 127) / 128), 128, 0, s>>>(c);
}

void launch_final_errors(const ClassDev& c, cudaStream_t s) {
  k_final_errors<<<(unsigned)c.n_isl, NT, 0, s>>>(c);
}

void launch_flux_marg(const ClassDev& c, cudaStream_t s) {
  k_flux_marg<<<(unsigned)c.n_isl, NT, 0, s>>>(c);
}

void launch_source_metrics(const ClassDev& c, cudaStream_t s) {
  if (c.nbg)
    k_source_metrics<true><<<(unsigned)(c.n_isl * c.nb), NT, 0, s>>>(c);
  else
    k_source_metrics<false><<<(unsigned)(c.n_isl * c.nb), NT, 0, s>>>(c);
  k_metrics_combine<<<(unsigned)((c.n_isl * c.N + 127) / 128), 128, 0, s>>>(c);
}

void launch_residual_coadd(const ClassDev& c, cudaStream_t s) {
  if (c.nbg)
    k_residual_coadd<true><<<(unsigned)c.n_isl, NT, 0, s>>>(c);
  else
    k_residual_coadd<false><<<(unsigned)c.n_isl, NT, 0, s>>>(c);
}

void launch_reprof_set(const ClassDev& c, int n, int j, float dk, cudaStream_t s) {
  k_reprof_set<<<(unsigned)c.n_isl, 64, 0, s>>>(c, n, j, dk);
}

void launch_reprof_store(const ClassDev& c, int n, int j, cudaStream_t s) {
  k_reprof_store<<<(unsigned)((c.n_isl + 127) / 128), 128, 0, s>>>(c, n, j);
}

void launch_copy_windows(const ClassDev& c, const float* fd, const float* fw, int fHp, int fWp,
                         const int* ox_f, const int* oy_f, cudaStream_t s) {
  k_copy_windows<<<(unsigned)(c.n_isl * c.nb), 256, 0, s>>>(c, fd, fw, fHp, fWp, ox_f, oy_f);
}

void launch_addback(const ClassDev& c, const float* seed, const float* msf, cudaStream_t s) {
  k_addback<<<(unsigned)(c.n_isl * c.nb), NT, 0, s>>>(c, seed, msf);
}

void launch_set_probe(const ClassDev& c, cudaStream_t s) {
  k_set_probe<<<(unsigned)((c.n_isl + 127) / 128), 128, 0, s>>>(c);
}

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

void launch_q_gram_lin(const QueueList& q, bool bg, bool reduce, size_t smem, int sms,
                       cudaStream_t s) {
  if (bg)
    kq_gram_lin<true><<<queue_grid(kq_gram_lin<true>, NT, smem, sms, q.cap[QK_GLIN], q.per_cta),
                        NT, smem, s>>>(q);
  else
    kq_gram_lin<false><<<queue_grid(kq_gram_lin<false>, NT, smem, sms, q.cap[QK_GLIN],
                                    q.per_cta), NT, smem, s>>>(q);
  if (reduce)
    kq_gram_lin_reduce<<<queue_grid(kq_gram_lin_reduce, NT, 0, sms, q.cap[QK_GLINR], q.per_cta),
                         NT, 0, s>>>(q);
}
void launch_q_assemble(const QueueList& q, size_t smem, int sms, cudaStream_t s) {
  kq_assemble<<<queue_grid(kq_assemble, NT, smem, sms, q.cap[QK_ASSEMBLE], q.per_cta), NT, smem, s>>>(q);
}
void launch_q_step(const QueueList& q, size_t smem, int sms, cudaStream_t s) {
  kq_step<<<queue_grid(kq_step, NT, smem, sms, q.cap[QK_STEP], q.per_cta), NT, smem, s>>>(q);
}
void launch_q_trial(const QueueList& q, bool bg, size_t smem, int sms, cudaStream_t s) {
  if (bg)
    kq_gram_trial<true><<<queue_grid(kq_gram_trial<true>, NT, smem, sms, q.cap[QK_TRIAL], q.per_cta), NT, smem, s>>>(q);
  else
    kq_gram_trial<false><<<queue_grid(kq_gram_trial<false>, NT, smem, sms, q.cap[QK_TRIAL], q.per_cta), NT, smem, s>>>(q);
}
void launch_q_accept(const QueueList& q, int sms, cudaStream_t s) {
  kq_accept<<<(unsigned)std::max(1, std::min(4 * sms, (q.cap[QK_ACCEPT] + 127) / 128)), 128,
              0, s>>>(q);
}
void launch_q_build(const ClassDev* cls, const int2* order, int n_total, const QueueList& q,
                    int phase, cudaStream_t s) {
  k_queue_build<<<1, QB_THREADS, 0, s>>>(cls, order, n_total, q, phase);
}
void launch_q_count(const ClassDev* cls, const int2* order, int n_total, int* out,
                    cudaStream_t s) {
  k_queue_count<<<1, NT, 0, s>>>(cls, order, n_total, out);
}

size_t gram_lin_smem_bytes(int Kmax) {
  // the largest staged-tile footprint over every K <= Kmax (the tile width
  // shrinks as K grows; the trial pass stages tiles for its residual even
  // when its Gram takes the small path), and the small path's partials
  size_t best = sizeof(float) * (size_t)(NT / 32) * 36;
  for (int K = 1; K <= Kmax; ++K) {
    const size_t b = sizeof(float) * (size_t)tile_floats(K);
    if (b > best) best = b;
  }
  return best;
}

size_t gram_trial_smem_bytes(int N) { return gram_lin_smem_bytes(N + UPH_MAXBG + 1); }

size_t assemble_smem_bytes(int nLmax, int N) {
  (void)N;
  return sizeof(double) * ((size_t)UPH_MAXLIN * (2 * UPH_MAXLIN + 1) +
                           3 * (size_t)nLmax * UPH_MAXLIN + 3 * UPH_MAXLIN);
}

size_t step_smem_bytes(int nLmax) {
  const int n = nLmax < UPH_LU_SMEM_N ? nLmax : UPH_LU_SMEM_N;
  return sizeof(double) * (size_t)n * (n + 1);
}

void launch_gram_lin(const ClassDev& c, cudaStream_t s) {
  dim3 grid((unsigned)(c.n_isl * c.nb), (unsigned)gram_lin_ydim(c));
  const size_t smem = gram_lin_smem_bytes(c.Kmax);
  if (c.Kmax <= 8) {
    if (c.nbg)
      k_gram_lin_small<true><<<grid, NT, smem, s>>>(c);
    else
      k_gram_lin_small<false><<<grid, NT, smem, s>>>(c);
  } else if (c.nbg) {
    k_gram_lin<true><<<grid, NT, smem, s>>>(c);
  } else {
    k_gram_lin<false><<<grid, NT, smem, s>>>(c);
  }
  if (c.gl_split > 1) k_gram_lin_reduce<<<(unsigned)(c.n_isl * c.nb), NT, 0, s>>>(c);
}

void launch_assemble(const ClassDev& c, cudaStream_t s) {
  k_assemble<<<(unsigned)(c.n_isl * c.nb), NT, assemble_smem_bytes(c.nLmax, c.N), s>>>(c);
}

void launch_gram_trial(const ClassDev& c, const float* P, int phase,
                       int final_mode, float* fout, float* cout, cudaStream_t s) {
  const unsigned grid = (unsigned)(c.n_isl * c.nb);
  const size_t smem = gram_trial_smem_bytes(c.N);
  if (c.nbg) {
    k_gram_trial<true><<<grid, NT, smem, s>>>(c, P, phase, final_mode, fout, cout);
  } else {
    k_gram_trial<false><<<grid, NT, smem, s>>>(c, P, phase, final_mode, fout, cout);
  }
}

void launch_step(const ClassDev& c, int phase, int probe_j, float probe_lam,
                 int probe_mode, cudaStream_t s) {
  k_step<<<(unsigned)c.n_isl, NT, step_smem_bytes(c.nLmax), s>>>(
      c, phase, probe_mode, probe_j, probe_lam);
}

void launch_accept(const ClassDev& c, int phase, cudaStream_t s) {
  k_accept<<<(unsigned)((c.n_isl + 127) / 128), 128, 0, s>>>(c, phase);
}

void launch_count_active(const ClassDev& c, cudaStream_t s) {
  k_count_active<<<1, NT, 0, s>>>(c);
}

void launch_diverged_compare(const ClassDev& c, uint8_t* out,
                             cudaStream_t s) {
  k_diverged_compare<<<(unsigned)((c.n_isl + 127) / 128), 128, 0, s>>>(c, out);
}

int uph_solve_setup() {
  cudaError_t e;
  e = cudaFuncSetAttribute(k_gram_lin<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)gram_lin_smem_bytes(UPH_MAXK));
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(k_gram_lin<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)gram_lin_smem_bytes(UPH_MAXK));
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(k_gram_trial<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)gram_trial_smem_bytes(UPH_MAXN));
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(k_gram_trial<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)gram_trial_smem_bytes(UPH_MAXN));
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(k_assemble, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)assemble_smem_bytes(UPH_MAXLIVE, UPH_MAXN));
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(k_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)step_smem_bytes(UPH_MAXLIVE));
  if (e != cudaSuccess) return (int)e;
  // the queue kernels take the same largest dynamic footprints
  for (auto f : {kq_gram_lin<false>, kq_gram_lin<true>}) {
    e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gram_lin_smem_bytes(UPH_MAXK));
    if (e != cudaSuccess) return (int)e;
  }
  for (auto f : {kq_gram_trial<false>, kq_gram_trial<true>}) {
    e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gram_trial_smem_bytes(UPH_MAXN));
    if (e != cudaSuccess) return (int)e;
  }
  e = cudaFuncSetAttribute(kq_assemble, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)assemble_smem_bytes(UPH_MAXLIVE, UPH_MAXN));
  if (e != cudaSuccess) return (int)e;
  e = cudaFuncSetAttribute(kq_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)step_smem_bytes(UPH_MAXLIVE));
  return (int)e;
}

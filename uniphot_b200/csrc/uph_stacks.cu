// Field-stack build on the device: the frozen per-tile planar background of
// pass 1 subtracted from the padded data stack (island_stage.py:1728-1751,
// there numpy on the host).  Over each tile's core rectangle [x0, x1) x
// [y0, y1) (unpadded pixels) and every band,
//
//   stack[b, pad + y, pad + x] -= sum_m basis_m(x, y) * coefs[t, b, m],
//
// with basis_m = X^i Y^j in the term order of make_bg_basis
// (bg_polynomial.py:125-178): X = (x - x_origin) / x_scale and Y likewise in
// float64, each product rounded once to float32, the sum over m a float32
// fused multiply-add chain in term order (the host's BLAS matrix-vector
// product sums the same way on the x86 hosts measured: bit-identical on
// all pixels of the order-1 golden case, all but 0.07% for order 2).  Tiles are applied one launch after another, so
// overlapping cores subtract in tile order as the host loop does.
// Elementwise and HBM-bound: a grid-stride loop over (band, row, column) of
// the tile, consecutive threads on consecutive columns.

#include <algorithm>

#include "uph_internal.cuh"

namespace {

constexpr int ST = 256;

// (i, j) exponents of X and Y per term, orders 0, 1, 2
__constant__ int kTermX[6] = {0, 1, 0, 2, 1, 0};
__constant__ int kTermY[6] = {0, 0, 1, 0, 1, 2};

__device__ inline double ipow(double v, int e) { return e == 0 ? 1.0 : (e == 1 ? v : v * v); }

__global__ void __launch_bounds__(ST) k_tile_bg_subtract(float* __restrict__ stack, int nb, int Hp,
                                                         int Wp, int pad, int x0, int y0, int w,
                                                         int h, const float* __restrict__ coefs,
                                                         int M, double xo, double xs, double yo,
                                                         double ys) {
  const size_t n = (size_t)nb * h * w;
  for (size_t e = (size_t)blockIdx.x * ST + threadIdx.x; e < n; e += (size_t)gridDim.x * ST) {
    const int c = (int)(e % w);
    const int r = (int)((e / w) % h);
    const int b = (int)(e / ((size_t)w * h));
    const double X = ((double)(x0 + c) - xo) / xs;
    const double Y = ((double)(y0 + r) - yo) / ys;
    float bg = 0.f;
    for (int m = 0; m < M; ++m) {
      const float basis = (float)(ipow(X, kTermX[m]) * ipow(Y, kTermY[m]));
      bg = __fmaf_rn(basis, coefs[(size_t)b * M + m], bg);
    }
    float* px = stack + ((size_t)b * Hp + pad + y0 + r) * Wp + pad + x0 + c;
    *px = __fsub_rn(*px, bg);
  }
}

}  // namespace

void launch_tile_bg_subtract(float* stack, int nb, int Hp, int Wp, int pad, int x0, int y0,
                             int w, int h, const float* coefs, int M, const double* norm,
                             int sms, cudaStream_t s) {
  const size_t n = (size_t)nb * h * w;
  if (n == 0) return;
  const unsigned grid = (unsigned)std::min<size_t>((n + ST - 1) / ST, (size_t)sms * 8);
  k_tile_bg_subtract<<<grid, ST, 0, s>>>(stack, nb, Hp, Wp, pad, x0, y0, w, h, coefs, M, norm[0],
                                         norm[1], norm[2], norm[3]);
}

// ---- Field-wide scene subtraction of the star models (island_stage.py:
// 2024-2118): stack[b, pad + iy + r, pad + ix + c] -= flux * stamp[r][c]
// over the part of each source's T x T stamp inside the padded stack,
// product and difference each rounded to float32 (the reference's numpy
// `dmb[...] -= f * st`).  The sources of one launch (a wave) have pairwise
// disjoint stamps, so no two threads touch a pixel; the host orders the
// waves so that a pixel covered by several stamps is reduced in source
// order.  One CTA per source of the wave, threads over its stamp pixels.
namespace {

__global__ void __launch_bounds__(ST) k_scene_sub(float* __restrict__ stack, int Hp, int Wp,
                                                  int pad, int T,
                                                  const int* __restrict__ srcs,
                                                  const float* __restrict__ stamps,
                                                  const int* __restrict__ ixt,
                                                  const int* __restrict__ iyt,
                                                  const float* __restrict__ flux) {
  const int s = srcs[blockIdx.x];
  const float f = flux[s];
  if (f == 0.f) return;
  const int ix = ixt[s] + pad, iy = iyt[s] + pad;
  const float* st = stamps + (size_t)s * T * T;
  for (int e = threadIdx.x; e < T * T; e += ST) {
    const int r = e / T, c = e - (e / T) * T;
    const int y = iy + r, x = ix + c;
    if (y < 0 || y >= Hp || x < 0 || x >= Wp) continue;
    float* px = stack + (size_t)y * Wp + x;
    *px = __fsub_rn(*px, __fmul_rn(f, st[e]));
  }
}

}  // namespace

void launch_scene_sub_wave(float* stack, int Hp, int Wp, int pad, int T, const int* srcs,
                           int count, const float* stamps, const int* ixt, const int* iyt,
                           const float* flux, cudaStream_t s) {
  if (count > 0)
    k_scene_sub<<<(unsigned)count, ST, 0, s>>>(stack, Hp, Wp, pad, T, srcs, stamps, ixt, iyt,
                                               flux);
}

// Island decomposition on the device (islands.py:361-470): sources i and j
// couple when dist(i, j) < r_i + r_j (float64, the reference's exact
// predicate); islands are the connected components of that graph.
//
//   k_isl_cells   cell of each source on a uniform grid of pitch 2 r_max
//                 (coupled sources lie in the same or adjacent cells) and a
//                 count per cell
//   k_isl_scan    exclusive prefix sum of the counts (one CTA)
//   k_isl_fill    sources bucketed by cell (order within a cell is free)
//   k_isl_union   one thread per source scans the 3 x 3 cells around its
//                 own; every coupled pair with j > i is united in a lock-free
//                 union-find whose roots point to the smaller index, so the
//                 root of every component is its minimum member index,
//                 whatever the order of the unions
//   k_isl_roots   the root of every source
//
// The union's compare-and-swap retry loop is bounded; a run that exceeds
// the bound sets an error flag that the host reports.

#include "uph_internal.cuh"

namespace {

constexpr int IT = 256;

__device__ __forceinline__ int find_root(const volatile int* parent, int x) {
  // parents only ever decrease, so the walk ends at a self-parented root;
  // volatile reads see other threads' links
  int p = parent[x];
  while (p != x) {
    x = p;
    p = parent[x];
  }
  return x;
}

__global__ void k_isl_cells(int n, const double* __restrict__ x, const double* __restrict__ y,
                            double x0, double y0, double cell, int ncx, int ncy,
                            int* __restrict__ cid, int* __restrict__ count,
                            int* __restrict__ parent) {
  const int i = blockIdx.x * IT + threadIdx.x;
  if (i >= n) return;
  int cx = (int)floor((x[i] - x0) / cell);
  int cy = (int)floor((y[i] - y0) / cell);
  cx = min(max(cx, 0), ncx - 1);
  cy = min(max(cy, 0), ncy - 1);
  const int c = cy * ncx + cx;
  cid[i] = c;
  atomicAdd(&count[c], 1);
  parent[i] = i;
}

__global__ void k_isl_scan(int ncell, const int* __restrict__ count, int* __restrict__ start,
                           int* __restrict__ cursor) {
  __shared__ int carry;
  __shared__ int buf[1024];
  const int tid = threadIdx.x;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < ncell; base += 1024) {
    const int i = base + tid;
    const int v = i < ncell ? count[i] : 0;
    buf[tid] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      const int t = tid >= off ? buf[tid - off] : 0;
      __syncthreads();
      buf[tid] += t;
      __syncthreads();
    }
    if (i < ncell) {
      const int ex = carry + buf[tid] - v;
      start[i] = ex;
      cursor[i] = ex;
    }
    __syncthreads();
    if (tid == 1023) carry += buf[1023];
    __syncthreads();
  }
  if (tid == 0) start[ncell] = carry;
}

__global__ void k_isl_fill(int n, const int* __restrict__ cid, int* __restrict__ cursor,
                           int* __restrict__ bucket) {
  const int i = blockIdx.x * IT + threadIdx.x;
  if (i >= n) return;
  bucket[atomicAdd(&cursor[cid[i]], 1)] = i;
}

__global__ void k_isl_union(int n, const double* __restrict__ x, const double* __restrict__ y,
                            const double* __restrict__ r, const uint8_t* __restrict__ single,
                            const int* __restrict__ cid, int ncx, int ncy,
                            const int* __restrict__ start, const int* __restrict__ bucket,
                            int* parent, int tries_max, int* __restrict__ err) {
  const int i = blockIdx.x * IT + threadIdx.x;
  if (i >= n) return;
  if (single && single[i]) return;
  const int c = cid[i];
  const int cx = c % ncx, cy = c / ncx;
  const double xi = x[i], yi = y[i], ri = r[i];
  for (int dy = -1; dy <= 1; ++dy) {
    const int yy = cy + dy;
    if (yy < 0 || yy >= ncy) continue;
    for (int dx = -1; dx <= 1; ++dx) {
      const int xx = cx + dx;
      if (xx < 0 || xx >= ncx) continue;
      const int cc = yy * ncx + xx;
      for (int q = start[cc]; q < start[cc + 1]; ++q) {
        const int j = bucket[q];
        if (j <= i) continue;
        if (single && single[j]) continue;
        const double ddx = xi - x[j], ddy = yi - y[j];
        const double rs = ri + r[j];
        if (!(ddx * ddx + ddy * ddy < rs * rs)) continue;
        // unite: hook the larger root under the smaller, at most tries_max
        // attempts (a lost CAS means another thread re-linked a root first)
        int tries = 0;
        while (true) {
          const int a = find_root(parent, i), b = find_root(parent, j);
          if (a == b) break;
          if (tries++ >= tries_max) {
            atomicExch(err, 1);
            break;
          }
          const int hi = a > b ? a : b, lo = a > b ? b : a;
          if (atomicCAS(&parent[hi], hi, lo) == hi) break;
        }
      }
    }
  }
}

__global__ void k_isl_roots(int n, const int* parent, int* __restrict__ root) {
  const int i = blockIdx.x * IT + threadIdx.x;
  if (i < n) root[i] = find_root(parent, i);
}

}  // namespace

void launch_island_roots(const IslandDev& d, cudaStream_t s) {
  const unsigned g = (unsigned)((d.n + IT - 1) / IT);
  k_isl_cells<<<g, IT, 0, s>>>(d.n, d.x, d.y, d.x0, d.y0, d.cell, d.ncx, d.ncy, d.cid, d.count,
                               d.parent);
  k_isl_scan<<<1, 1024, 0, s>>>(d.ncx * d.ncy, d.count, d.start, d.cursor);
  k_isl_fill<<<g, IT, 0, s>>>(d.n, d.cid, d.cursor, d.bucket);
  k_isl_union<<<g, IT, 0, s>>>(d.n, d.x, d.y, d.r, d.single, d.cid, d.ncx, d.ncy, d.start,
                               d.bucket, d.parent, d.tries, d.err);
  k_isl_roots<<<g, IT, 0, s>>>(d.n, d.parent, d.root);
}

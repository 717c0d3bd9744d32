// Weighted Gram of the VarPro rows on the 5th-generation tensor cores.
//
// G = Z W Z^T for Z = [dm/dtheta (nL); m (nr); r (1)] over the island
// window of one band, computed with tcgen05.mma.  The last row is the
// residual r = d - M^T fc at the fluxes fc solved at the same parameters (the
// FP32 Gram of k_gram_lin uses the data row instead): at high signal to noise
// the gradient D W (d - M^T f) is a small difference of large Gram entries,
// which a BF16-split Gram cannot resolve, while D W r is formed directly
// (k_assemble works in the corresponding residual form).  Z is split per
// element into a BF16 pair
// Z = Zh + Zl (Zl = bf16(Z - Zh)), and
//     G ~= Zh Zh^T + Zh Zl^T + Zl Zh^T
// is accumulated in FP32 in tensor memory (the dropped Zl Zl^T term and the
// pair's representation error are ~2^-16 relative per product).
//
// One CTA per (island, band) with K = nL + nr + 1 rows (stored padded to R =
// 128 * ceil(K / 128) rows; the padding rows are zeroed once and never
// rewritten); pixels stream through shared memory in chunks of 64,
// double-buffered: all threads convert chunk c + 1 while the tensor core
// consumes chunk c.  A chunk's window coordinates, weights and residuals are
// decoded once into shared memory; each lane then converts 8 pixels of one
// row (8 independent loads) into one 16-byte store per half of the pair,
// consecutive lanes taking consecutive rows so that a warp fills whole core
// matrices without bank conflicts.  Shared memory is sized by the class's
// largest row count, so classes with at most 128 rows fit three CTAs per SM.
// Operands are K-major (pixels contiguous) in the no-swizzle canonical
// layout: 8-row x 16-byte core matrices, consecutive 8-row groups 128 B apart
// (SBO), the two 8-pixel halves of a 16-pixel MMA step R * 16 B apart (LBO).  One elected thread issues M = 128, N = ceil16
// (K) <= 256, K-step = 16 MMAs; tcgen05.commit arrives on the stage's
// mbarrier.  Waits are bounded: on expiry the kernel raises the chunk's error
// flag, drains, frees its tensor memory and returns.
#include <cuda_bf16.h>

#include <algorithm>

#include "uph_internal.cuh"

namespace {

constexpr int NT = 256;
constexpr int KC = 64;                  // pixels per chunk
constexpr int NG = KC / 8;              // 8-pixel groups per chunk
constexpr unsigned SPIN_LIMIT = 1u << 24;

// Stored rows for at most kmax Gram rows (one or two M = 128 halves), and
// the bytes of one stage (Zh and Zl, bf16).
__host__ __device__ constexpr int rows_cap(int kmax) { return ((kmax + 127) / 128) * 128; }
__host__ __device__ constexpr size_t stage_bytes(int rcap) { return (size_t)2 * rcap * KC * 2; }

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor, K-major, no swizzle (sm100 version 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo,
                                              uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;               // descriptor version (Blackwell)
  return d;                             // base offset 0, layout SWIZZLE_NONE
}

// Instruction descriptor: kind::f16, A = B = BF16, D = F32, K-major both,
// M = 128, N = n.
__device__ __forceinline__ uint32_t umma_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t adesc,
                                         uint64_t bdesc, uint32_t idesc,
                                         uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
      :
      : "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Bounded wait on an mbarrier phase; false on expiry.
__device__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
  for (unsigned i = 0; i < SPIN_LIMIT; ++i)
    if (mbar_try(bar, phase)) return true;
  return false;
}

__device__ __forceinline__ int gram_rows(const ClassDev& c, int isl) {
  return gram_K(c, isl);
}

// One (island, band, pixel split) Gram on the tensor cores.  RELINQUISH:
// the CTA frees its tensor-memory allocation permit after allocating (a CTA
// that runs one unit); a persistent CTA that allocates again for its next
// unit keeps the permit.  Returns true when a bounded wait expired (the
// error flag is raised and the unit's Gram is not written).
template <bool RELINQUISH>
__device__ __forceinline__ bool gram_tc_body(const ClassDev& c, int rcap, int bx) {
  extern __shared__ __align__(1024) uint8_t tsm[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  __shared__ int4 box[UPH_MAXN];
  __shared__ float fcs[UPH_MAXN];
  __shared__ float bgs[UPH_MAXBG];    // background coefficients of the residual
  __shared__ int16_t srk[UPH_MAXK], srs[UPH_MAXK];
  __shared__ float swt[2][KC];
  __shared__ float rsd[2][KC];
  __shared__ int pwy[2][KC], pwx[2][KC];   // window pixel of each chunk slot
  __shared__ int abort_flag;
  const int split = bx % c.tc_split;
  const int ib = bx / c.tc_split;
  const int isl = ib / c.nb, b = ib % c.nb;
  if (isl >= c.n_isl || !isl_active(c.flags[isl], PH_LIN)) return false;
  const int K = gram_rows(c, isl);
  if (!tc_island(c, isl, K)) return false;   // handled by k_gram_lin
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Mh = (K + 127) / 128;            // M = 128 halves
  const int R = Mh * 128;                    // stored rows
  const int N = (K + 15) & ~15;              // MMA N (<= 256)
  int ncols = 32;
  while (ncols < Mh * N) ncols <<= 1;        // power of two >= 32
  const int16_t* rk = c.row_k + (size_t)isl * c.Kmax;
  const int16_t* rs = c.row_s + (size_t)isl * c.Kmax;
  const int nr = c.isl_nr[isl];
  for (int k = tid; k < c.N; k += NT) {
    MemberBox mb = member_box(c, isl, c.p, k);
    box[k] = make_int4(mb.wx0, mb.wy0, mb.bw, mb.bh);
    fcs[k] = c.fcur[((size_t)isl * c.nb + b) * c.NL + k];
  }
  for (int j = tid; j < c.nbg; j += NT)
    bgs[j] = c.fcur[((size_t)isl * c.nb + b) * c.NL + c.N + j];
  for (int r = tid; r < K; r += NT) {
    srk[r] = rk[r];
    srs[r] = rs[r];
  }
  const size_t sbytes = stage_bytes(rcap);
  {
    // rows K..R-1 of both stages stay zero for the whole kernel
    uint4* z = reinterpret_cast<uint4*>(tsm);
    const int n16 = (int)(2 * sbytes / 16);
    for (int i = tid; i < n16; i += NT) z[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  if (tid == 0) {
    abort_flag = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&tmem_base)), "r"(ncols));
    if (RELINQUISH) asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    asm volatile("tcgen05.fence::before_thread_sync;");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tbase = tmem_base;
  if (tid == 0 && split == 0) gram_work(c, WK_GRAM_TC, rk, rs, K, box);
  const int B = c.B, Sz = c.Sz, npix = B * B;
  const size_t plane = (size_t)c.Hp * c.Wp;
  const float* dbase = c.dstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
  const float* wbase = c.wstack + b * plane + (size_t)c.oy[isl] * c.Wp + c.ox[isl];
  const int nchunk = (npix + KC - 1) / KC;
  const int cps = (nchunk + c.tc_split - 1) / c.tc_split;   // chunks per split
  const int ch0 = split * cps, ch1 = min(nchunk, ch0 + cps);
  const uint32_t idesc = umma_idesc(N);
  const uint32_t lbo = (uint32_t)R * 16u;    // between the two 8-pixel halves
  const uint32_t sbo = 128u;                 // between 8-row groups
  uint32_t phase[2] = {0u, 0u};   // next parity to wait for, per stage
  int issued[2] = {0, 0}, waited[2] = {0, 0};
  for (int ch = ch0; ch < ch1; ++ch) {
    const int lc = ch - ch0;   // chunk index within this split
    const int st = lc & 1;
    uint8_t* zh = tsm + st * sbytes;
    uint8_t* zl = zh + (size_t)rcap * KC * 2;
    if (lc >= 2) {
      // the MMAs of chunk lc - 2 read this stage: wait for their commit
      // (an expired wait is not counted as observed: the drain below waits
      // for that commit again before the tensor memory is freed)
      if (tid == 0) {
        if (mbar_wait(&mbar[st], phase[st])) {
          phase[st] ^= 1u;
          ++waited[st];
        } else {
          abort_flag = 1;
        }
      }
      __syncthreads();
      if (abort_flag) break;
    }
    const int pix0 = ch * KC;
    if (tid < KC) {
      // window pixel, sqrt(w) and the weighted residual sqrt(w) (d - sum_k fc_k m_k)
      const int pix = pix0 + tid;
      int wy = -1, wx = 0;
      float sw = 0.f, rv = 0.f;
      if (pix < npix) {
        wy = pix / B;
        wx = pix - wy * B;
        sw = sqrtf(wbase[(size_t)wy * c.Wp + wx]);
        float model = 0.f;
        for (int k = 0; k < nr; ++k) {
          const int4 bx = box[k];
          const int ly = wy - bx.y, lx = wx - bx.x;
          if (ly >= 0 && ly < bx.w && lx >= 0 && lx < bx.z)
            model = fmaf(fcs[k], c.stamps[stamp_slot(c, isl, b, k, 0) + (size_t)ly * Sz + lx],
                         model);
        }
        for (int j = 0; j < c.nbg; ++j) model = fmaf(bgs[j], bg_basis(j, wy, wx, B), model);
        rv = sw * (dbase[(size_t)wy * c.Wp + wx] - model);
      }
      pwy[st][tid] = wy;
      pwx[st][tid] = wx;
      swt[st][tid] = sw;
      rsd[st][tid] = rv;
    }
    __syncthreads();
    // warp tiles of (8-pixel group g, 32 consecutive rows); lane = row
    const int ntile = NG * ((K + 31) >> 5);
    for (int t = warp; t < ntile; t += NT / 32) {
      const int g = t & (NG - 1);
      const int r = (t >> 3) * 32 + lane;
      if (r >= K) continue;
      float v[8];
      const int s = srs[r];
      if (s <= -2) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int q = g * 8 + j;
          v[j] = pwy[st][q] >= 0 ? bg_basis(-2 - s, pwy[st][q], pwx[st][q], B) * swt[st][q]
                                 : 0.f;
        }
      } else if (s < 0) {
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = rsd[st][g * 8 + j];
      } else {
        const int k = srk[r];
        const int4 bx = box[k];
        const float* sp = c.stamps + stamp_slot(c, isl, b, k, s);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int q = g * 8 + j;
          const int ly = pwy[st][q] - bx.y, lx = pwx[st][q] - bx.x;
          float val = 0.f;
          if (pwy[st][q] >= 0 && ly >= 0 && ly < bx.w && lx >= 0 && lx < bx.z)
            val = sp[(size_t)ly * Sz + lx] * swt[st][q];
          v[j] = val;
        }
      }
      uint32_t hw[4], lw[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const __nv_bfloat16 h0 = __float2bfloat16_rn(v[2 * j]);
        const __nv_bfloat16 h1 = __float2bfloat16_rn(v[2 * j + 1]);
        const __nv_bfloat16 l0 = __float2bfloat16_rn(v[2 * j] - __bfloat162float(h0));
        const __nv_bfloat16 l1 = __float2bfloat16_rn(v[2 * j + 1] - __bfloat162float(h1));
        hw[j] = pack_bf16(h0, h1);
        lw[j] = pack_bf16(l0, l1);
      }
      const uint32_t off = (uint32_t)((g * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16);
      *reinterpret_cast<uint4*>(zh + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
      *reinterpret_cast<uint4*>(zl + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
    // make the generic-proxy stores visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t ah = smem_u32(zh), al = smem_u32(zl);
      for (int s = 0; s < KC / 16; ++s) {
        const uint32_t koff = (uint32_t)(2 * s * (R >> 3)) * 128u;
        for (int h = 0; h < Mh; ++h) {
          const uint32_t moff = (uint32_t)(h * 16) * 128u;
          const uint32_t dt = tbase + (uint32_t)(h * N);
          const uint32_t acc0 = (lc > 0 || s > 0) ? 1u : 0u;
          mma_bf16(dt, umma_desc(ah + koff + moff, lbo, sbo),
                   umma_desc(ah + koff, lbo, sbo), idesc, acc0);
          mma_bf16(dt, umma_desc(ah + koff + moff, lbo, sbo),
                   umma_desc(al + koff, lbo, sbo), idesc, 1u);
          mma_bf16(dt, umma_desc(al + koff + moff, lbo, sbo),
                   umma_desc(ah + koff, lbo, sbo), idesc, 1u);
        }
      }
      mma_commit(&mbar[st]);
      ++issued[st];
    }
  }
  // drain: wait for every commit not yet observed, so that no MMA this CTA
  // issued still writes the tensor memory when it is freed below.  Each
  // wait is bounded; after an expiry the commit gets one more bounded wait
  // before the kernel gives up on it (error flag raised, memory freed).
  if (tid == 0) {
    for (int st = 0; st < 2; ++st) {
      while (waited[st] < issued[st]) {
        if (!mbar_wait(&mbar[st], phase[st])) {
          abort_flag = 1;
          if (!mbar_wait(&mbar[st], phase[st])) break;
        }
        phase[st] ^= 1u;
        ++waited[st];
      }
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (abort_flag) {
    if (tid == 0) atomicExch(c.err, 1);
  } else if (warp < 4) {
    float* out = (c.tc_split > 1 ? c.gpart + (size_t)split * c.n_isl * c.nb * c.Kmax * c.Kmax
                                  : c.gram) +
                 ((size_t)isl * c.nb + b) * c.Kmax * c.Kmax;
    const int ld = c.Kmax;
    for (int h = 0; h < Mh; ++h) {
      const int row = h * 128 + warp * 32 + lane;
      for (int c0 = 0; c0 < N; c0 += 16) {
        uint32_t v[16];
        const uint32_t ta = tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(h * N + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
              "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
              "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(ta));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < K)
          for (int j = 0; j < 16; ++j)
            if (c0 + j < K) out[row * ld + c0 + j] = ch1 > ch0 ? __uint_as_float(v[j]) : 0.f;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(ncols));
  return abort_flag != 0;
}

__global__ void __launch_bounds__(NT) k_gram_tc(ClassDev c, int rcap) {
  gram_tc_body<true>(c, rcap, blockIdx.x);
}

// Sum of the tc_split partial Grams of every tensor-core island, in split
// order (deterministic), into the chunk's Gram.
__device__ __forceinline__ void gram_tc_reduce_body(const ClassDev& c, int bx) {
  const int isl = bx / c.nb, b = bx % c.nb;
  if (isl >= c.n_isl || !isl_active(c.flags[isl], PH_LIN)) return;
  const int K = gram_rows(c, isl);
  if (!tc_island(c, isl, K)) return;
  const size_t mat = (size_t)c.Kmax * c.Kmax;
  const size_t stride = (size_t)c.n_isl * c.nb * mat;
  const float* src = c.gpart + ((size_t)isl * c.nb + b) * mat;
  float* dst = c.gram + ((size_t)isl * c.nb + b) * mat;
  for (int e = threadIdx.x; e < K * K; e += NT) {
    const int r = e / K, q = e - (e / K) * K;
    const size_t o = (size_t)r * c.Kmax + q;
    float t = src[o];
    for (int sp = 1; sp < c.tc_split; ++sp) t += src[sp * stride + o];
    dst[o] = t;
  }
}

__global__ void __launch_bounds__(NT) k_gram_tc_reduce(ClassDev c) {
  gram_tc_reduce_body(c, blockIdx.x);
}

// Queue kernels of the LM loop: the tensor-core Grams of every active island
// of the job (a persistent CTA allocates and frees tensor memory per unit and
// keeps its allocation permit; it stops after an expired wait), and their
// split reductions.
__global__ void __launch_bounds__(NT, 3) kq_gram_tc(QueueList q) {
  queue_run(q, QK_GTC, 1, [&](const ClassDev& c, int isl, int u) {
    const int kmax = c.Kmax < UPH_MAXK ? c.Kmax : UPH_MAXK;
    return gram_tc_body<false>(c, rows_cap(kmax), isl * c.nb * c.tc_split + u);
  });
}

__global__ void __launch_bounds__(NT) kq_gram_tc_reduce(QueueList q) {
  queue_run(q, QK_GTCR, 1, [&](const ClassDev& c, int isl, int u) {
    gram_tc_reduce_body(c, isl * c.nb + u);
    return false;
  });
}

}  // namespace

void launch_q_gram_tc(const QueueList& q, size_t smem, bool reduce, int sms, cudaStream_t s) {
  int per = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kq_gram_tc, NT, smem) != cudaSuccess ||
      per < 1)
    per = 1;
  kq_gram_tc<<<(unsigned)std::max(1, q.per_cta ? q.cap[QK_GTC] : std::min(per * sms, q.cap[QK_GTC])),
               NT, smem, s>>>(q);
  if (reduce) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kq_gram_tc_reduce, NT, 0) !=
            cudaSuccess || per < 1)
      per = 1;
    kq_gram_tc_reduce<<<(unsigned)std::max(
                            1, q.per_cta ? q.cap[QK_GTCR] : std::min(per * sms, q.cap[QK_GTCR])),
                        NT, 0, s>>>(q);
  }
}

int gram_tc_splits(int n_isl, int nb, int B, int sm_count) {
  // enough CTAs for about four per SM, each over at least 8 pixel chunks
  const int nchunk = (B * B + KC - 1) / KC;
  const int cap = std::max(1, std::min(16, nchunk / 8));
  const int want = (4 * sm_count + n_isl * nb - 1) / (n_isl * nb);
  return std::max(1, std::min(cap, want));
}

size_t gram_tc_smem_bytes(int kmax) { return 2 * stage_bytes(rows_cap(kmax)); }

void launch_gram_tc(const ClassDev& c, cudaStream_t s) {
  const int kmax = c.Kmax < UPH_MAXK ? c.Kmax : UPH_MAXK;
  k_gram_tc<<<(unsigned)(c.n_isl * c.nb * c.tc_split), NT, gram_tc_smem_bytes(kmax), s>>>(
      c, rows_cap(kmax));
  if (c.tc_split > 1) k_gram_tc_reduce<<<(unsigned)(c.n_isl * c.nb), NT, 0, s>>>(c);
}

int uph_gram_tc_setup() {
  const cudaError_t e = cudaFuncSetAttribute(k_gram_tc,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)gram_tc_smem_bytes(UPH_MAXK));
  if (e != cudaSuccess) return (int)e;
  return (int)cudaFuncSetAttribute(kq_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)gram_tc_smem_bytes(UPH_MAXK));
}

// Mixed-precision ISDF matvec on the 5th-generation tensor cores (sm_100a).
//
// H = p(C) with C = R^2 + 4 R^1/2 (C_isdf^T M C_isdf) R^1/2 is applied as
//   T = C_isdf (R^1/2 x)          GEMM1: (n_isdf x ncv) . (ncv x nb)
//   Z = D^T T,  D = M C_isdf      GEMM2: (ncv x n_isdf) . (n_isdf x nb)
//   C x = R^2 x + 4 R^1/2 Z       (diagonal part in FP64, fused in GEMM2's epilogue)
// so M is folded into the second operand once per operator.  Both GEMMs are
// tcgen05.mma kind::f16 (BF16 in, FP32 accumulate in TMEM), operands staged by
// TMA (128-byte swizzle, no multicast), with a split-BF16 compensated product:
// every FP64/FP32 operand is stored as hi = bf16(x), lo = bf16(x - hi) and the
// product is hi*hi + hi*lo + lo*hi, accumulated in one TMEM tile.
//
// The polynomial p is evaluated by the Clenshaw recurrence in the Chebyshev
// basis of the interval [lo, hi] containing the spectrum of C (the same
// polynomial as the reference's monomial Horner form, re-expanded on the host):
//   b_n = g_n v ; b_k = g_k v + 2 Chat b_{k+1} - b_{k+2} ; p(C) v = g_0 v + Chat b_1 - b_2
//   Chat = (C - c0) / c1, c0 = (hi+lo)/2, c1 = (hi-lo)/2.
// The Clenshaw combine is fused into GEMM2's epilogue, which also writes the
// split-BF16 operand of the next GEMM1.  Lanczos vectors stay FP64.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>
#include <vector>

#include <cooperative_groups.h>

#include "ngw_internal.h"
#include "tc_gemm.cuh"

namespace cg = cooperative_groups;

namespace ngw {

using bf16 = __nv_bfloat16;

constexpr int BM = 128;
constexpr int BK = 64;

enum EpiKind { EPI_SPLIT = 0, EPI_CLENSHAW = 1 };

struct EpiParams {
  int kind;
  int Mv, Nv;            // valid rows / cols of D
  // EPI_SPLIT: D(m, n) -> out_hi/lo[n * ldo + m]
  bf16 *out_hi, *out_lo;
  int ldo;
  // split-K partials (EPI_SPLIT with nsplit > 1), reduced by k_splitk_reduce
  float *ws;
  // EPI_CLENSHAW: rows m = pair index, cols n = chain
  const double *s;       // sqrtR (Mv)
  const float *x;        // b_{k+1}  [n * ldx + m]
  const float *b2;       // b_{k+2}  (nullable)
  const float *v;        // the vector p is applied to (deflated), FP32 [n * ldx + m]
  int ldx, ldv;          // ldv: leading dimension of out64
  // final step only: out64 += Up(m, :) . xo(:, n) (deflated eigenpairs, FP64)
  const double *Up;      // (ncv, kdef) column-major
  const double *xo;      // (kdef, nb) column-major
  int kdef;
  double gamma, alpha, c0, beta;
  int tda;
  float *out32;          // b_k (nullable)
  double *out64;         // final p(C) v (nullable)
  bf16 *s_hi, *s_lo;     // split of (R^1/2 or 1) * out  [n * lds + m] (nullable)
  int lds;
  int ring;              // EPI_CLENSHAW in k_tc_gemm: operands through the TMA chunk ring
  int dense;             // EPI_CLENSHAW as a plain product: out64 = z (+ deflated term), no operands
};

struct GemmArgs {
  int num_kb;            // k-blocks per segment
  int nseg;              // 1..3 split segments
  int nsplit;            // split-K factor
};

__device__ __forceinline__ void split_bf16(float v, bf16 &hi, bf16 &lo) {
  hi = __float2bfloat16_rn(v);
  lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

constexpr int NTHREADS = 256;

// Clenshaw operands b_{k+1}, b_{k+2} and v of row m for the 8 columns from
// nbase (zero past the valid rows / columns and for absent vectors).
__device__ __forceinline__ void clenshaw_operands(const EpiParams &ep, bool mv, int m, int nbase, float *x,
                                                  float *b2, float *v) {
  const int nj = mv ? min(8, ep.Nv - nbase) : 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const size_t o = (size_t)(nbase + j) * ep.ldx + m;
    x[j] = (j < nj && ep.x) ? __ldg(ep.x + o) : 0.f;
    b2[j] = (j < nj && ep.b2) ? __ldg(ep.b2 + o) : 0.f;
    v[j] = (j < nj && ep.v) ? __ldg(ep.v + o) : 0.f;
  }
}

// The same for the 4 columns n, n + step, ... below n_end.
__device__ __forceinline__ void clenshaw_operands4(const EpiParams &ep, bool mv, int m, int n, int step, int n_end,
                                                   float *x, float *b2, float *v) {
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int nn = n + j * step;
    const bool ok = mv && nn < n_end && nn < ep.Nv;
    const size_t o = (size_t)nn * ep.ldx + m;
    x[j] = (ok && ep.x) ? __ldg(ep.x + o) : 0.f;
    b2[j] = (ok && ep.b2) ? __ldg(ep.b2 + o) : 0.f;
    v[j] = (ok && ep.v) ? __ldg(ep.v + o) : 0.f;
  }
}

// Clenshaw step in FP32.  The row coefficient (R^2 or R) - c0 is formed in
// FP64 once per row and rounded once, so the combine
//   out = gamma v + alpha ((R^2 - c0) x + 4 R^1/2 z) - beta b2   (TDA: R, 2)
// has no cancellation of R^2 x against c0 x and runs as three FP32 FMAs; its
// inputs and outputs are FP32 (or split BF16) anyway, so FP64 here only cost
// issue slots (FP64 and conversion pipes are narrow on this part).
struct ClenCoef {
  float d;             // (R^2 or R) - c0
  float kz;            // 4 R^1/2 or 2
  float sc;            // R^1/2 or 1: scale of the split output
  float ga, al, mbe;   // gamma, alpha, -beta
};

__device__ __forceinline__ ClenCoef clen_coef(const EpiParams &ep, double si) {
  ClenCoef k;
  if (ep.dense) {   // out = z
    k.d = 0.f;
    k.kz = 1.f;
    k.sc = 1.f;
    k.ga = 0.f;
    k.al = 1.f;
    k.mbe = 0.f;
    return k;
  }
  const double s2 = si * si;
  k.d = (float)((ep.tda ? s2 : s2 * s2) - ep.c0);
  k.kz = (float)(ep.tda ? 2.0 : 4.0 * si);
  k.sc = (float)(ep.tda ? 1.0 : si);
  k.ga = (float)ep.gamma;
  k.al = (float)ep.alpha;
  k.mbe = (float)(-ep.beta);
  return k;
}

__device__ __forceinline__ float clen_out(const ClenCoef &k, float x, float z, float v, float b2) {
  const float t = fmaf(k.d, x, k.kz * z);
  return fmaf(k.al, t, fmaf(k.ga, v, k.mbe * b2));
}

// Stores of one Clenshaw output element (row m, chain n).
__device__ __forceinline__ void clen_store(const EpiParams &ep, const ClenCoef &k, int m, int n, float o) {
  if (ep.out32) ep.out32[(size_t)n * ep.ldx + m] = o;
  if (ep.out64) {
    double od = (double)o;
    for (int q = 0; q < ep.kdef; ++q) od += ep.Up[(size_t)q * ep.Mv + m] * ep.xo[(size_t)n * ep.kdef + q];
    ep.out64[(size_t)n * ep.ldv + m] = od;
  }
  if (ep.s_hi) {
    bf16 hi, lo;
    split_bf16(k.sc * o, hi, lo);
    ep.s_hi[(size_t)n * ep.lds + m] = hi;
    ep.s_lo[(size_t)n * ep.lds + m] = lo;
  }
}

// One 128 x BN output tile (rows m0.., columns n0.., split-K slice `split`,
// `tile` its index for the split-K workspace) of a CTA: warp 0 issues
// the TMA loads, warp 1 the MMAs into TMEM, then all 8 warps run the epilogue.
template <int BN, int STAGES, bool FUSED, bool CRED>
__device__ __forceinline__ void tc_gemm_tile(const CUtensorMap *tA_hi, const CUtensorMap *tA_lo,
                                             const CUtensorMap *tB_hi, const CUtensorMap *tB_lo,
                                             const CUtensorMap *tRx, const CUtensorMap *tRb2,
                                             const CUtensorMap *tRv, const GemmArgs &ga, const EpiParams &ep,
                                             int m0, int n0, int split, int tile, int *status) {
  // FUSED: one stage holds A_hi, A_lo, B_hi, B_lo of a k-block and carries all
  // three split products; otherwise one stage is one (A, B) pair of a segment.
  constexpr uint32_t A_BYTES = BM * BK * 2;
  constexpr uint32_t B_BYTES = BN * BK * 2;
  constexpr uint32_t STAGE_BYTES = FUSED ? 2 * (A_BYTES + B_BYTES) : A_BYTES + B_BYTES;
  constexpr uint32_t TMEM_COLS = (BN <= 32) ? 32 : (BN <= 64) ? 64 : (BN <= 128) ? 128 : 256;
  constexpr uint32_t IDESC = tc::idesc_bf16_f32(BM, BN);
  constexpr int NCH = BN / 16;             // 16-column chunks
  constexpr int NCH0 = (NCH + 1) / 2;      // chunks of warpgroup 0

  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  __shared__ __align__(8) uint64_t full_bar[STAGES];
  __shared__ __align__(8) uint64_t empty_bar[STAGES];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ __align__(8) uint64_t ring_bar[2][4];   // Clenshaw operand ring, per warpgroup
  __shared__ uint32_t tmem_base_sh;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int total_kb = FUSED ? ga.num_kb : ga.num_kb * ga.nseg;
  const int kb_per = (total_kb + ga.nsplit - 1) / ga.nsplit;
  const int kb_begin = split * kb_per;
  const int kb_end = min(total_kb, kb_begin + kb_per);
  const int nkb = max(0, kb_end - kb_begin);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(tc::smem_u32(&full_bar[s]), 1);
      tc::mbar_init(tc::smem_u32(&empty_bar[s]), 1);
    }
    tc::mbar_init(tc::smem_u32(&done_bar), 1);
    for (int g = 0; g < 2; ++g)
      for (int r = 0; r < 4; ++r) tc::mbar_init(tc::smem_u32(&ring_bar[g][r]), 1);
    tc::fence_barrier_init();
    tc::prefetch_tmap(tA_hi);
    tc::prefetch_tmap(tB_hi);
  }
  if (warp == 2) {
    tc::tmem_alloc(tc::smem_u32(&tmem_base_sh), TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem_d = tmem_base_sh;
  tc::pdl_wait();                 // operands / epilogue inputs come from the previous kernel
  tc::pdl_launch_dependents();

  if (warp == 0 && lane == 0) {
    // ---- TMA producer: k-blocks of the concatenated segments ----
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      if (i >= STAGES) {
        if (!tc::mbar_wait(tc::smem_u32(&empty_bar[s]), ((i / STAGES) - 1) & 1, status)) break;
      }
      const int kbg = kb_begin + i;
      const uint32_t bar = tc::smem_u32(&full_bar[s]);
      const uint32_t sa = tc::smem_u32(smem + s * STAGE_BYTES);
      tc::mbar_arrive_expect_tx(bar, STAGE_BYTES);
      if (FUSED) {
        tc::tma_load_2d(sa, tA_hi, bar, kbg * BK, m0);
        tc::tma_load_2d(sa + A_BYTES, tA_lo, bar, kbg * BK, m0);
        tc::tma_load_2d(sa + 2 * A_BYTES, tB_hi, bar, kbg * BK, n0);
        tc::tma_load_2d(sa + 2 * A_BYTES + B_BYTES, tB_lo, bar, kbg * BK, n0);
      } else {
        const int seg = kbg / ga.num_kb;
        const int kb = kbg - seg * ga.num_kb;
        const CUtensorMap *ta = (seg == 2) ? tA_lo : tA_hi;   // (hi,hi) (hi,lo) (lo,hi)
        const CUtensorMap *tb = (seg == 1) ? tB_lo : tB_hi;
        tc::tma_load_2d(sa, ta, bar, kb * BK, m0);
        tc::tma_load_2d(sa + A_BYTES, tb, bar, kb * BK, n0);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer (single thread) ----
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      if (!tc::mbar_wait(tc::smem_u32(&full_bar[s]), (i / STAGES) & 1, status)) break;
      tc::tc_fence_after();
      const uint32_t sa = tc::smem_u32(smem + s * STAGE_BYTES);
      if (FUSED) {
        const uint32_t sal = sa + A_BYTES, sbh = sa + 2 * A_BYTES, sbl = sbh + B_BYTES;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
          const uint32_t acc0 = (i > 0 || kk > 0) ? 1u : 0u;
          tc::mma_bf16(tmem_d, tc::smem_desc_sw128(sa + kk * 32), tc::smem_desc_sw128(sbh + kk * 32), IDESC, acc0);
          tc::mma_bf16(tmem_d, tc::smem_desc_sw128(sa + kk * 32), tc::smem_desc_sw128(sbl + kk * 32), IDESC, 1u);
          tc::mma_bf16(tmem_d, tc::smem_desc_sw128(sal + kk * 32), tc::smem_desc_sw128(sbh + kk * 32), IDESC, 1u);
        }
      } else {
        const uint32_t sb = sa + A_BYTES;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
          const uint64_t ad = tc::smem_desc_sw128(sa + kk * 32);
          const uint64_t bd = tc::smem_desc_sw128(sb + kk * 32);
          tc::mma_bf16(tmem_d, ad, bd, IDESC, (i > 0 || kk > 0) ? 1u : 0u);
        }
      }
      tc::mma_commit(tc::smem_u32(&empty_bar[s]));
    }
    tc::mma_commit(tc::smem_u32(&done_bar));
  }
  __syncwarp();

  // ---- epilogue: 8 warps; warp w reads TMEM lanes 32*(w%4).., warpgroup w/4
  // takes one half of the 16-column chunks ----
  const int wl = warp & 3, wg = warp >> 2;
  const int mloc = wl * 32 + lane;
  const int m = m0 + mloc;
  const uint32_t trow = tmem_d + ((uint32_t)(wl * 32) << 16);
  const int ch_begin = wg == 0 ? 0 : NCH0;
  const int ch_end = wg == 0 ? NCH0 : NCH;
  // The Clenshaw operands (b_{k+1}, b_{k+2}, v) do not depend on the product:
  // the first 8-column chunk of them is loaded while the MMAs still run, and
  // every later chunk one iteration ahead of its use.
  const bool clenshaw = !CRED && ep.kind == EPI_CLENSHAW;
  const bool mv = m < ep.Mv;
  float px[8], pb[8], pv[8];
  double si = 0.0;
  if (clenshaw) {
    if (mv) si = ep.s[m];
    if (!ep.ring) clenshaw_operands(ep, mv, m, n0 + 16 * ch_begin, px, pb, pv);
  }
  // Cluster split-K: this CTA finishes the tile columns [c_lo, c_hi); thread
  // row crow takes c_first, c_first + cstep, ... in groups of 4, the Clenshaw
  // operands of each group loaded one group ahead (the first before the wait).
  int c_lo = 0, c_hi = 0;
  if constexpr (CRED) {
    const int cpr = (BN + ga.nsplit - 1) / ga.nsplit;
    c_lo = (int)cg::this_cluster().block_rank() * cpr;
    c_hi = min(BN, c_lo + cpr);
  }
  constexpr int cstep = NTHREADS / BM;
  const int crow = threadIdx.x % BM;
  const int c_first = c_lo + (int)threadIdx.x / BM;
  const int mm = m0 + crow;
  const bool cred_clenshaw = CRED && ep.kind == EPI_CLENSHAW;
  float qx[4], qb[4], qv[4];
  double csi = 0.0;
  if (cred_clenshaw) {
    if (mm < ep.Mv) csi = ep.s[mm];
    clenshaw_operands4(ep, mm < ep.Mv, mm, n0 + c_first, cstep, n0 + c_hi, qx, qb, qv);
  }
  const bool have = tc::mbar_wait(tc::smem_u32(&done_bar), 0, status) && nkb > 0;
  tc::tc_fence_after();

  if (CRED) {
    // Split-K inside a thread-block cluster (the nsplit CTAs of this tile):
    // every CTA stages its FP32 partial tile in its own shared memory (the
    // pipeline stages are free now), then CTA r sums the column slice r over
    // the cluster's CTAs in split order through distributed shared memory
    // and finishes those columns with the epilogue: the split-BF16 result
    // (the same sums, in the same order, as k_splitk_reduce, without the
    // global round trip and the extra launch) or the Clenshaw step.
    float *part = reinterpret_cast<float *>(smem);
    for (int ch = 2 * ch_begin; ch < 2 * ch_end; ++ch) {
      const int c = ch * 8;
      float v[8];
      if (have) {
        tc::tmem_ld8(trow + c, v);
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = 0.f;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) part[(c + j) * BM + mloc] = v[j];
    }
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    const int ns = ga.nsplit;
    const ClenCoef kc = clen_coef(ep, csi);
    for (int c = c_first; c < c_hi; c += 4 * cstep) {
      float cx[4], cb[4], cv[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        cx[j] = qx[j];
        cb[j] = qb[j];
        cv[j] = qv[j];
      }
      if (cred_clenshaw && c + 4 * cstep < c_hi)
        clenshaw_operands4(ep, mm < ep.Mv, mm, n0 + c + 4 * cstep, cstep, n0 + c_hi, qx, qb, qv);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int cc = c + j * cstep;
        if (cc >= c_hi) break;
        float acc = 0.f;
        for (int q = 0; q < ns; ++q) acc += cl.map_shared_rank(part, q)[cc * BM + crow];
        const int n = n0 + cc;
        if (mm >= ep.Mv || n >= ep.Nv) continue;
        if (ep.kind == EPI_SPLIT) {
          bf16 hi, lo;
          split_bf16(acc, hi, lo);
          ep.out_hi[(size_t)n * ep.ldo + mm] = hi;
          ep.out_lo[(size_t)n * ep.ldo + mm] = lo;
        } else {
          // the Clenshaw step of the EPI_CLENSHAW branch below, for one element
          clen_store(ep, kc, mm, n, clen_out(kc, cx[j], acc, cv[j], cb[j]));
        }
      }
    }
    cl.sync();   // no CTA leaves while another still reads its shared memory
  } else if (ep.kind == EPI_SPLIT) {
    const bool partial = ga.nsplit > 1;
    float *wsl = partial ? ep.ws + ((size_t)tile * ga.nsplit + split) * (size_t)(BN * BM) : nullptr;
    for (int ch = 2 * ch_begin; ch < 2 * ch_end; ++ch) {
      const int c = ch * 8;
      float v[8];
      if (have) {
        tc::tmem_ld8(trow + c, v);
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = 0.f;
      }
      if (partial) {
#pragma unroll
        for (int j = 0; j < 8; ++j) wsl[(size_t)(c + j) * BM + mloc] = v[j];
      } else if (m < ep.Mv) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int n = n0 + c + j;
          if (n < ep.Nv) {
            bf16 hi, lo;
            split_bf16(v[j], hi, lo);
            ep.out_hi[(size_t)n * ep.ldo + m] = hi;
            ep.out_lo[(size_t)n * ep.ldo + m] = lo;
          }
        }
      }
    }
  } else {
    // EPI_CLENSHAW: out = gamma v + alpha ((R^2 - c0) x + 4 R^1/2 z) - beta b2
    // (TDA: R - c0, 2 z) in FP32 (clen_out); split((R^1/2 or 1) out).
    // 8-column chunks keep the register count low enough for 2 CTAs per SM.
    const ClenCoef kc = clen_coef(ep, si);
    if (ep.ring) {
      // Operand ring in the stage memory the MMAs no longer need: per
      // warpgroup RS slots of one 8-column chunk (b_{k+1} | b_{k+2} | v,
      // 128 rows each).  The warpgroup's first thread fills a slot with
      // three bulk tensor copies and refills it once all four warps have
      // read it (named barrier), RS chunks ahead of its use.
      constexpr uint32_t OP8 = BM * 8 * 4;
      constexpr uint32_t CHUNK = 3 * OP8;
      constexpr int RS = (int)((STAGES * STAGE_BYTES) / (2 * CHUNK)) < 4 ? (int)((STAGES * STAGE_BYTES) / (2 * CHUNK)) : 4;
      static_assert(RS >= 1, "stage memory too small for the operand ring");
      const uint32_t ring = tc::smem_u32(smem) + (uint32_t)(wg * RS) * CHUNK;
      const float *ringf = reinterpret_cast<const float *>(smem + (size_t)wg * RS * CHUNK);
      const bool leader = (threadIdx.x & 127) == 0;
      const int nq = 2 * (ch_end - ch_begin);
      const int c_first = 16 * ch_begin;
      const uint32_t bytes = OP8 * (1u + (ep.b2 ? 1u : 0u) + (ep.v ? 1u : 0u));
      const uint64_t pol_once = tc::l2_evict_first(), pol_keep = tc::l2_evict_last();
      auto issue = [&](int q) {
        const int r = q % RS;
        const uint32_t bar = tc::smem_u32(&ring_bar[wg][r]);
        const uint32_t dst = ring + (uint32_t)r * CHUNK;
        const int nc = n0 + c_first + 8 * q;
        tc::mbar_arrive_expect_tx(bar, bytes);
        // b_{k+1}, b_{k+2}: one more read each at most; v: read by every GEMM2 of the step
        tc::tma_load_2d_hint(dst, tRx, bar, m0, nc, pol_once);
        if (ep.b2) tc::tma_load_2d_hint(dst + OP8, tRb2, bar, m0, nc, pol_once);
        if (ep.v) tc::tma_load_2d_hint(dst + 2 * OP8, tRv, bar, m0, nc, pol_keep);
      };
      if (leader)
        for (int q = 0; q < nq && q < RS; ++q) issue(q);
      for (int q = 0; q < nq; ++q) {
        const int r = q % RS;
        const int c = c_first + 8 * q;
        float z[8];
        if (have) {
          tc::tmem_ld8(trow + c, z);
        } else {
#pragma unroll
          for (int j = 0; j < 8; ++j) z[j] = 0.f;
        }
        const bool ok = tc::mbar_wait(tc::smem_u32(&ring_bar[wg][r]), (uint32_t)((q / RS) & 1), status);
        if (mv && ok) {
          const float *sl = ringf + (size_t)r * (CHUNK / 4) + mloc;
          const int nbase = n0 + c;
          const int nj = min(8, ep.Nv - nbase);
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            if (j >= nj) break;
            const float x = sl[j * BM];
            const float b2 = ep.b2 ? sl[OP8 / 4 + j * BM] : 0.f;
            const float v = ep.v ? sl[2 * (OP8 / 4) + j * BM] : 0.f;
            clen_store(ep, kc, m, nbase + j, clen_out(kc, x, z[j], v, b2));
          }
        }
        if (wg == 0)   // slot r read by the warpgroup (literal barrier ids 1 / 2)
          asm volatile("bar.sync 1, 128;" ::: "memory");
        else
          asm volatile("bar.sync 2, 128;" ::: "memory");
        if (leader && q + RS < nq) issue(q + RS);
      }
    } else
    for (int ch = 2 * ch_begin; ch < 2 * ch_end; ++ch) {
      const int c = ch * 8;
      float z[8];
      if (have) {
        tc::tmem_ld8(trow + c, z);
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) z[j] = 0.f;
      }
      float xv[8], b2v[8], vf[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        xv[j] = px[j];
        b2v[j] = pb[j];
        vf[j] = pv[j];
      }
      if (ch + 1 < 2 * ch_end) clenshaw_operands(ep, mv, m, n0 + c + 8, px, pb, pv);
      if (!mv) continue;
      const int nbase = n0 + c;
      const int nj = min(8, ep.Nv - nbase);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (j >= nj) break;
        clen_store(ep, kc, m, nbase + j, clen_out(kc, xv[j], z[j], vf[j], b2v[j]));
      }
    }
  }

  tc::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem_d, TMEM_COLS);
  }
}


template <int BN, int STAGES, int MINB, bool FUSED, bool CRED = false>
__global__ void __launch_bounds__(NTHREADS, MINB)
    k_tc_gemm(const __grid_constant__ CUtensorMap tA_hi, const __grid_constant__ CUtensorMap tA_lo,
              const __grid_constant__ CUtensorMap tB_hi, const __grid_constant__ CUtensorMap tB_lo,
              const __grid_constant__ CUtensorMap tRx, const __grid_constant__ CUtensorMap tRb2,
              const __grid_constant__ CUtensorMap tRv, GemmArgs ga, EpiParams ep, int *status) {
  tc_gemm_tile<BN, STAGES, FUSED, CRED>(&tA_hi, &tA_lo, &tB_hi, &tB_lo, &tRx, &tRb2, &tRv, ga, ep,
                                        blockIdx.x * BM, blockIdx.y * BN, blockIdx.z,
                                        blockIdx.y * gridDim.x + blockIdx.x, status);
}

// ---------------------------------------------------------------------------
// Grouped launch across molecules: one grid holds the tiles of several
// problems (one per molecule of a batch), each with its own operand tensor
// maps, shapes and epilogue in a device table.  Block b belongs to the entry
// g with tb[g] <= b < tb[g+1]; its tile t = b - tb[g] is (t % tiles_m,
// t / tiles_m).  nv[g] is the entry's chain count at this launch (chains that
// finished are not scheduled).  Fused stages, 64-wide N tiles, no split-K:
// the molecules together fill the GPU.  Per tile the arithmetic is that of
// k_tc_gemm<64, 4, 1, true> (variant 3), so a pinned variant-3 single call
// gives the same bits.
struct __align__(64) GroupEntry {
  CUtensorMap tA_hi, tA_lo, tB_hi, tB_lo;
  EpiParams ep;
  GemmArgs ga;
  int tiles_m;
};

constexpr int GBN = 64, GSTAGES = 4;

__global__ void __launch_bounds__(NTHREADS, 1)
    k_tc_gemm_grouped(const GroupEntry *__restrict__ tab, const int *__restrict__ tb, const int *__restrict__ nv,
                      int ng, int *status) {
  __shared__ EpiParams sep;
  __shared__ GemmArgs sga;
  __shared__ int sg, stile, stm;
  if (threadIdx.x == 0) {
    int g = 0;
    while (g + 1 < ng && (int)blockIdx.x >= tb[g + 1]) ++g;
    // the tensor maps sit in global memory (written by a host copy): order
    // those writes before this thread's tensor-map reads (it is the thread
    // that issues the TMA loads)
    const GroupEntry *eg = tab + g;
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&eg->tA_hi) : "memory");
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&eg->tA_lo) : "memory");
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&eg->tB_hi) : "memory");
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&eg->tB_lo) : "memory");
    sg = g;
    stile = (int)blockIdx.x - tb[g];
    stm = tab[g].tiles_m;
    sep = tab[g].ep;
    sep.Nv = nv[g];
    sga = tab[g].ga;
  }
  __syncthreads();
  const GroupEntry *e = tab + sg;
  const int t = stile, tm = stm;
  tc_gemm_tile<GBN, GSTAGES, true, false>(&e->tA_hi, &e->tA_lo, &e->tB_hi, &e->tB_lo, &e->tA_hi, &e->tA_hi,
                                          &e->tA_hi, sga, sep, (t % tm) * BM, (t / tm) * GBN, 0, t, status);
}

// ---------------------------------------------------------------------------
// Persistent, warp-specialised variant.  One CTA per SM walks a static list
// of work items (tile_m fastest, then tile_n, then split); each stage of the
// TMA ring holds A_hi, A_lo, B_hi and B_lo of one 64-wide k-block, so the three
// split-BF16 products (hi*hi, hi*lo, lo*hi) are 12 MMAs on operands loaded
// once.  Two TMEM accumulators alternate between tiles: the MMA thread fills
// one while the two epilogue warpgroups (warps 4-11) drain the other.
constexpr int PTHREADS = 384;

template <int BN, int STAGES>
__global__ void __launch_bounds__(PTHREADS, 1)
    k_tc_gemm_p(const __grid_constant__ CUtensorMap tA_hi, const __grid_constant__ CUtensorMap tA_lo,
                const __grid_constant__ CUtensorMap tB_hi, const __grid_constant__ CUtensorMap tB_lo,
                GemmArgs ga, EpiParams ep, int tiles_m, int tiles_n, int *status) {
  constexpr uint32_t A_BYTES = BM * BK * 2;
  constexpr uint32_t B_BYTES = BN * BK * 2;
  constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  constexpr uint32_t TMEM_COLS = (2 * BN <= 128) ? 128 : (2 * BN <= 256) ? 256 : 512;
  constexpr uint32_t ACC_STRIDE = TMEM_COLS / 2;   // accumulator buffers on aligned columns
  constexpr uint32_t IDESC = tc::idesc_bf16_f32(BM, BN);
  constexpr int NCH = BN / 8;               // 8-column chunks
  constexpr int NCH0 = (NCH + 1) / 2;       // chunks of epilogue warpgroup 0

  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  __shared__ __align__(8) uint64_t full_bar[STAGES];
  __shared__ __align__(8) uint64_t empty_bar[STAGES];
  __shared__ __align__(8) uint64_t accf_bar[2];
  __shared__ __align__(8) uint64_t acce_bar[2];
  __shared__ uint32_t tmem_base_sh;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int total_kb = ga.num_kb;           // k-blocks of the reduction (fused segments)
  const int kb_per = (total_kb + ga.nsplit - 1) / ga.nsplit;
  const int nwork = tiles_m * tiles_n * ga.nsplit;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(tc::smem_u32(&full_bar[s]), 1);
      tc::mbar_init(tc::smem_u32(&empty_bar[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(tc::smem_u32(&accf_bar[b]), 1);
      tc::mbar_init(tc::smem_u32(&acce_bar[b]), 256);
    }
    tc::fence_barrier_init();
    tc::prefetch_tmap(&tA_hi);
    tc::prefetch_tmap(&tA_lo);
    tc::prefetch_tmap(&tB_hi);
    tc::prefetch_tmap(&tB_lo);
  }
  if (warp == 2) {
    tc::tmem_alloc(tc::smem_u32(&tmem_base_sh), TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem_base = tmem_base_sh;
  tc::pdl_wait();                 // operands / epilogue inputs come from the previous kernel
  tc::pdl_launch_dependents();

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer ----
      int it = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < nwork && ok; w += gridDim.x) {
        const int tm = w % tiles_m, tn = (w / tiles_m) % tiles_n, sp = w / (tiles_m * tiles_n);
        const int kb0 = sp * kb_per, kb1 = min(total_kb, kb0 + kb_per);
        for (int kb = kb0; kb < kb1; ++kb, ++it) {
          const int s = it % STAGES;
          if (it >= STAGES && !tc::mbar_wait(tc::smem_u32(&empty_bar[s]), ((it / STAGES) - 1) & 1, status)) {
            ok = false;
            break;
          }
          const uint32_t bar = tc::smem_u32(&full_bar[s]);
          const uint32_t sa = tc::smem_u32(smem + s * STAGE_BYTES);
          tc::mbar_arrive_expect_tx(bar, STAGE_BYTES);
          tc::tma_load_2d(sa, &tA_hi, bar, kb * BK, tm * BM);
          tc::tma_load_2d(sa + A_BYTES, &tA_lo, bar, kb * BK, tm * BM);
          tc::tma_load_2d(sa + 2 * A_BYTES, &tB_hi, bar, kb * BK, tn * BN);
          tc::tma_load_2d(sa + 2 * A_BYTES + B_BYTES, &tB_lo, bar, kb * BK, tn * BN);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer ----
      int it = 0, t = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < nwork && ok; w += gridDim.x, ++t) {
        const int sp = w / (tiles_m * tiles_n);
        const int kb0 = sp * kb_per, kb1 = min(total_kb, kb0 + kb_per);
        const int buf = t & 1;
        if (t >= 2 && !tc::mbar_wait(tc::smem_u32(&acce_bar[buf]), ((t >> 1) - 1) & 1, status)) break;
        tc::tc_fence_after();
        const uint32_t tacc = tmem_base + buf * ACC_STRIDE;
        for (int kb = kb0; kb < kb1; ++kb, ++it) {
          const int s = it % STAGES;
          if (!tc::mbar_wait(tc::smem_u32(&full_bar[s]), (it / STAGES) & 1, status)) {
            ok = false;
            break;
          }
          tc::tc_fence_after();
          const uint32_t sa = tc::smem_u32(smem + s * STAGE_BYTES);
          const uint32_t sah = sa, sal = sa + A_BYTES, sbh = sa + 2 * A_BYTES, sbl = sbh + B_BYTES;
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
            const uint32_t acc0 = (kb > kb0 || kk > 0) ? 1u : 0u;
            tc::mma_bf16(tacc, tc::smem_desc_sw128(sah + kk * 32), tc::smem_desc_sw128(sbh + kk * 32), IDESC, acc0);
            tc::mma_bf16(tacc, tc::smem_desc_sw128(sah + kk * 32), tc::smem_desc_sw128(sbl + kk * 32), IDESC, 1u);
            tc::mma_bf16(tacc, tc::smem_desc_sw128(sal + kk * 32), tc::smem_desc_sw128(sbh + kk * 32), IDESC, 1u);
          }
          tc::mma_commit(tc::smem_u32(&empty_bar[s]));
        }
        tc::mma_commit(tc::smem_u32(&accf_bar[buf]));
      }
    }
  } else if (warp >= 4) {
    // ---- epilogue: warps 4..11, lanes 32*(warp%4).., warpgroup (warp-4)/4 ----
    const int wl = warp & 3, wg = (warp - 4) >> 2;
    const int mloc = wl * 32 + lane;
    const int ch_begin = wg == 0 ? 0 : NCH0;
    const int ch_end = wg == 0 ? NCH0 : NCH;
    int t = 0;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x, ++t) {
      const int tm = w % tiles_m, tn = (w / tiles_m) % tiles_n, sp = w / (tiles_m * tiles_n);
      const int kb0 = sp * kb_per, kb1 = min(total_kb, kb0 + kb_per);
      const int buf = t & 1;
      const int m0 = tm * BM, n0 = tn * BN;
      const int m = m0 + mloc;
      // Clenshaw operands of the first chunk, loaded before the accumulator is ready
      const bool mv = m < ep.Mv;
      float px[8], pb[8], pv[8];
      double si = 0.0;
      if (ep.kind == EPI_CLENSHAW) {
        if (mv) si = ep.s[m];
        clenshaw_operands(ep, mv, m, n0 + 8 * ch_begin, px, pb, pv);
      }
      const bool have = tc::mbar_wait(tc::smem_u32(&accf_bar[buf]), (t >> 1) & 1, status) && kb1 > kb0;
      tc::tc_fence_after();
      const uint32_t trow = tmem_base + buf * ACC_STRIDE + ((uint32_t)(wl * 32) << 16);
      if (ep.kind == EPI_SPLIT) {
        const bool partial = ga.nsplit > 1;
        const int tile = tn * tiles_m + tm;
        float *wsl = partial ? ep.ws + ((size_t)tile * ga.nsplit + sp) * (size_t)(BN * BM) : nullptr;
        for (int ch = ch_begin; ch < ch_end; ++ch) {
          const int c = ch * 8;
          float v[8];
          if (have) {
            tc::tmem_ld8(trow + c, v);
          } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = 0.f;
          }
          if (partial) {
#pragma unroll
            for (int j = 0; j < 8; ++j) wsl[(size_t)(c + j) * BM + mloc] = v[j];
          } else if (m < ep.Mv) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int n = n0 + c + j;
              if (n < ep.Nv) {
                bf16 hi, lo;
                split_bf16(v[j], hi, lo);
                ep.out_hi[(size_t)n * ep.ldo + m] = hi;
                ep.out_lo[(size_t)n * ep.ldo + m] = lo;
              }
            }
          }
        }
      } else {
        const ClenCoef kc = clen_coef(ep, si);
        for (int ch = ch_begin; ch < ch_end; ++ch) {
          const int c = ch * 8;
          float z[8];
          if (have) {
            tc::tmem_ld8(trow + c, z);
          } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) z[j] = 0.f;
          }
          float xv[8], b2v[8], vf[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            xv[j] = px[j];
            b2v[j] = pb[j];
            vf[j] = pv[j];
          }
          if (ch + 1 < ch_end) clenshaw_operands(ep, mv, m, n0 + c + 8, px, pb, pv);
          if (!mv) continue;
          const int nbase = n0 + c;
          const int nj = min(8, ep.Nv - nbase);
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            if (j >= nj) break;
            clen_store(ep, kc, m, nbase + j, clen_out(kc, xv[j], z[j], vf[j], b2v[j]));
          }
        }
      }
      tc::tc_fence_before();
      tc::mbar_arrive(tc::smem_u32(&acce_bar[buf]));
    }
  }

  tc::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem_base, TMEM_COLS);
  }
}

// ---------------------------------------------------------------------------
// GEMM2 with the Clenshaw operands staged by TMA (variant 7).  Fused hi/lo
// stages as variants 3 / 4, one CTA per SM; the CTA's 128 x BN tiles of
// b_{k+1}, b_{k+2} and v (FP32) are loaded into their own shared-memory
// region by three bulk tensor copies issued as soon as the previous kernel's
// results are visible, so they arrive while the MMAs run and the epilogue
// reads them from shared memory: no per-element global loads, no registers
// held for prefetch.  Epilogue arithmetic and stores as k_tc_gemm.
template <int BN, int STAGES>
__global__ void __launch_bounds__(NTHREADS, 1)
    k_tc_gemm_te(const __grid_constant__ CUtensorMap tA_hi, const __grid_constant__ CUtensorMap tA_lo,
                 const __grid_constant__ CUtensorMap tB_hi, const __grid_constant__ CUtensorMap tB_lo,
                 const __grid_constant__ CUtensorMap tX, const __grid_constant__ CUtensorMap tB2,
                 const __grid_constant__ CUtensorMap tV, GemmArgs ga, EpiParams ep, int *status) {
  constexpr uint32_t A_BYTES = BM * BK * 2;
  constexpr uint32_t B_BYTES = BN * BK * 2;
  constexpr uint32_t STAGE_BYTES = 2 * (A_BYTES + B_BYTES);
  constexpr uint32_t OPER_BYTES = BM * BN * 4;          // one FP32 operand tile
  constexpr uint32_t TMEM_COLS = (BN <= 32) ? 32 : (BN <= 64) ? 64 : 128;
  constexpr uint32_t IDESC = tc::idesc_bf16_f32(BM, BN);
  constexpr int NCH = BN / 16;
  constexpr int NCH0 = (NCH + 1) / 2;

  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  float *eop = reinterpret_cast<float *>(smem + STAGES * STAGE_BYTES);   // x | b2 | v tiles
  __shared__ __align__(8) uint64_t full_bar[STAGES];
  __shared__ __align__(8) uint64_t empty_bar[STAGES];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ __align__(8) uint64_t epi_bar;
  __shared__ uint32_t tmem_base_sh;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int nkb = ga.num_kb;
  const bool has_b2 = ep.b2 != nullptr, has_v = ep.v != nullptr;

  if (threadIdx.x == 0) {
    for (int st = 0; st < STAGES; ++st) {
      tc::mbar_init(tc::smem_u32(&full_bar[st]), 1);
      tc::mbar_init(tc::smem_u32(&empty_bar[st]), 1);
    }
    tc::mbar_init(tc::smem_u32(&done_bar), 1);
    tc::mbar_init(tc::smem_u32(&epi_bar), 1);
    tc::fence_barrier_init();
    tc::prefetch_tmap(&tA_hi);
    tc::prefetch_tmap(&tB_hi);
    tc::prefetch_tmap(&tX);
  }
  if (warp == 2) {
    tc::tmem_alloc(tc::smem_u32(&tmem_base_sh), TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem_d = tmem_base_sh;
  tc::pdl_wait();                 // operands / epilogue inputs come from the previous kernel
  tc::pdl_launch_dependents();

  if (warp == 0 && lane == 0) {
    // the Clenshaw operand tiles first (they are read last but have no
    // dependence on the MMAs), then the k-blocks of the product
    const uint32_t eb = tc::smem_u32(&epi_bar);
    tc::mbar_arrive_expect_tx(eb, OPER_BYTES * (1u + (has_b2 ? 1u : 0u) + (has_v ? 1u : 0u)));
    const uint64_t pol_once = tc::l2_evict_first(), pol_keep = tc::l2_evict_last();
    tc::tma_load_2d_hint(tc::smem_u32(eop), &tX, eb, m0, n0, pol_once);
    if (has_b2) tc::tma_load_2d_hint(tc::smem_u32(eop) + OPER_BYTES, &tB2, eb, m0, n0, pol_once);
    if (has_v) tc::tma_load_2d_hint(tc::smem_u32(eop) + 2 * OPER_BYTES, &tV, eb, m0, n0, pol_keep);
    for (int i = 0; i < nkb; ++i) {
      const int st = i % STAGES;
      if (i >= STAGES) {
        if (!tc::mbar_wait(tc::smem_u32(&empty_bar[st]), ((i / STAGES) - 1) & 1, status)) break;
      }
      const uint32_t bar = tc::smem_u32(&full_bar[st]);
      const uint32_t sa = tc::smem_u32(smem + st * STAGE_BYTES);
      tc::mbar_arrive_expect_tx(bar, STAGE_BYTES);
      tc::tma_load_2d(sa, &tA_hi, bar, i * BK, m0);
      tc::tma_load_2d(sa + A_BYTES, &tA_lo, bar, i * BK, m0);
      tc::tma_load_2d(sa + 2 * A_BYTES, &tB_hi, bar, i * BK, n0);
      tc::tma_load_2d(sa + 2 * A_BYTES + B_BYTES, &tB_lo, bar, i * BK, n0);
    }
  } else if (warp == 1 && lane == 0) {
    for (int i = 0; i < nkb; ++i) {
      const int st = i % STAGES;
      if (!tc::mbar_wait(tc::smem_u32(&full_bar[st]), (i / STAGES) & 1, status)) break;
      tc::tc_fence_after();
      const uint32_t sa = tc::smem_u32(smem + st * STAGE_BYTES);
      const uint32_t sal = sa + A_BYTES, sbh = sa + 2 * A_BYTES, sbl = sbh + B_BYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const uint32_t acc0 = (i > 0 || kk > 0) ? 1u : 0u;
        tc::mma_bf16(tmem_d, tc::smem_desc_sw128(sa + kk * 32), tc::smem_desc_sw128(sbh + kk * 32), IDESC, acc0);
        tc::mma_bf16(tmem_d, tc::smem_desc_sw128(sa + kk * 32), tc::smem_desc_sw128(sbl + kk * 32), IDESC, 1u);
        tc::mma_bf16(tmem_d, tc::smem_desc_sw128(sal + kk * 32), tc::smem_desc_sw128(sbh + kk * 32), IDESC, 1u);
      }
      tc::mma_commit(tc::smem_u32(&empty_bar[st]));
    }
    tc::mma_commit(tc::smem_u32(&done_bar));
  }
  __syncwarp();

  const int wl = warp & 3, wg = warp >> 2;
  const int mloc = wl * 32 + lane;
  const int m = m0 + mloc;
  const uint32_t trow = tmem_d + ((uint32_t)(wl * 32) << 16);
  const int ch_begin = wg == 0 ? 0 : NCH0;
  const int ch_end = wg == 0 ? NCH0 : NCH;
  const bool mv = m < ep.Mv;
  const ClenCoef kc = clen_coef(ep, mv ? ep.s[m] : 0.0);
  bool have = tc::mbar_wait(tc::smem_u32(&done_bar), 0, status) && nkb > 0;
  const bool have_ops = tc::mbar_wait(tc::smem_u32(&epi_bar), 0, status);
  tc::tc_fence_after();
  for (int ch = 2 * ch_begin; ch < 2 * ch_end; ++ch) {
    const int c = ch * 8;
    float z[8];
    if (have) {
      tc::tmem_ld8(trow + c, z);
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) z[j] = 0.f;
    }
    if (!mv || !have_ops) continue;
    const int nbase = n0 + c;
    const int nj = min(8, ep.Nv - nbase);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (j >= nj) break;
      const int e = (c + j) * BM + mloc;
      const float x = eop[e];
      const float b2 = has_b2 ? eop[BM * BN + e] : 0.f;
      const float v = has_v ? eop[2 * BM * BN + e] : 0.f;
      clen_store(ep, kc, m, nbase + j, clen_out(kc, x, z[j], v, b2));
    }
  }

  tc::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem_d, TMEM_COLS);
  }
}

// Deterministic split-K reduction: D(m, n) = sum_s partial_s(m, n) in split
// order, written as the split-BF16 pair.  One thread per output element,
// consecutive threads on consecutive rows (coalesced partial reads).
__global__ void k_splitk_reduce(const float *__restrict__ ws, int nsplit, int BN, int tiles_m,
                                int Mv, int Nv, bf16 *__restrict__ out_hi, bf16 *__restrict__ out_lo,
                                int ldo) {
  tc::pdl_wait();
  tc::pdl_launch_dependents();
  const size_t total = (size_t)Mv * Nv;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int n = (int)(idx / Mv), m = (int)(idx % Mv);
    const int tile = (n / BN) * tiles_m + m / BM;
    const float *p = ws + (size_t)tile * nsplit * (size_t)(BN * BM) + (size_t)(n % BN) * BM + (m % BM);
    float acc = 0.f;
    for (int s = 0; s < nsplit; ++s) acc += __ldcg(p + (size_t)s * (BN * BM));
    bf16 hi, lo;
    split_bf16(acc, hi, lo);
    out_hi[(size_t)n * ldo + m] = hi;
    out_lo[(size_t)n * ldo + m] = lo;
  }
}

// ---------------------------------------------------------------------------
// host side

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
static std::once_flag g_encode_once;

static int get_encode() {
  std::call_once(g_encode_once, []() {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  if (!g_encode) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return NGW_ERR_CUDA;
  }
  return NGW_OK;
}

// rows x cols (cols contiguous, multiple of 64) BF16 matrix, box 64 x box_rows
static int make_tmap(CUtensorMap *map, const void *ptr, int rows, int cols, int box_rows) {
  NGW_TRY(get_encode());
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d) rows=%d cols=%d box_rows=%d", (int)r, rows, cols,
              box_rows);
    return NGW_ERR_CUDA;
  }
  return NGW_OK;
}

// FP32 column-major matrix (rows contiguous, leading dimension rows) as 2-D
// tiles of 128 rows x box_cols columns, no swizzle: the tile lands in shared
// memory column after column, row r of column c at word c * 128 + r.
static int make_tmap_f32(CUtensorMap *map, const void *ptr, int rows, int cols, int box_cols) {
  NGW_TRY(get_encode());
  cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
  cuuint64_t strides[1] = {(cuuint64_t)rows * 4};
  cuuint32_t box[2] = {(cuuint32_t)BM, (cuuint32_t)box_cols};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(ptr), dims, strides,
                        box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled (FP32) failed (%d) rows=%d cols=%d box_cols=%d", (int)r, rows, cols,
              box_cols);
    return NGW_ERR_CUDA;
  }
  return NGW_OK;
}

// Launch with the programmatic-stream-serialisation attribute so the kernel's
// prologue overlaps the previous kernel's tail (disable with NGW_PDL=0).
static bool pdl_enabled() {
  static int en = -1;
  if (en < 0) {
    const char *e = getenv("NGW_PDL");
    en = (e && e[0] == '0') ? 0 : 1;
  }
  return en == 1;
}

template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

template <int BN, int STAGES, int MINB, bool FUSED = false>
static int launch_tc(const CUtensorMap &a_hi, const CUtensorMap &a_lo, const CUtensorMap &b_hi,
                     const CUtensorMap &b_lo, int tiles_m, int tiles_n, const GemmArgs &ga,
                     const EpiParams &ep, int *status, cudaStream_t st, const CUtensorMap *rm) {
  constexpr size_t smem = (size_t)STAGES * (BM * BK * 2 + BN * BK * 2) * (FUSED ? 2 : 1) + 1024;
  static std::atomic<unsigned long long> attr{0};
  NGW_CUDA(smem_limit_once(k_tc_gemm<BN, STAGES, MINB, FUSED>, (int)smem, attr));
  dim3 grid(tiles_m, tiles_n, ga.nsplit);
  // operand-ring maps (x, b2, v) of the Clenshaw epilogue; unused (ring = 0) otherwise
  const CUtensorMap &rx = rm ? rm[0] : a_hi, &rb2 = rm ? rm[1] : a_hi, &rv = rm ? rm[2] : a_hi;
  NGW_CUDA(launch_pdl(k_tc_gemm<BN, STAGES, MINB, FUSED>, grid, dim3(NTHREADS), smem, st, a_hi, a_lo,
                      b_hi, b_lo, rx, rb2, rv, ga, ep, status));
  return NGW_OK;
}

// Cluster-reduced split-K launch: the nsplit CTAs of a tile form one cluster.
template <int BN, int STAGES, int MINB>
static int launch_tc_cluster(const CUtensorMap &a_hi, const CUtensorMap &a_lo, const CUtensorMap &b_hi,
                             const CUtensorMap &b_lo, int tiles_m, int tiles_n, const GemmArgs &ga,
                             const EpiParams &ep, int *status, cudaStream_t st) {
  constexpr size_t smem = (size_t)STAGES * (BM * BK * 2 + BN * BK * 2) * 2 + 1024;
  static_assert((size_t)BN * BM * 4 <= smem - 1024, "partial tile must fit the stage buffers");
  static std::atomic<unsigned long long> attr{0};
  NGW_CUDA(smem_limit_once(k_tc_gemm<BN, STAGES, MINB, true, true>, (int)smem, attr));
  if (ga.nsplit < 2 || ga.nsplit > 8) {
    set_error("cluster split-K needs 2..8 splits (got %d)", ga.nsplit);
    return NGW_ERR_ARG;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(tiles_m, tiles_n, ga.nsplit);
  cfg.blockDim = dim3(NTHREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attrs[2];
  attrs[0].id = cudaLaunchAttributeClusterDimension;
  attrs[0].val.clusterDim.x = 1;
  attrs[0].val.clusterDim.y = 1;
  attrs[0].val.clusterDim.z = ga.nsplit;
  attrs[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attrs[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attrs;
  cfg.numAttrs = pdl_enabled() ? 2 : 1;
  NGW_CUDA(cudaLaunchKernelEx(&cfg, k_tc_gemm<BN, STAGES, MINB, true, true>, a_hi, a_lo, b_hi, b_lo, a_hi,
                              a_hi, a_hi, ga, ep, status));
  return NGW_OK;
}

template <int BN, int STAGES>
static int launch_tc_p(const CUtensorMap &a_hi, const CUtensorMap &a_lo, const CUtensorMap &b_hi,
                       const CUtensorMap &b_lo, int tiles_m, int tiles_n, const GemmArgs &ga,
                       const EpiParams &ep, int *status, cudaStream_t st) {
  constexpr size_t smem = (size_t)STAGES * (2 * BM * BK * 2 + 2 * BN * BK * 2) + 1024;
  static std::atomic<unsigned long long> attr{0};
  NGW_CUDA(smem_limit_once(k_tc_gemm_p<BN, STAGES>, (int)smem, attr));
  GemmArgs g2 = ga;
  g2.num_kb = ga.num_kb;   // fused segments: one k-block carries all three products
  const int nwork = tiles_m * tiles_n * ga.nsplit;
  const int grid = std::min(nwork, 148);
  NGW_CUDA(launch_pdl(k_tc_gemm_p<BN, STAGES>, dim3(grid), dim3(PTHREADS), smem, st, a_hi, a_lo, b_hi,
                      b_lo, g2, ep, tiles_m, tiles_n, status));
  return NGW_OK;
}

template <int BN, int STAGES>
static int launch_tc_te(const CUtensorMap &a_hi, const CUtensorMap &a_lo, const CUtensorMap &b_hi,
                        const CUtensorMap &b_lo, const CUtensorMap &tx, const CUtensorMap &tb2,
                        const CUtensorMap &tv, int tiles_m, int tiles_n, const GemmArgs &ga,
                        const EpiParams &ep, int *status, cudaStream_t st) {
  constexpr size_t smem = (size_t)STAGES * 2 * (BM * BK * 2 + BN * BK * 2) + (size_t)3 * BM * BN * 4 + 1024;
  static_assert(smem <= 232448 - 256, "variant 7 tile does not fit shared memory");
  static std::atomic<unsigned long long> attr{0};
  NGW_CUDA(smem_limit_once(k_tc_gemm_te<BN, STAGES>, (int)smem, attr));
  NGW_CUDA(launch_pdl(k_tc_gemm_te<BN, STAGES>, dim3(tiles_m, tiles_n, 1), dim3(NTHREADS), smem, st, a_hi,
                      a_lo, b_hi, b_lo, tx, tb2, tv, ga, ep, status));
  return NGW_OK;
}

// variant 7 (GEMM2 only): fused stages + Clenshaw operands staged by TMA
static bool has_te(int BN) { return BN == 32 || BN == 48 || BN == 64 || BN == 80; }

static int dispatch_te(int BN, const CUtensorMap &a_hi, const CUtensorMap &a_lo, const CUtensorMap &b_hi,
                       const CUtensorMap &b_lo, const CUtensorMap &tx, const CUtensorMap &tb2,
                       const CUtensorMap &tv, int tiles_m, int tiles_n, const GemmArgs &ga,
                       const EpiParams &ep, int *status, cudaStream_t st) {
  switch (BN) {
    case 32: return launch_tc_te<32, 4>(a_hi, a_lo, b_hi, b_lo, tx, tb2, tv, tiles_m, tiles_n, ga, ep, status, st);
    case 48: return launch_tc_te<48, 3>(a_hi, a_lo, b_hi, b_lo, tx, tb2, tv, tiles_m, tiles_n, ga, ep, status, st);
    case 64: return launch_tc_te<64, 2>(a_hi, a_lo, b_hi, b_lo, tx, tb2, tv, tiles_m, tiles_n, ga, ep, status, st);
    case 80: return launch_tc_te<80, 2>(a_hi, a_lo, b_hi, b_lo, tx, tb2, tv, tiles_m, tiles_n, ga, ep, status, st);
  }
  set_error("variant 7 has no N tile %d", BN);
  return NGW_ERR_ARG;
}

static bool has_persistent(int BN) { return BN <= 160; }
// variants 5 / 6: fused stages with the split-K sum inside a cluster, 1 / 2 CTAs per SM
static bool is_cluster_var(int var) { return var == 5 || var == 6; }
static bool has_fused(int BN) { return BN <= 128; }
static bool has_fused2(int BN) { return BN <= 64; }

// Supported N tiles (multiples of 16, <= 256).  Variant 0 ("deep"): one CTA
// per SM with a long TMA ring; variant 1 ("shallow", N <= 256; two stages
// above N = 160): 3-4 stages
// and <= 128 registers so two CTAs share an SM and one CTA's epilogue
// overlaps the other's main loop.
static const int kBNs[] = {32, 48, 64, 80, 96, 128, 144, 160, 192, 240, 256};

static bool has_shallow(int BN) { return BN <= 256; }

static int dispatch_tc(int BN, int var, const CUtensorMap &a_hi, const CUtensorMap &a_lo,
                       const CUtensorMap &b_hi, const CUtensorMap &b_lo, int tiles_m, int tiles_n,
                       const GemmArgs &ga, const EpiParams &ep, int *status, cudaStream_t st,
                       const CUtensorMap *rm = nullptr) {
#define NGW_TC(BNV, ST, MB) \
  return launch_tc<BNV, ST, MB>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st, rm)
#define NGW_TCP(BNV, ST) \
  return launch_tc_p<BNV, ST>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st)
  if (var == 2) {
    switch (BN) {
      case 32: NGW_TCP(32, 4);
      case 48: NGW_TCP(48, 4);
      case 64: NGW_TCP(64, 4);
      case 80: NGW_TCP(80, 4);
      case 96: NGW_TCP(96, 4);
      case 128: NGW_TCP(128, 3);
      case 144: NGW_TCP(144, 3);
      case 160: NGW_TCP(160, 3);
    }
  }
#undef NGW_TCP
#define NGW_TCF(BNV, ST, MB) \
  return launch_tc<BNV, ST, MB, true>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st, rm)
  if (var == 3) {
    switch (BN) {
      case 32: NGW_TCF(32, 5, 1);
      case 48: NGW_TCF(48, 4, 1);
      case 64: NGW_TCF(64, 4, 1);
      case 80: NGW_TCF(80, 4, 1);
      case 96: NGW_TCF(96, 3, 1);
      case 128: NGW_TCF(128, 3, 1);
    }
  }
  if (var == 4) {
    switch (BN) {
      case 32: NGW_TCF(32, 2, 2);
      case 48: NGW_TCF(48, 2, 2);
      case 64: NGW_TCF(64, 2, 2);
    }
  }
#undef NGW_TCF
#define NGW_TCC(BNV, ST, MB) \
  return launch_tc_cluster<BNV, ST, MB>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st)
  if (var == 5) {
    switch (BN) {
      case 32: NGW_TCC(32, 5, 1);
      case 48: NGW_TCC(48, 4, 1);
      case 64: NGW_TCC(64, 4, 1);
      case 80: NGW_TCC(80, 4, 1);
      case 96: NGW_TCC(96, 3, 1);
      case 128: NGW_TCC(128, 3, 1);
      // wide tiles for the dense p(C) GEMM (fewer re-reads of H and of the
      // chain vectors; the split-K inside the cluster keeps every SM busy)
      case 160: NGW_TCC(160, 3, 1);
      case 192: NGW_TCC(192, 2, 1);
      case 240: NGW_TCC(240, 2, 1);
      case 256: NGW_TCC(256, 2, 1);
    }
  }
  if (var == 6) {
    switch (BN) {
      case 32: NGW_TCC(32, 2, 2);
      case 48: NGW_TCC(48, 2, 2);
      case 64: NGW_TCC(64, 2, 2);
    }
  }
#undef NGW_TCC
  if (var == 0) {
    switch (BN) {
      case 32: NGW_TC(32, 8, 1);
      case 48: NGW_TC(48, 8, 1);
      case 64: NGW_TC(64, 8, 1);
      case 80: NGW_TC(80, 8, 1);
      case 96: NGW_TC(96, 7, 1);
      case 128: NGW_TC(128, 6, 1);
      case 144: NGW_TC(144, 6, 1);
      case 160: NGW_TC(160, 5, 1);
      case 192: NGW_TC(192, 5, 1);
      case 240: NGW_TC(240, 4, 1);
      case 256: NGW_TC(256, 4, 1);
    }
  } else {
    switch (BN) {
      case 32: NGW_TC(32, 4, 2);
      case 48: NGW_TC(48, 4, 2);
      case 64: NGW_TC(64, 4, 2);
      case 80: NGW_TC(80, 4, 2);
      case 96: NGW_TC(96, 3, 2);
      case 128: NGW_TC(128, 3, 2);
      case 144: NGW_TC(144, 3, 2);
      case 160: NGW_TC(160, 3, 2);
      // wide tiles (fewer re-reads of A) at two stages: 2 x 48 KB + TMEM 256 columns per CTA
      case 192: NGW_TC(192, 2, 2);
      case 240: NGW_TC(240, 2, 2);
      case 256: NGW_TC(256, 2, 2);
    }
  }
#undef NGW_TC
  set_error("unsupported N tile %d / variant %d", BN, var);
  return NGW_ERR_ARG;
}

// ---------------------------------------------------------------------------
// operand preparation kernels

// C (n_isdf, ncv) FP64 column-major (pair index slowest)  ->  A1[mu][cv] hi/lo
// (row length ldk = padded ncv).  Tile transpose through shared memory.
__global__ void k_split_transpose(const double *__restrict__ C, int n_isdf, int ncv,
                                  bf16 *__restrict__ hi, bf16 *__restrict__ lo, int ldk) {
  __shared__ double tile[32][33];
  const int cv0 = blockIdx.x * 32, mu0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int cv = cv0 + r, mu = mu0 + threadIdx.x;
    tile[r][threadIdx.x] = (cv < ncv && mu < n_isdf) ? C[(size_t)cv * n_isdf + mu] : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int mu = mu0 + r, cv = cv0 + threadIdx.x;
    if (mu < n_isdf && cv < ncv) {
      const double x = tile[threadIdx.x][r];
      const bf16 h = __double2bfloat16(x);
      const bf16 l = __double2bfloat16(x - (double)__bfloat162float(h));
      hi[(size_t)mu * ldk + cv] = h;
      lo[(size_t)mu * ldk + cv] = l;
    }
  }
}

// rows (ncv, ncol) FP64 column-major scaled per pair by 1/(f*s) -> out rows
// [row0 + j][cv] (A1 extension, row length ldk)
__global__ void k_split_cols_to_rows(const double *__restrict__ X, int ncv, int ncol,
                                     const double *__restrict__ s, double f, bf16 *__restrict__ hi,
                                     bf16 *__restrict__ lo, int ldk, int row0) {
  const int j = blockIdx.y;
  for (int cv = blockIdx.x * blockDim.x + threadIdx.x; cv < ncv; cv += gridDim.x * blockDim.x) {
    const double x = X[(size_t)j * ncv + cv] / (f * (s ? s[cv] : 1.0));
    const bf16 h = __double2bfloat16(x);
    const bf16 l = __double2bfloat16(x - (double)__bfloat162float(h));
    hi[(size_t)(row0 + j) * ldk + cv] = h;
    lo[(size_t)(row0 + j) * ldk + cv] = l;
  }
}

// D (n_isdf, ncv) FP64 column-major -> A3[cv][mu] hi/lo (row length ldk);
// extra columns mu = n_isdf + j hold -U(cv, j) / (4 s(cv))
__global__ void k_split_rows(const double *__restrict__ D, int n_isdf, int ncv,
                             const double *__restrict__ U, int k, const double *__restrict__ s,
                             bf16 *__restrict__ hi, bf16 *__restrict__ lo, int ldk) {
  for (int cv = blockIdx.y; cv < ncv; cv += gridDim.y)
    for (int mu = blockIdx.x * blockDim.x + threadIdx.x; mu < n_isdf + k; mu += gridDim.x * blockDim.x) {
      const double x = (mu < n_isdf) ? D[(size_t)cv * n_isdf + mu]
                                     : -U[(size_t)(mu - n_isdf) * ncv + cv] / (4.0 * s[cv]);
      const bf16 h = __double2bfloat16(x);
      const bf16 l = __double2bfloat16(x - (double)__bfloat162float(h));
      hi[(size_t)cv * ldk + mu] = h;
      lo[(size_t)cv * ldk + mu] = l;
    }
}

// Up(:, j) = U(:, j) * p(lambda_j) for the deflated Ritz vectors (ncv x k,
// column-major); the mixed plan deflates at most kMaxDeflation pairs (it
// asks the eigen-solver for 64).
constexpr int kMaxDeflation = 64;
struct DeflationValues {
  double v[kMaxDeflation];
};
__global__ void k_scale_cols(const double *__restrict__ U, int ncv, DeflationValues pv,
                             double *__restrict__ Up) {
  const int j = blockIdx.y;
  const double f = pv.v[j];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncv; i += gridDim.x * blockDim.x)
    Up[(size_t)j * ncv + i] = U[(size_t)j * ncv + i] * f;
}

// Clenshaw start: v_perp = v - U xo (deflated part, stored FP32), b_n = g v_perp
// (FP32) and split((R^1/2 or 1) * b_n) for the first GEMM1.
__global__ void k_cheb_start(const double *__restrict__ v, int ldv, const double *__restrict__ U,
                             const double *__restrict__ xo, int kdef, const double *__restrict__ s,
                             int ncv, int nb, double g, int tda, float *__restrict__ vp,
                             float *__restrict__ bn, int ldx, bf16 *__restrict__ shi,
                             bf16 *__restrict__ slo, int lds) {
  for (int j = blockIdx.y; j < nb; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncv; i += gridDim.x * blockDim.x) {
      double x = v[(size_t)j * ldv + i];
      for (int q = 0; q < kdef; ++q) x -= U[(size_t)q * ncv + i] * xo[(size_t)j * kdef + q];
      vp[(size_t)j * ldx + i] = (float)x;
      const double b = g * x;
      bn[(size_t)j * ldx + i] = (float)b;
      const double u = tda ? b : s[i] * b;
      bf16 h, l;
      split_bf16((float)u, h, l);
      shi[(size_t)j * lds + i] = h;
      slo[(size_t)j * lds + i] = l;
    }
}

struct MixedOperator {
  int n_isdf = 0, ncv = 0, kdef = 0, tda = 0;
  int mu_pad = 0;     // rows of A1 = n_isdf + kdef, padded to 128
  int mu_k = 0;       // K of GEMM2 = n_isdf + kdef, padded to 64
  int cv_pad = 0;     // K of GEMM1 / rows of A3 (multiple of 128)
  bf16 *A1_hi = nullptr, *A1_lo = nullptr, *A3_hi = nullptr, *A3_lo = nullptr;
  CUtensorMap tA1hi, tA1lo, tA3hi, tA3lo;
  size_t op_bytes = 0;
  double *Up = nullptr;      // (ncv, kdef) U p(Lambda) for the current polynomial
  // chain buffers
  int nb_cap = 0, nb_pad = 0;
  // tile choice (autotuned per chain count): N tile, kernel variant, split-K
  int BN1 = 128, var1 = 0, split1 = 1, BN2 = 128, var2 = 0, split2 = 1;
  int tuned_nb = -1, maps_bn1 = -1, maps_bn2 = -1;
  size_t ws_bytes = 0;
  bf16 *S_hi = nullptr, *S_lo = nullptr, *T_hi = nullptr, *T_lo = nullptr;
  CUtensorMap tShi, tSlo, tThi, tTlo;
  float *bb[3] = {nullptr, nullptr, nullptr};
  float *vperp = nullptr;
  CUtensorMap tBB[3], tVp;   // FP32 tiles of bb[i] / vperp for variant 7 (N tile maps_te_bn)
  int maps_te_bn = -1;
  CUtensorMap tR[4];         // 128 x 8 FP32 chunks of bb[0..2], vperp (the epilogue operand ring)
  bool maps_ring = false;
  double *xo = nullptr;
  float *ws = nullptr;
  size_t buf_bytes = 0;
  // dense form (small N_cv): H = P_perp p(Chat_perp) as one split-BF16 matrix
  // H[m][k] (rows cv_pad, row length kpad), built in FP64 for the polynomial
  // dense_g on [dense_c0 - dense_c1, dense_c0 + dense_c1]
  bf16 *H_hi = nullptr, *H_lo = nullptr;
  CUtensorMap tHhi, tHlo;
  int kpad = 0;
  bool dense_ok = false;
  bool dense_last = false;      // the session's last mixed plan used H
  std::vector<double> dense_g;
  double dense_c0 = 0.0, dense_c1 = 0.0;
  size_t dense_bytes = 0;
  // dense GEMM tiles (N tile, variant), tuned per chain count; S_hi / S_lo
  // as its B operand with that N tile
  int BNd = 128, vard = 3, splitd = 1, tuned_nbd = -1, maps_bnd = -1;
  // side stream of the dense step: xo = U^T v runs beside the split
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  CUtensorMap tVhi, tVlo;
};

static int round_up(int a, int b) { return (a + b - 1) / b * b; }

// A temporary device buffer of one call, returned to the pool (stream-ordered)
// when the scope ends, on error paths too.
struct PoolTmp {
  ngw_session *s;
  void *p = nullptr;
  explicit PoolTmp(ngw_session *s_) : s(s_) {}
  ~PoolTmp() { pool_free(s, p); }
};

static void free_chain_buffers(ngw_session *s, MixedOperator *op) {
  void *ptrs[] = {op->S_hi, op->S_lo, op->T_hi, op->T_lo, op->bb[0], op->bb[1], op->bb[2],
                  op->ws,   op->vperp, op->xo};
  for (void *p : ptrs)
    pool_free(s, p);
  op->S_hi = op->S_lo = op->T_hi = op->T_lo = nullptr;
  op->bb[0] = op->bb[1] = op->bb[2] = nullptr;
  op->ws = nullptr;
  op->vperp = nullptr;
  op->xo = nullptr;
  s->bytes -= op->buf_bytes;
  op->buf_bytes = 0;
  op->nb_cap = 0;
  op->maps_bn1 = op->maps_bn2 = -1;
  op->maps_te_bn = -1;
  op->maps_ring = false;
  op->tuned_nb = -1;
  op->maps_bnd = -1;
  op->tuned_nbd = -1;
}

static void free_dense(ngw_session *s, MixedOperator *op) {
  pool_free(s, op->H_hi);
  pool_free(s, op->H_lo);
  op->H_hi = op->H_lo = nullptr;
  s->bytes -= op->dense_bytes;
  op->dense_bytes = 0;
  op->dense_ok = false;
}

void mixed_free(ngw_session *s) {
  MixedOperator *op = s->mixed;
  if (!op) return;
  free_chain_buffers(s, op);
  free_dense(s, op);
  if (op->ev_fork) cudaEventDestroy(op->ev_fork);
  if (op->ev_join) cudaEventDestroy(op->ev_join);
  if (op->aux) cudaStreamDestroy(op->aux);
  void *ptrs[] = {op->A1_hi, op->A1_lo, op->A3_hi, op->A3_lo, op->Up};
  for (void *p : ptrs)
    pool_free(s, p);
  s->bytes -= op->op_bytes;
  delete op;
  s->mixed = nullptr;
}

int mixed_kdef(ngw_session *s) { return s->mixed ? s->mixed->kdef : -1; }

// current tile choice (part of the CUDA-graph key)
void extern_mixed_tune(ngw_session *s, int *tune) {
  MixedOperator *op = s->mixed;
  tune[0] = op->BN1 * 16 + op->var1;
  tune[1] = op->split1;
  tune[2] = (op->BN2 * 16 + op->var2) * 16 + op->split2;
  tune[3] = op->nb_cap;
  tune[4] = (op->BNd * 16 + op->vard) * 16 + op->splitd;
  tune[5] = op->dense_ok ? 1 : 0;
}

// Build A1 = [C_isdf ; G^T] (G = (C U) / R^1/2, k rows) and
// A3 = [(M C_isdf)^T | -U / (4 R^1/2)] in split-BF16 from the FP64 operator;
// U = the first kdef Ritz vectors in s->eig_U (kdef = 0: no deflation).
int mixed_build_operator(ngw_session *s, int kdef, int tda) {
  MixedOperator *op = s->mixed;
  // an operator of the same shapes is rebuilt in its own buffers (addresses
  // held by captured graphs stay valid); otherwise it is reallocated
  const bool reuse = op && op->n_isdf == s->n_isdf && op->ncv == s->ncv && op->kdef == kdef &&
                     op->tda == tda;
  const size_t a1 = (size_t)round_up(s->n_isdf + kdef, BM) * round_up(s->ncv, BM) * sizeof(bf16);
  const size_t a3 = (size_t)round_up(s->ncv, BM) * round_up(s->n_isdf + kdef, BK) * sizeof(bf16);
  s->mixed_dirty = false;
  if (!reuse) {
    bump_generation(s);
    mixed_free(s);
    op = new MixedOperator();
    s->mixed = op;
    op->n_isdf = s->n_isdf;
    op->ncv = s->ncv;
    op->kdef = kdef;
    op->tda = tda;
    op->mu_pad = round_up(s->n_isdf + kdef, BM);
    op->mu_k = round_up(s->n_isdf + kdef, BK);
    op->cv_pad = round_up(s->ncv, BM);
    NGW_CUDA(pool_alloc(s, (void **)&op->A1_hi, a1));
    NGW_CUDA(pool_alloc(s, (void **)&op->A1_lo, a1));
    NGW_CUDA(pool_alloc(s, (void **)&op->A3_hi, a3));
    NGW_CUDA(pool_alloc(s, (void **)&op->A3_lo, a3));
    op->op_bytes = 2 * (a1 + a3);
    if (kdef > 0) {
      NGW_CUDA(pool_alloc(s, (void **)&op->Up, (size_t)s->ncv * kdef * 8));
      op->op_bytes += (size_t)s->ncv * kdef * 8;
    }
    s->bytes += op->op_bytes;
  }
  op->dense_ok = false;   // H (if any) belongs to the previous operator values
  cudaStream_t st = s->stream;
  NGW_CUDA(cudaMemsetAsync(op->A1_hi, 0, a1, st));
  NGW_CUDA(cudaMemsetAsync(op->A1_lo, 0, a1, st));
  NGW_CUDA(cudaMemsetAsync(op->A3_hi, 0, a3, st));
  NGW_CUDA(cudaMemsetAsync(op->A3_lo, 0, a3, st));
  {
    dim3 grid((s->ncv + 31) / 32, (s->n_isdf + 31) / 32);
    k_split_transpose<<<grid, dim3(32, 8), 0, st>>>(s->d_C, s->n_isdf, s->ncv, op->A1_hi,
                                                    op->A1_lo, op->cv_pad);
    NGW_CUDA(cudaGetLastError());
  }
  const double one = 1.0, zero = 0.0;
  if (kdef > 0) {
    // G = (C U) / s  in FP64: C applied to the Ritz vectors as the matvec's
    // three products (C_isdf hs, M t1, C_isdf^T t2) on the FP64 tensor-core
    // GEMM, then the same combine (R^2 x + 4 R^1/2 z; TDA R x + 2 z)
    const int ni = s->n_isdf, nc = s->ncv;
    PoolTmp ths(s), tcu(s), tt1(s), tt2(s), tz(s), tws(s);
    const size_t wsb = std::min(dgemm_ws_bytes(std::max(ni, nc), kdef, 0), (size_t)64 << 20);
    NGW_CUDA(pool_alloc(s, &ths.p, (size_t)nc * kdef * 8));
    NGW_CUDA(pool_alloc(s, &tcu.p, (size_t)nc * kdef * 8));
    NGW_CUDA(pool_alloc(s, &tt1.p, (size_t)ni * kdef * 8));
    NGW_CUDA(pool_alloc(s, &tt2.p, (size_t)ni * kdef * 8));
    NGW_CUDA(pool_alloc(s, &tz.p, (size_t)nc * kdef * 8));
    NGW_CUDA(pool_alloc(s, &tws.p, wsb));
    double *hs = static_cast<double *>(ths.p), *CU = static_cast<double *>(tcu.p);
    double *t1 = static_cast<double *>(tt1.p), *t2 = static_cast<double *>(tt2.p);
    double *z = static_cast<double *>(tz.p), *ws = static_cast<double *>(tws.p);
    launch_scale_rows(s->d_sqrtR, s->eig_U, nc, hs, nc, nc, kdef, tda, st);
    NGW_CUDA(dgemm(st, false, false, ni, kdef, nc, one, s->d_C, ni, hs, nc, zero, t1, ni, ws, wsb));
    NGW_CUDA(dgemm(st, false, false, ni, kdef, ni, one, s->d_M, ni, t1, ni, zero, t2, ni, ws, wsb));
    NGW_CUDA(dgemm(st, true, false, nc, kdef, ni, one, s->d_C, ni, t2, ni, zero, z, nc, ws, wsb));
    launch_matvec_combine(s->d_sqrtR, hs, z, CU, nullptr, nc, kdef, tda, 0, 0.0, 0.0, nullptr, st);
    int bx = std::min(64, (nc + 255) / 256);
    // TDA: the pair scaling is 1 (A x uses x, not R^1/2 x)
    k_split_cols_to_rows<<<dim3(bx, kdef), 256, 0, st>>>(CU, nc, kdef, tda ? nullptr : s->d_sqrtR, 1.0,
                                                        op->A1_hi, op->A1_lo, op->cv_pad, ni);
    NGW_CUDA(cudaGetLastError());
    // the temporaries go back to the pool in stream order (PoolTmp), after
    // the kernels above on the session stream
  }
  // D = M * C (FP64 tensor-core GEMM), then split into A3[cv][mu] with the -U/(4s) columns
  PoolTmp td(s);
  NGW_CUDA(pool_alloc(s, &td.p, (size_t)s->n_isdf * s->ncv * sizeof(double)));
  double *D = static_cast<double *>(td.p);
  NGW_CUDA(dgemm(st, false, false, s->n_isdf, s->ncv, s->n_isdf, one, s->d_M, s->n_isdf, s->d_C, s->n_isdf,
                 zero, D, s->n_isdf));
  {
    int bx = (s->n_isdf + kdef + 127) / 128;
    k_split_rows<<<dim3(bx, ygrid(s->ncv)), 128, 0, st>>>(D, s->n_isdf, s->ncv, s->eig_U, kdef,
                                                   s->d_sqrtR, op->A3_hi, op->A3_lo, op->mu_k);
    NGW_CUDA(cudaGetLastError());
  }
  NGW_CUDA(cudaStreamSynchronize(st));
  NGW_TRY(make_tmap(&op->tA1hi, op->A1_hi, op->mu_pad, op->cv_pad, BM));
  NGW_TRY(make_tmap(&op->tA1lo, op->A1_lo, op->mu_pad, op->cv_pad, BM));
  NGW_TRY(make_tmap(&op->tA3hi, op->A3_hi, op->cv_pad, op->mu_k, BM));
  NGW_TRY(make_tmap(&op->tA3lo, op->A3_lo, op->cv_pad, op->mu_k, BM));
  return NGW_OK;
}

// Up = U diag(pvals) for the current polynomial (device, ncv x kdef)
int mixed_set_deflation_values(ngw_session *s, const double *pvals) {
  MixedOperator *op = s->mixed;
  if (!op || op->kdef == 0) return NGW_OK;
  if (op->kdef > kMaxDeflation) {
    set_error("deflation: more eigenpairs than the column scaling holds");
    return NGW_ERR_ARG;
  }
  DeflationValues pv;
  for (int j = 0; j < op->kdef; ++j) pv.v[j] = pvals[j];
  const int bx = std::min(64, (s->ncv + 255) / 256);
  k_scale_cols<<<dim3(bx, op->kdef), 256, 0, s->stream>>>(s->eig_U, s->ncv, pv, op->Up);
  NGW_CUDA(cudaGetLastError());
  return NGW_OK;
}

static int encode_chain_maps(MixedOperator *op, int bn1, int bn2) {
  if (op->maps_bn1 != bn1) {
    NGW_TRY(make_tmap(&op->tShi, op->S_hi, op->nb_pad, op->cv_pad, bn1));
    NGW_TRY(make_tmap(&op->tSlo, op->S_lo, op->nb_pad, op->cv_pad, bn1));
    op->maps_bn1 = bn1;
  }
  if (op->maps_bn2 != bn2) {
    NGW_TRY(make_tmap(&op->tThi, op->T_hi, op->nb_pad, op->mu_k, bn2));
    NGW_TRY(make_tmap(&op->tTlo, op->T_lo, op->nb_pad, op->mu_k, bn2));
    op->maps_bn2 = bn2;
  }
  return NGW_OK;
}

static int run_gemm1(ngw_session *s, int nb);
static int run_gemm2(ngw_session *s, int nb, const float *x, const float *b2, const float *v,
                     int ldv, double gamma, double alpha, double c0, double beta, int tda,
                     float *out32, double *out64, bool write_split, bool add_defl = false);

// Admissible tile choices (N tile, kernel variant, split-K) of GEMM1 (c1) and
// GEMM2 (c2) for the operator's shapes and nb chains: the tuner's candidates.
struct TileC {
  int bn, var, sp;
};
static void tune_candidates(const MixedOperator *op, int nb, std::vector<TileC> &c1, std::vector<TileC> &c2) {
  c1.clear();
  c2.clear();
  const int total_kb1 = 3 * (op->cv_pad / BK);
  const int tiles_m1 = op->mu_pad / BM;
  for (int bn : kBNs) {
    if (bn > round_up(nb, 16) && bn != kBNs[0]) continue;
    const int waste = round_up(nb, bn) - nb;
    if (waste * 8 > nb && bn != kBNs[0]) continue;     // at most 12.5% padding
    for (int var = 0; var < 7; ++var) {
      if (var == 1 && !has_shallow(bn)) continue;
      if (var == 2 && !has_persistent(bn)) continue;
      if ((var == 3 || var == 5) && !has_fused(bn)) continue;
      if ((var == 4 || var == 6) && !has_fused2(bn)) continue;
      if (!is_cluster_var(var)) {
        c2.push_back({bn, var, 1});
      } else {
        const int kb2 = op->mu_k / BK;   // GEMM2 k-blocks (fused stages)
        for (int sp : {2, 3, 4})
          if (kb2 / sp >= 2) c2.push_back({bn, var, sp});
      }
      const int tiles = tiles_m1 * ((nb + bn - 1) / bn);
      const int tkb = (var >= 2) ? total_kb1 / 3 : total_kb1;
      for (int sp : {1, 2, 3, 4, 6, 8, 12, 16}) {
        if (sp > 1 && tkb / sp < 3) break;
        if (is_cluster_var(var) && (sp < 2 || sp > 8)) continue;
        if (!is_cluster_var(var) && (size_t)tiles * sp * bn * BM * sizeof(float) > op->ws_bytes && sp > 1)
          break;
        if (tiles * sp > 4 * 148) break;
        c1.push_back({bn, var, sp});
      }
    }
  }
  // variant 7 (GEMM2 only): Clenshaw operands staged by TMA
  for (int bn : kBNs) {
    if (!has_te(bn)) continue;
    if (bn > round_up(nb, 16) && bn != kBNs[0]) continue;
    if ((round_up(nb, bn) - nb) * 8 > nb && bn != kBNs[0]) continue;
    c2.push_back({bn, 7, 1});
  }
}

// Autotuner (on a quiet device: other sessions' solves are held off).  Candidates: every admissible (N tile, variant, split-K) for
// GEMM1 and (N tile, variant) for GEMM2.  Each candidate is timed inside the
// alternating GEMM1 -> GEMM2 sequence a Clenshaw step runs (so L2 holds what
// it holds in the solve, and split-K partials compete with the next GEMM's
// operands as they do there), best of two trials.  GEMM1 is tuned with a
// fixed GEMM2, then GEMM2 with the chosen GEMM1.
static int autotune(ngw_session *s, int nb) {
  MixedOperator *op = s->mixed;
  // time on a quiet device: wait for the solves other sessions have in flight
  std::unique_lock<std::shared_mutex> quiet(gpu_quiet_lock(s->device));
  cudaEvent_t e0, e1;
  NGW_CUDA(cudaEventCreate(&e0));
  NGW_CUDA(cudaEventCreate(&e1));
  const bool verbose = getenv("NGW_TUNE_VERBOSE") != nullptr;
  auto g1 = [&]() { return run_gemm1(s, nb); };
  auto g2 = [&]() {
    return run_gemm2(s, nb, op->bb[0], op->bb[1], nullptr, 0, 0.0, 1.0, 0.0, 1.0, op->tda, op->bb[2],
                     nullptr, true);
  };
  auto timed = [&](int reps, float *ms) -> int {
    NGW_CUDA(cudaEventRecord(e0, s->stream));
    for (int r = 0; r < reps; ++r) {
      NGW_TRY(g1());
      NGW_TRY(g2());
    }
    NGW_CUDA(cudaEventRecord(e1, s->stream));
    NGW_CUDA(cudaEventSynchronize(e1));
    NGW_CUDA(cudaEventElapsedTime(ms, e0, e1));
    *ms /= reps;
    return NGW_OK;
  };
  auto time_pair = [&](float *ms) -> int {
    NGW_TRY(g1());
    NGW_TRY(g2());
    float one = 0;
    NGW_TRY(timed(1, &one));
    const int reps = one > 2.0f ? 1 : (one > 0.2f ? 3 : 8);
    const int trials = one > 2.0f ? 0 : 2;
    float best = one;
    for (int t = 0; t < trials; ++t) {
      float x = 0;
      NGW_TRY(timed(reps, &x));
      best = std::min(best, x);
    }
    *ms = best;
    return NGW_OK;
  };
  using C1 = TileC;
  using C2 = TileC;
  std::vector<C1> c1;
  std::vector<C2> c2;
  tune_candidates(op, nb, c1, c2);
  // GEMM2 fixed while GEMM1 is tuned: the 64-wide (or smallest) non-fused tile
  C2 fix2 = c2.front();
  for (const C2 &c : c2)
    if (c.var == 0 && c.bn == 64) fix2 = c;
  op->BN2 = fix2.bn;
  op->var2 = fix2.var;
  op->split2 = fix2.sp;
  // Two stages per GEMM: every candidate briefly (one warm pair and one timed
  // pair, the mean of three more below 0.5 ms), then time_pair for the
  // `refine` fastest (NGW_TUNE_REFINE, default 6; 0 = every candidate).
  static const int refine = [] {
    const char *e = getenv("NGW_TUNE_REFINE");
    return e ? atoi(e) : 6;
  }();
  auto time_quick = [&](float *ms) -> int {
    NGW_TRY(g1());
    NGW_TRY(g2());
    NGW_TRY(timed(1, ms));
    if (*ms < 0.5f) NGW_TRY(timed(3, ms));   // short pairs: the mean of three
    return NGW_OK;
  };
  auto pick = [&](int nc, auto set, const char *name) -> int {
    std::vector<std::pair<float, int>> quick;
    for (int i = 0; i < nc; ++i) {
      NGW_TRY(set(i));
      float ms = 0;
      NGW_TRY(time_quick(&ms));
      quick.push_back({ms, i});
    }
    std::stable_sort(quick.begin(), quick.end(),
                     [](const std::pair<float, int> &x, const std::pair<float, int> &y) { return x.first < y.first; });
    const int nref = (refine <= 0) ? nc : std::min(nc, refine);
    float best = 1e30f;
    int bi = quick.empty() ? 0 : quick[0].second;
    for (int r = 0; r < nref; ++r) {
      const int i = quick[r].second;
      NGW_TRY(set(i));
      float ms = 0;
      NGW_TRY(time_pair(&ms));
      if (verbose)
        fprintf(stderr, "tune %s candidate %d: %.2f us (first pass %.2f us)\n", name, i, 1e3f * ms,
                1e3f * quick[r].first);
      if (ms < best) {
        best = ms;
        bi = i;
      }
    }
    return bi;
  };
  auto set1 = [&](int i) -> int {
    op->BN1 = c1[i].bn;
    op->var1 = c1[i].var;
    op->split1 = c1[i].sp;
    return encode_chain_maps(op, c1[i].bn, op->BN2);
  };
  const int i1 = pick((int)c1.size(), set1, "gemm1");
  NGW_TRY(set1(i1));
  if (verbose)
    fprintf(stderr, "tune gemm1 chosen bn=%d var=%d split=%d\n", op->BN1, op->var1, op->split1);
  auto set2 = [&](int i) -> int {
    op->BN2 = c2[i].bn;
    op->var2 = c2[i].var;
    op->split2 = c2[i].sp;
    return encode_chain_maps(op, op->BN1, c2[i].bn);
  };
  const int i2 = pick((int)c2.size(), set2, "gemm2");
  const C2 b2 = c2[i2];
  if (verbose)
    fprintf(stderr, "tune gemm2 chosen bn=%d var=%d split=%d\n", b2.bn, b2.var, b2.sp);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  op->BN2 = b2.bn;
  op->var2 = b2.var;
  op->split2 = b2.sp;
  NGW_TRY(encode_chain_maps(op, op->BN1, op->BN2));
  // buffers used for timing held scratch values: clear the operands again
  NGW_CUDA(cudaMemsetAsync(op->T_hi, 0, (size_t)op->nb_pad * op->mu_k * sizeof(bf16), s->stream));
  NGW_CUDA(cudaMemsetAsync(op->T_lo, 0, (size_t)op->nb_pad * op->mu_k * sizeof(bf16), s->stream));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  op->tuned_nb = nb;
  return check_status(s);
}

// Process-wide cache of tile choices, keyed by the GEMM shapes: every session
// with the same shapes uses the same tiles (and therefore the same summation
// order), so a request gives bit-identical results alone or among others.
struct TuneKey {
  int mu_pad, cv_pad, mu_k, kdef, n_isdf, ncv, nb, tda;
  bool operator<(const TuneKey &o) const {
    return std::tie(mu_pad, cv_pad, mu_k, kdef, n_isdf, ncv, nb, tda) <
           std::tie(o.mu_pad, o.cv_pad, o.mu_k, o.kdef, o.n_isdf, o.ncv, o.nb, o.tda);
  }
};
struct TuneVal {
  int bn1, var1, split1, bn2, var2, split2;
};
static std::mutex g_tune_mu;
static std::map<TuneKey, TuneVal> g_tune;

// Chain buffers for nb chains and the tuned tile choice (bn1/bn2/split1 > 0
// force a choice instead of tuning).
int mixed_prepare_chains(ngw_session *s, int nb, int bn1, int bn2, int split1) {
  MixedOperator *op = s->mixed;
  if (!op) {
    set_error("mixed operator not built");
    return NGW_ERR_STATE;
  }
  if (op->nb_cap < nb) {
    bump_generation(s);
    free_chain_buffers(s, op);
    const int nbp = round_up(nb, 256);
    op->nb_pad = nbp;
    const size_t sbytes = (size_t)nbp * op->cv_pad * sizeof(bf16);
    const size_t tbytes = (size_t)nbp * op->mu_k * sizeof(bf16);
    const size_t bbytes = (size_t)nbp * op->cv_pad * sizeof(float);
    const size_t vbytes = (size_t)nbp * op->cv_pad * sizeof(float);
    const size_t xbytes = (size_t)nbp * std::max(op->kdef, 1) * sizeof(double);
    // split-K partials: enough for 16 splits of the smallest tile grid
    const size_t wsbytes = (size_t)(op->mu_pad / BM) * ((nbp + 63) / 64) * 16 * 64 * BM * sizeof(float);
    NGW_CUDA(pool_alloc(s, (void **)&op->S_hi, sbytes));
    NGW_CUDA(pool_alloc(s, (void **)&op->S_lo, sbytes));
    NGW_CUDA(pool_alloc(s, (void **)&op->T_hi, tbytes));
    NGW_CUDA(pool_alloc(s, (void **)&op->T_lo, tbytes));
    for (int i = 0; i < 3; ++i) NGW_CUDA(pool_alloc(s, (void **)&op->bb[i], bbytes));
    NGW_CUDA(pool_alloc(s, (void **)&op->vperp, vbytes));
    NGW_CUDA(pool_alloc(s, (void **)&op->xo, xbytes));
    NGW_CUDA(pool_alloc(s, (void **)&op->ws, wsbytes));
    op->ws_bytes = wsbytes;
    op->buf_bytes = 2 * sbytes + 2 * tbytes + 3 * bbytes + vbytes + xbytes + wsbytes;
    s->bytes += op->buf_bytes;
    NGW_CUDA(cudaMemsetAsync(op->S_hi, 0, sbytes, s->stream));
    NGW_CUDA(cudaMemsetAsync(op->S_lo, 0, sbytes, s->stream));
    NGW_CUDA(cudaMemsetAsync(op->T_hi, 0, tbytes, s->stream));
    NGW_CUDA(cudaMemsetAsync(op->T_lo, 0, tbytes, s->stream));
    for (int i = 0; i < 3; ++i) NGW_CUDA(cudaMemsetAsync(op->bb[i], 0, bbytes, s->stream));
    op->nb_cap = nbp;
    op->maps_bn1 = op->maps_bn2 = -1;
    op->tuned_nb = -1;
  }
  if (bn1 > 0 && bn2 > 0) {
    op->BN1 = bn1;
    op->BN2 = bn2;
    op->var1 = op->var2 = 0;
    op->split1 = split1 > 0 ? split1 : 1;
    op->split2 = 1;
    op->tuned_nb = -2;
    return encode_chain_maps(op, bn1, bn2);
  }
  // NGW_TILES="bn1,var1,split1,bn2,var2[,split2]" fixes the tiles (reproducible profiling)
  if (const char *env = getenv("NGW_TILES")) {
    int t[6] = {0, 0, 0, 0, 0, 1};
    if (sscanf(env, "%d,%d,%d,%d,%d,%d", &t[0], &t[1], &t[2], &t[3], &t[4], &t[5]) >= 5) {
      op->BN1 = t[0];
      op->var1 = t[1];
      op->split1 = t[2];
      op->BN2 = t[3];
      op->var2 = t[4];
      op->split2 = t[5] > 0 ? t[5] : 1;
      op->tuned_nb = nb;
      return encode_chain_maps(op, t[0], t[3]);
    }
  }
  if (op->tuned_nb != nb) {
    const TuneKey key{op->mu_pad, op->cv_pad, op->mu_k, op->kdef, op->n_isdf, op->ncv, nb, op->tda};
    // The cache lookup and the nearest-shape reuse run under g_tune_mu; the
    // tuning itself (device-exclusive, 0.3-1.5 s) runs without it, so other
    // sessions' lookups do not wait behind one device's tuning.  Two sessions
    // that miss on the same shape at once both tune it; the last result stays.
    std::unique_lock<std::mutex> lk(g_tune_mu);
    auto use = [&](const TuneVal &v) {
      op->BN1 = v.bn1;
      op->var1 = v.var1;
      op->split1 = v.split1;
      op->BN2 = v.bn2;
      op->var2 = v.var2;
      op->split2 = v.split2;
      op->tuned_nb = nb;
      return encode_chain_maps(op, op->BN1, op->BN2);
    };
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return use(it->second);
    // A request stream brings new shapes with almost every molecule: reuse
    // the choice of the nearest tuned shape (same padded N_mu and K of GEMM2,
    // deflation and TDA classes, N_cv and chain count within 25 %) when it is
    // admissible here, instead of tuning again.  NGW_TUNE_EXACT=1 tunes every
    // new shape.
    static const bool exact = [] {
      const char *e = getenv("NGW_TUNE_EXACT");
      return e && e[0] == '1';
    }();
    if (!exact) {
      const TuneVal *best = nullptr;
      double best_d = 1e30;
      for (const auto &kv : g_tune) {
        const TuneKey &k = kv.first;
        if (k.mu_pad != key.mu_pad || k.mu_k != key.mu_k || (k.kdef > 0) != (key.kdef > 0) || k.tda != key.tda)
          continue;
        const double rc = std::log((double)k.cv_pad / key.cv_pad), rn = std::log((double)k.nb / key.nb);
        if (std::fabs(rc) > std::log(1.25) || std::fabs(rn) > std::log(1.25)) continue;
        const double d = std::fabs(rc) + std::fabs(rn);
        if (d < best_d) {
          best_d = d;
          best = &kv.second;
        }
      }
      if (best) {
        std::vector<TileC> c1, c2;
        tune_candidates(op, nb, c1, c2);
        const TuneVal v = *best;
        const bool ok1 = std::any_of(c1.begin(), c1.end(), [&](const TileC &c) {
          return c.bn == v.bn1 && c.var == v.var1 && c.sp == v.split1;
        });
        const bool ok2 = std::any_of(c2.begin(), c2.end(), [&](const TileC &c) {
          return c.bn == v.bn2 && c.var == v.var2 && c.sp == v.split2;
        });
        if (ok1 && ok2) {
          g_tune[key] = v;
          return use(v);
        }
      }
    }
    lk.unlock();
    NGW_TRY(autotune(s, nb));
    lk.lock();
    g_tune[key] = TuneVal{op->BN1, op->var1, op->split1, op->BN2, op->var2, op->split2};
  }
  return NGW_OK;
}

// One GEMM1 ([T; q] = A1 S) with split output into T_hi/T_lo.
static int run_gemm1(ngw_session *s, int nb) {
  MixedOperator *op = s->mixed;
  GemmArgs ga;
  ga.num_kb = op->cv_pad / BK;
  ga.nseg = 3;
  ga.nsplit = op->split1;
  EpiParams ep;
  std::memset(&ep, 0, sizeof(ep));
  ep.kind = EPI_SPLIT;
  ep.Mv = op->n_isdf + op->kdef;
  ep.Nv = nb;
  ep.out_hi = op->T_hi;
  ep.out_lo = op->T_lo;
  ep.ldo = op->mu_k;
  ep.ws = op->ws;
  const int tiles_m = op->mu_pad / BM;
  const int tiles_n = (nb + op->BN1 - 1) / op->BN1;
  NGW_TRY(dispatch_tc(op->BN1, op->var1, op->tA1hi, op->tA1lo, op->tShi, op->tSlo, tiles_m, tiles_n,
                      ga, ep, s->d_status, s->stream));
  if (op->split1 > 1 && !is_cluster_var(op->var1)) {
    const size_t total = (size_t)ep.Mv * nb;
    int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 8);
    NGW_CUDA(launch_pdl(k_splitk_reduce, dim3(blocks), dim3(256), 0, s->stream, (const float *)op->ws,
                        op->split1, op->BN1, tiles_m, ep.Mv, nb, op->T_hi, op->T_lo, op->mu_k));
  }
  return NGW_OK;
}

// One GEMM2 with the Clenshaw epilogue.
static int run_gemm2(ngw_session *s, int nb, const float *x, const float *b2, const float *v,
                     int ldv, double gamma, double alpha, double c0, double beta, int tda,
                     float *out32, double *out64, bool write_split, bool add_defl) {
  MixedOperator *op = s->mixed;
  GemmArgs ga;
  ga.num_kb = op->mu_k / BK;
  ga.nseg = 3;
  ga.nsplit = is_cluster_var(op->var2) ? op->split2 : 1;
  EpiParams ep;
  std::memset(&ep, 0, sizeof(ep));
  ep.kind = EPI_CLENSHAW;
  ep.Mv = op->ncv;
  ep.Nv = nb;
  ep.s = s->d_sqrtR;
  ep.x = x;
  ep.b2 = b2;
  ep.v = v;
  ep.ldx = op->cv_pad;
  ep.ldv = ldv;
  ep.gamma = gamma;
  ep.alpha = alpha;
  ep.c0 = c0;
  ep.beta = beta;
  ep.tda = tda;
  ep.out32 = out32;
  ep.out64 = out64;
  ep.s_hi = write_split ? op->S_hi : nullptr;
  ep.s_lo = write_split ? op->S_lo : nullptr;
  ep.lds = op->cv_pad;
  if (add_defl && op->kdef > 0) {
    ep.Up = op->Up;
    ep.xo = op->xo;
    ep.kdef = op->kdef;
  }
  const int tiles_m = op->cv_pad / BM;
  const int tiles_n = (nb + op->BN2 - 1) / op->BN2;
  if (op->var2 == 7) {
    // operands are chain buffers: FP32 tensor maps of each, built per N tile
    if (op->maps_te_bn != op->BN2) {
      for (int i = 0; i < 3; ++i) NGW_TRY(make_tmap_f32(&op->tBB[i], op->bb[i], op->cv_pad, op->nb_pad, op->BN2));
      NGW_TRY(make_tmap_f32(&op->tVp, op->vperp, op->cv_pad, op->nb_pad, op->BN2));
      op->maps_te_bn = op->BN2;
    }
    auto pick = [&](const float *p) -> const CUtensorMap * {
      for (int i = 0; i < 3; ++i)
        if (p == op->bb[i]) return &op->tBB[i];
      return p == op->vperp ? &op->tVp : nullptr;
    };
    const CUtensorMap *mx = pick(x), *mb2 = b2 ? pick(b2) : &op->tBB[0], *mvv = v ? pick(v) : &op->tBB[0];
    if (!mx || !mb2 || !mvv) {
      set_error("GEMM2 variant 7: Clenshaw operand outside the chain buffers");
      return NGW_ERR_ARG;
    }
    ga.nsplit = 1;
    return dispatch_te(op->BN2, op->tA3hi, op->tA3lo, op->tThi, op->tTlo, *mx, *mb2, *mvv, tiles_m, tiles_n,
                       ga, ep, s->d_status, s->stream);
  }
  // variants 0, 1, 3, 4: Clenshaw operands through the TMA chunk ring
  static const bool ring_on = [] {
    const char *e = getenv("NGW_RING");
    return !(e && e[0] == '0');
  }();
  if (ring_on && (op->var2 == 0 || op->var2 == 1 || op->var2 == 3 || op->var2 == 4)) {
    if (!op->maps_ring) {
      for (int i = 0; i < 3; ++i) NGW_TRY(make_tmap_f32(&op->tR[i], op->bb[i], op->cv_pad, op->nb_pad, 8));
      NGW_TRY(make_tmap_f32(&op->tR[3], op->vperp, op->cv_pad, op->nb_pad, 8));
      op->maps_ring = true;
    }
    auto slot = [&](const float *p) -> int {
      for (int i = 0; i < 3; ++i)
        if (p == op->bb[i]) return i;
      return p == op->vperp ? 3 : -1;
    };
    const int ix = slot(x), ib2 = b2 ? slot(b2) : 0, iv = v ? slot(v) : 0;
    if (ix < 0 || ib2 < 0 || iv < 0) {
      set_error("GEMM2: Clenshaw operand outside the chain buffers");
      return NGW_ERR_ARG;
    }
    const CUtensorMap rm[3] = {op->tR[ix], op->tR[ib2], op->tR[iv]};
    ep.ring = 1;
    return dispatch_tc(op->BN2, op->var2, op->tA3hi, op->tA3lo, op->tThi, op->tTlo, tiles_m, tiles_n,
                       ga, ep, s->d_status, s->stream, rm);
  }
  return dispatch_tc(op->BN2, op->var2, op->tA3hi, op->tA3lo, op->tThi, op->tTlo, tiles_m, tiles_n,
                     ga, ep, s->d_status, s->stream);
}

// Clenshaw start of p(C) v on stream st: xo = U^T v (deflated eigenpairs),
// v_perp = v - U xo, b_n = g_n v_perp and the split operand of the first GEMM1.
static int mixed_poly_start(ngw_session *s, int nb, const double *v, int ldv, double gn, int tda,
                            cudaStream_t st) {
  MixedOperator *op = s->mixed;
  const int ncv = s->ncv, k = op->kdef;
  if (k > 0)   // xo = U^T v (FP64); v_perp and the U p(Lambda) xo term are fused below
    NGW_CUDA(dgemm(st, true, false, k, nb, ncv, 1.0, s->eig_U, ncv, v, ldv, 0.0, op->xo, k,
                   reinterpret_cast<double *>(op->ws), op->ws_bytes));
  int bx = (ncv + 255) / 256;
  if (bx > 16) bx = 16;
  k_cheb_start<<<dim3(bx, ygrid(nb)), 256, 0, st>>>(v, ldv, s->eig_U, op->xo, k, s->d_sqrtR, ncv, nb, gn, tda,
                                                    op->vperp, op->bb[0], op->cv_pad, op->S_hi, op->S_lo,
                                                    op->cv_pad);
  NGW_CUDA(cudaGetLastError());
  return NGW_OK;
}

// out64 (ncv x nb, ld ldv) = p(C) v with p given by Chebyshev coefficients
// g[0..n] on [c0 - c1, c0 + c1] for the deflated part and U p(Lambda) U^T v
// for the deflated eigenpairs.  Launch-only (no host synchronisation).
int mixed_poly_apply(ngw_session *s, int nb, const double *v, int ldv, const double *g, int n,
                     double c0, double c1, int tda, double *out64) {
  MixedOperator *op = s->mixed;
  if (!op || op->nb_cap < nb) {
    set_error("mixed chain buffers not prepared");
    return NGW_ERR_STATE;
  }
  if (n < 1) {
    set_error("polynomial degree must be >= 1");
    return NGW_ERR_ARG;
  }
  NGW_TRY(mixed_poly_start(s, nb, v, ldv, g[n], tda, s->stream));
  const float *vin = op->vperp;
  int cur = 0, prev = -1;   // slots of b_{k+1}, b_{k+2}
  for (int kk = n - 1; kk >= 1; --kk) {
    NGW_TRY(run_gemm1(s, nb));
    // b_k goes to the slot that is neither b_{k+1} nor b_{k+2}
    const int outb = (prev < 0) ? 1 : 3 - cur - prev;
    NGW_TRY(run_gemm2(s, nb, op->bb[cur], prev < 0 ? nullptr : op->bb[prev], vin, ldv, g[kk],
                      2.0 / c1, c0, 1.0, tda, op->bb[outb], nullptr, true));
    prev = cur;
    cur = outb;
  }
  NGW_TRY(run_gemm1(s, nb));
  // final step: p(C) v = g_0 v_perp + Chat b_1 - b_2 + U p(Lambda) xo
  NGW_TRY(run_gemm2(s, nb, op->bb[cur], prev < 0 ? nullptr : op->bb[prev], vin, ldv, g[0],
                    1.0 / c1, c0, 1.0, tda, nullptr, out64, false, true));
  return NGW_OK;
}

// ---------------------------------------------------------------------------
// Dense form of p(C) for small N_cv.  When N_cv is small against the ISDF
// rank the operator itself is cheaper to apply than its factors:
//   H = P_perp p(Chat_perp),  Chat_perp = (P_perp C P_perp - c0) / c1,
// P_perp = I - U U^T (the deflated Ritz vectors), is formed once per operator
// and polynomial in FP64 (C = R^2 + 4 R^1/2 (C_isdf^T M C_isdf) R^1/2, the
// deflation as rank-k updates, then the Chebyshev series of the vector form
// in Paterson-Stockmeyer form: T_0..T_m of X = Chat P by the three-term
// recurrence and a Horner scheme in T_m over the series' base-T_m digits,
// about 2 sqrt(n) FP64 tensor-core GEMMs for degree n), split into
// BF16 hi/lo rows, and every p(C) v of the Lanczos recurrence is then ONE
// tcgen05 GEMM H v (split-BF16, FP32 accumulation) whose epilogue adds the
// deflated eigenpairs' U p(Lambda) U^T v in FP64 -- the same quantity the
// Clenshaw recurrence on vectors delivers, with 2 N_cv^2 instead of
// 4 p (N_mu + k) N_cv multiply-adds per chain.

// C(i, j) = 4 s_i K(i, j) s_j + delta_ij s_i^4   (s = R^1/2), in place
__global__ void k_dense_casida(double *__restrict__ K, const double *__restrict__ s, int n) {
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    double v = 4.0 * s[i] * K[e] * s[j];
    if (i == j) v += s[i] * s[i] * s[i] * s[i];
    K[e] = v;
  }
}

__global__ void k_dense_identity(double *__restrict__ A, int n) {
  const size_t total = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x)
    A[e] = ((int)(e % n) == (int)(e / n)) ? 1.0 : 0.0;
}

// out = sum_r c_r T_r (up to 16 terms), elementwise
struct MatCombo {
  const double *t[16];
  double c[16];
  int n;
};
__global__ void k_dense_combo(MatCombo mc, size_t total, double *__restrict__ out) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int r = 0; r < mc.n; ++r) acc = fma(mc.c[r], mc.t[r][e], acc);
    out[e] = acc;
  }
}

// X = (C_perp - c0 P) / c1 = Chat P (C_perp P = C_perp)
__global__ void k_dense_x(const double *__restrict__ Cp, const double *__restrict__ P, double c0, double f,
                          size_t total, double *__restrict__ X) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x)
    X[e] = (Cp[e] - c0 * P[e]) * f;
}

// xo(:, j) = U^T v_j in FP64 on the FP64 tensor cores: a CTA takes eight
// chains, each of its DP_W warps a K slice of ncv and runs mma.sync m8n8k4
// f64 over it per eight eigenpairs (A = U^T: q x k, B = v: k x chain; lane
// (g, t) = (lane / 4, lane % 4) holds A[g][t], B[t][g] and C[g][2t],
// C[g][2t+1]); the warps' 8 x 8 tiles are summed in warp order
// (deterministic).  U is read once per eight chains.
constexpr int DP_W = 32;
__device__ __forceinline__ void dmma_f64(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}
__global__ void __launch_bounds__(DP_W * 32) k_dense_xo(const double *__restrict__ V, int ldv, int ncv, int nb,
                                                       const double *__restrict__ U, int k,
                                                       double *__restrict__ xo) {
  __shared__ double red[DP_W][64];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, grp = lane >> 2, tig = lane & 3;
  const int j0 = blockIdx.x * 8;
  const int nj = min(8, nb - j0);
  const int kc = (((ncv + DP_W - 1) / DP_W) + 3) & ~3;
  const int kb = w * kc, ke = min(ncv, kb + kc);
  const bool jv = grp < nj;
  const double *vj = V + (size_t)(j0 + (jv ? grp : 0)) * ldv;
  for (int q0 = 0; q0 < k; q0 += 8) {
    const bool qv = q0 + grp < k;
    const double *uq = U + (size_t)(qv ? q0 + grp : 0) * ncv;
    double c0 = 0.0, c1 = 0.0;
    for (int kbase = kb; kbase < ke; kbase += 32) {
      double bv[8], av[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int kx = kbase + 4 * u + tig;
        const bool in = kx < ke;
        bv[u] = (jv && in) ? vj[kx] : 0.0;
        av[u] = (qv && in) ? uq[kx] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) dmma_f64(c0, c1, av[u], bv[u]);
    }
    red[w][grp * 8 + 2 * tig] = c0;
    red[w][grp * 8 + 2 * tig + 1] = c1;
    __syncthreads();
    if (tid < 64) {
      const int q = tid >> 3, n = tid & 7;
      double sum = 0.0;
      for (int ww = 0; ww < DP_W; ++ww) sum += red[ww][tid];
      if (q0 + q < k && n < nj) xo[(size_t)(j0 + n) * k + q0 + q] = sum;
    }
    __syncthreads();
  }
}

// the split-BF16 rows [j][cv] of the chain vectors: four consecutive
// elements per thread (hi through FP32, lo the FP64 remainder)
__global__ void k_split_chains(const double *__restrict__ V, int ldv, int ncv, int nb, bf16 *__restrict__ hi,
                               bf16 *__restrict__ lo, int lds) {
  const int j = blockIdx.y;
  const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (j >= nb || i0 >= ncv) return;
  double x[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) x[u] = i0 + u < ncv ? V[(size_t)j * ldv + i0 + u] : 0.0;
#pragma unroll
  for (int u = 0; u < 4; ++u)
    if (i0 + u < ncv) {
      const bf16 h = __float2bfloat16_rn((float)x[u]);
      hi[(size_t)j * lds + i0 + u] = h;
      lo[(size_t)j * lds + i0 + u] = __float2bfloat16_rn((float)(x[u] - (double)__bfloat162float(h)));
    }
}

static unsigned elem_blocks(size_t total) {
  return (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
}

void mixed_dense_mark(ngw_session *s, bool used) {
  if (s->mixed) s->mixed->dense_last = used;
}

bool mixed_dense_ready(ngw_session *s, const double *g, int n, double c0, double c1) {
  const MixedOperator *op = s->mixed;
  if (!op || !op->dense_ok || op->dense_c0 != c0 || op->dense_c1 != c1 || (int)op->dense_g.size() != n + 1)
    return false;
  for (int i = 0; i <= n; ++i)
    if (op->dense_g[i] != g[i]) return false;
  return true;
}

// Paterson-Stockmeyer digits of a Chebyshev series g[0..n] in base T_m:
// p = d_0 + T_m (d_1 + T_m (... + T_m d_Q)), deg d_q < m, by repeated
// division by T_m with T_i = 2 T_m T_{i-m} - T_{|2m-i|} (long double).
static std::vector<std::vector<double>> cheb_digits(const double *g, int n, int m) {
  std::vector<long double> cur(g, g + n + 1);
  std::vector<std::vector<double>> d;
  while ((int)cur.size() - 1 >= m) {
    std::vector<long double> a = cur;
    const int deg = (int)a.size() - 1;
    std::vector<long double> q(deg - m + 1, 0.0L);
    for (int i = deg; i >= m; --i) {
      const long double c = a[i];
      if (c == 0.0L) continue;
      a[i] = 0.0L;
      if (i == m) {
        q[0] += c;
      } else {
        q[i - m] += 2.0L * c;
        a[std::abs(2 * m - i)] -= c;
      }
    }
    d.emplace_back(a.begin(), a.begin() + m);
    cur = q;
  }
  d.emplace_back(cur.begin(), cur.end());
  return d;
}

int mixed_dense_build(ngw_session *s, const double *g, int n, double c0, double c1) {
  MixedOperator *op = s->mixed;
  if (!op || op->tda || n < 1 || c1 == 0.0) {
    set_error("dense p(C): needs the mixed operator (not TDA) and a polynomial of degree >= 1");
    return NGW_ERR_STATE;
  }
  if (mixed_dense_ready(s, g, n, c0, c1)) return NGW_OK;
  if (!op->aux) {
    NGW_CUDA(cudaStreamCreateWithFlags(&op->aux, cudaStreamNonBlocking));
    NGW_CUDA(cudaEventCreateWithFlags(&op->ev_fork, cudaEventDisableTiming));
    NGW_CUDA(cudaEventCreateWithFlags(&op->ev_join, cudaEventDisableTiming));
  }
  const int N = s->ncv, ni = s->n_isdf, k = op->kdef;
  const int kpad = round_up(N, BK);
  const size_t hbytes = (size_t)op->cv_pad * kpad * sizeof(bf16);
  if (!op->H_hi || op->kpad != kpad) {
    bump_generation(s);
    free_dense(s, op);
    NGW_CUDA(pool_alloc(s, (void **)&op->H_hi, hbytes));
    NGW_CUDA(pool_alloc(s, (void **)&op->H_lo, hbytes));
    op->kpad = kpad;
    op->dense_bytes = 2 * hbytes;
    s->bytes += op->dense_bytes;
  }
  op->dense_ok = false;
  cudaStream_t st = s->stream;
  const size_t nn = (size_t)N * N;
  // Paterson-Stockmeyer in the Chebyshev basis: T_r P (r <= m) of X = Chat P
  // by the three-term recurrence, then the Horner form in T_m over the
  // digits -- (m - 1) + Q FP64 GEMMs instead of the n of the Clenshaw form
  const int m = std::max(2, (int)std::ceil(std::sqrt((double)n + 1.0)));
  const std::vector<std::vector<double>> dig = cheb_digits(g, n, m);
  const int Q = (int)dig.size() - 1;
  const int rmax = Q > 0 ? m : n;          // highest T_r needed
  if (m > 16) {
    set_error("dense p(C): polynomial degree %d too high for the dense form", n);
    return NGW_ERR_ARG;
  }
  std::deque<PoolTmp> tm;   // element addresses stay fixed as it grows
  auto mat = [&](size_t elems) -> double * {
    tm.emplace_back(s);
    if (pool_alloc(s, &tm.back().p, elems * 8) != cudaSuccess) return nullptr;
    return static_cast<double *>(tm.back().p);
  };
  double *Cm = mat(nn), *D = mat((size_t)ni * N);
  std::vector<double *> T(rmax + 1, nullptr);
  for (int r = 0; r <= rmax; ++r) T[r] = mat(nn);
  double *Y0 = mat(nn), *Y1 = mat(nn);
  if (!Cm || !D || !Y0 || !Y1 || std::find(T.begin(), T.end(), nullptr) != T.end()) {
    set_error("dense p(C): out of device memory for the FP64 formation (N_cv %d)", N);
    return NGW_ERR_OOM;
  }
  double *P = T[0];
  // C = R^2 + 4 R^1/2 (C_isdf^T (M C_isdf)) R^1/2
  NGW_CUDA(dgemm(st, false, false, ni, N, ni, 1.0, s->d_M, ni, s->d_C, ni, 0.0, D, ni));
  NGW_CUDA(dgemm(st, true, false, N, N, ni, 1.0, s->d_C, ni, D, ni, 0.0, Cm, N));
  k_dense_casida<<<elem_blocks(nn), 256, 0, st>>>(Cm, s->d_sqrtR, N);
  k_dense_identity<<<elem_blocks(nn), 256, 0, st>>>(P, N);
  NGW_CUDA(cudaGetLastError());
  if (k > 0) {
    // P C P = C - U G^T - Y U^T with G = C U, Y = G - U (U^T G); P = I - U U^T
    double *G = mat(((size_t)2 * N * k + (size_t)k * k));
    if (!G) {
      set_error("dense p(C): out of device memory");
      return NGW_ERR_OOM;
    }
    double *Yk = G + (size_t)N * k, *Wk = Yk + (size_t)N * k;
    const double *U = s->eig_U;
    NGW_CUDA(dgemm(st, false, false, N, k, N, 1.0, Cm, N, U, N, 0.0, G, N));
    NGW_CUDA(dgemm(st, true, false, k, k, N, 1.0, U, N, G, N, 0.0, Wk, k));
    NGW_CUDA(cudaMemcpyAsync(Yk, G, (size_t)N * k * 8, cudaMemcpyDeviceToDevice, st));
    NGW_CUDA(dgemm(st, false, false, N, k, k, -1.0, U, N, Wk, k, 1.0, Yk, N));
    NGW_CUDA(dgemm(st, false, true, N, N, k, -1.0, U, N, G, N, 1.0, Cm, N));
    NGW_CUDA(dgemm(st, false, true, N, N, k, -1.0, Yk, N, U, N, 1.0, Cm, N));
    NGW_CUDA(dgemm(st, false, true, N, N, k, -1.0, U, N, U, N, 1.0, P, N));
  }
  if (rmax >= 1) k_dense_x<<<elem_blocks(nn), 256, 0, st>>>(Cm, P, c0, 1.0 / c1, nn, T[1]);
  for (int r = 2; r <= rmax; ++r) {
    // T_r = 2 X T_{r-1} - T_{r-2}
    MatCombo mc{};
    mc.t[0] = T[r - 2];
    mc.c[0] = -1.0;
    mc.n = 1;
    k_dense_combo<<<elem_blocks(nn), 256, 0, st>>>(mc, nn, T[r]);
    NGW_CUDA(cudaGetLastError());
    NGW_CUDA(dgemm(st, false, false, N, N, N, 2.0, T[1], N, T[r - 1], N, 1.0, T[r], N));
  }
  auto digit = [&](int q, double *out) -> int {
    MatCombo mc{};
    mc.n = (int)dig[q].size();
    for (int r = 0; r < mc.n; ++r) {
      mc.t[r] = T[r];
      mc.c[r] = dig[q][r];
    }
    k_dense_combo<<<elem_blocks(nn), 256, 0, st>>>(mc, nn, out);
    NGW_CUDA(cudaGetLastError());
    return NGW_OK;
  };
  double *Yc = Y0, *Yn = Y1;
  NGW_TRY(digit(Q, Yc));
  for (int q = Q - 1; q >= 0; --q) {
    NGW_TRY(digit(q, Yn));
    NGW_CUDA(dgemm(st, false, false, N, N, N, 1.0, T[m], N, Yc, N, 1.0, Yn, N));
    std::swap(Yc, Yn);
  }
  double *Hm = Yc;
  // H -> split BF16 rows H[m][k]; padding rows / columns zero
  NGW_CUDA(cudaMemsetAsync(op->H_hi, 0, hbytes, st));
  NGW_CUDA(cudaMemsetAsync(op->H_lo, 0, hbytes, st));
  {
    dim3 grid((N + 31) / 32, (N + 31) / 32);
    k_split_transpose<<<grid, dim3(32, 8), 0, st>>>(Hm, N, N, op->H_hi, op->H_lo, kpad);
    NGW_CUDA(cudaGetLastError());
  }
  NGW_CUDA(cudaStreamSynchronize(st));
  NGW_TRY(make_tmap(&op->tHhi, op->H_hi, op->cv_pad, kpad, BM));
  NGW_TRY(make_tmap(&op->tHlo, op->H_lo, op->cv_pad, kpad, BM));
  op->dense_g.assign(g, g + n + 1);
  op->dense_c0 = c0;
  op->dense_c1 = c1;
  op->dense_ok = true;
  return check_status(s);
}

static int encode_dense_maps(MixedOperator *op, int bn) {
  if (op->maps_bnd != bn) {
    NGW_TRY(make_tmap(&op->tVhi, op->S_hi, op->nb_pad, op->cv_pad, bn));
    NGW_TRY(make_tmap(&op->tVlo, op->S_lo, op->nb_pad, op->cv_pad, bn));
    op->maps_bnd = bn;
  }
  return NGW_OK;
}

// out64 (ncv x nb, ld ldv) = H S + U p(Lambda) xo, S = the split chain vectors
static int run_dense_gemm(ngw_session *s, int nb, double *out64, int ldv) {
  MixedOperator *op = s->mixed;
  GemmArgs ga;
  ga.num_kb = op->kpad / BK;
  ga.nseg = 3;
  ga.nsplit = op->vard == 5 ? op->splitd : 1;
  EpiParams ep;
  std::memset(&ep, 0, sizeof(ep));
  ep.kind = EPI_CLENSHAW;
  ep.dense = 1;
  ep.Mv = s->ncv;
  ep.Nv = nb;
  ep.s = s->d_sqrtR;
  ep.ldx = op->cv_pad;
  ep.ldv = ldv;
  ep.out64 = out64;
  if (op->kdef > 0) {
    ep.Up = op->Up;
    ep.xo = op->xo;
    ep.kdef = op->kdef;
  }
  const int tiles_m = op->cv_pad / BM;
  const int tiles_n = (nb + op->BNd - 1) / op->BNd;
  return dispatch_tc(op->BNd, op->vard, op->tHhi, op->tHlo, op->tVhi, op->tVlo, tiles_m, tiles_n, ga, ep,
                     s->d_status, s->stream);
}

// out64 = p(C) v through the dense operator.  Launch-only.
int mixed_dense_apply(ngw_session *s, int nb, const double *v, int ldv, double *out64) {
  MixedOperator *op = s->mixed;
  if (!op || !op->dense_ok || op->nb_cap < nb || op->maps_bnd != op->BNd || !op->aux) {
    set_error("dense p(C): operator or chain buffers not prepared");
    return NGW_ERR_STATE;
  }
  // xo = U^T v (FP64 tensor cores) on the side stream beside the split B
  // operand on the session stream (two branches of a captured graph)
  cudaStream_t st = s->stream;
  if (op->kdef > 0) {
    NGW_CUDA(cudaEventRecord(op->ev_fork, st));
    NGW_CUDA(cudaStreamWaitEvent(op->aux, op->ev_fork, 0));
    k_dense_xo<<<(nb + 7) / 8, DP_W * 32, 0, op->aux>>>(v, ldv, s->ncv, nb, s->eig_U, op->kdef, op->xo);
    NGW_CUDA(cudaEventRecord(op->ev_join, op->aux));
  }
  k_split_chains<<<dim3((s->ncv + 1023) / 1024, nb), 256, 0, st>>>(v, ldv, s->ncv, nb, op->S_hi, op->S_lo,
                                                                  op->cv_pad);
  if (op->kdef > 0) NGW_CUDA(cudaStreamWaitEvent(st, op->ev_join, 0));
  NGW_CUDA(cudaGetLastError());
  return run_dense_gemm(s, nb, out64, ldv);
}

// Tile choice of the dense GEMM for nb chains: process-wide cache keyed by
// the shapes (so a request gives the same bits alone or among others), else
// every admissible (N tile, variant) timed on a quiet device.
// NGW_DENSE_TILES="bn,var" fixes it.
struct DenseKey {
  int cv_pad, kpad, nb, defl;
  bool operator<(const DenseKey &o) const {
    return std::tie(cv_pad, kpad, nb, defl) < std::tie(o.cv_pad, o.kpad, o.nb, o.defl);
  }
};
static std::mutex g_dtune_mu;
static std::map<DenseKey, TileC> g_dtune;

int mixed_prepare_dense(ngw_session *s, int nb) {
  MixedOperator *op = s->mixed;
  if (!op || !op->dense_ok) return NGW_OK;
  if (op->nb_cap < nb) {
    set_error("dense p(C): chain buffers not prepared");
    return NGW_ERR_STATE;
  }

  if (op->tuned_nbd == nb && op->maps_bnd == op->BNd) return NGW_OK;
  if (const char *env = getenv("NGW_DENSE_TILES")) {
    int bn = 0, var = 0, sp = 1;
    if (sscanf(env, "%d,%d,%d", &bn, &var, &sp) >= 2) {
      op->BNd = bn;
      op->vard = var;
      op->splitd = var == 5 ? std::max(2, sp) : 1;
      op->tuned_nbd = nb;
      return encode_dense_maps(op, bn);
    }
  }
  const DenseKey key{op->cv_pad, op->kpad, nb, op->kdef > 0 ? 1 : 0};
  {
    std::lock_guard<std::mutex> lk(g_dtune_mu);
    auto it = g_dtune.find(key);
    if (it != g_dtune.end()) {
      op->BNd = it->second.bn;
      op->vard = it->second.var;
      op->splitd = it->second.sp;
      op->tuned_nbd = nb;
      return encode_dense_maps(op, op->BNd);
    }
  }
  std::vector<TileC> cand;
  for (int bn : kBNs) {
    if (bn > round_up(nb, 16) && bn != kBNs[0]) continue;
    if ((round_up(nb, bn) - nb) * 8 > nb && bn != kBNs[0]) continue;
    for (int var : {0, 1, 2, 3, 4}) {
      if (var == 1 && !has_shallow(bn)) continue;
      if (var == 2 && !has_persistent(bn)) continue;
      if (var == 3 && !has_fused(bn)) continue;
      if (var == 4 && !has_fused2(bn)) continue;
      cand.push_back({bn, var, 1});
    }
    // cluster split-K (variant 5) with the wide tiles too
    if (bn >= 64) {
      const int tiles = (op->cv_pad / BM) * ((nb + bn - 1) / bn);
      for (int sp : {2, 3, 4})
        if (op->kpad / BK / sp >= 4 && tiles * sp <= 2 * 148) cand.push_back({bn, 5, sp});
    }
  }
  PoolTmp tout(s);
  NGW_CUDA(pool_alloc(s, &tout.p, (size_t)s->ncv * nb * 8));
  double *out = static_cast<double *>(tout.p);
  std::unique_lock<std::shared_mutex> quiet(gpu_quiet_lock(s->device));
  NGW_CUDA(cudaMemsetAsync(op->xo, 0, (size_t)nb * std::max(op->kdef, 1) * 8, s->stream));
  cudaEvent_t e0, e1;
  NGW_CUDA(cudaEventCreate(&e0));
  NGW_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  TileC pick = cand.empty() ? TileC{128, 3, 1} : cand[0];
  const bool verbose = getenv("NGW_TUNE_VERBOSE") != nullptr;
  int rc = NGW_OK;
  for (const auto &c : cand) {
    op->BNd = c.bn;
    op->vard = c.var;
    op->splitd = c.sp;
    if ((rc = encode_dense_maps(op, c.bn)) != NGW_OK) break;
    if ((rc = run_dense_gemm(s, nb, out, s->ncv)) != NGW_OK) break;
    float ms = 0.f;
    cudaEventRecord(e0, s->stream);
    for (int r = 0; r < 3 && rc == NGW_OK; ++r) rc = run_dense_gemm(s, nb, out, s->ncv);
    cudaEventRecord(e1, s->stream);
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
      set_error("dense GEMM tuning failed");
      rc = NGW_ERR_CUDA;
    }
    if (rc != NGW_OK) break;
    if (verbose) fprintf(stderr, "tune dense bn=%d var=%d split=%d: %.2f us\n", c.bn, c.var, c.sp, 1e3f * ms / 3);
    if (ms < best) {
      best = ms;
      pick = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  NGW_TRY(rc);
  op->BNd = pick.bn;
  op->vard = pick.var;
  op->splitd = pick.sp;
  op->tuned_nbd = nb;
  NGW_TRY(encode_dense_maps(op, op->BNd));
  {
    std::lock_guard<std::mutex> lk(g_dtune_mu);
    g_dtune[key] = pick;
  }
  return check_status(s);
}

// ---------------------------------------------------------------------------
// p(C) v for several molecules with the GEMMs grouped: per Clenshaw term one
// grouped GEMM1 and one grouped GEMM2 over every molecule still running
// (k_tc_gemm_grouped), the Clenshaw start per molecule.  The tables are
// built once per batch (group_build) and read by the kernels at execution
// time, so a captured graph replays them.
size_t group_bytes(int G, int n, int steps) {
  return (size_t)(1 + 2 * n) * G * sizeof(GroupEntry) + (size_t)steps * (3 * G + 2) * sizeof(int) + 256;
}

// Fill the tables into buf (device, group_bytes() long).  The members' chain
// buffers must be prepared for their chain counts.
int group_build(std::vector<GroupMember> &mem, int n, int tda, int steps, void *buf, cudaStream_t st,
                GroupPlan &P) {
  const int G = (int)mem.size();
  P.G = G;
  P.n = n;
  P.tda = tda;
  P.steps = steps;
  std::vector<GroupEntry> tab((size_t)(1 + 2 * n) * G);
  for (int i = 0; i < G; ++i) {
    ngw_session *s = mem[i].s;
    MixedOperator *op = s->mixed;
    if (!op || op->nb_cap < mem[i].nb) {
      set_error("grouped Sigma_c: chain buffers of member %d not prepared", i);
      return NGW_ERR_STATE;
    }
    // GEMM1: [T; q] = A1 S, split output, no split-K
    GroupEntry &e1 = tab[i];
    std::memset(&e1, 0, sizeof(e1));
    e1.tA_hi = op->tA1hi;
    e1.tA_lo = op->tA1lo;
    NGW_TRY(make_tmap(&e1.tB_hi, op->S_hi, op->nb_pad, op->cv_pad, GBN));
    NGW_TRY(make_tmap(&e1.tB_lo, op->S_lo, op->nb_pad, op->cv_pad, GBN));
    e1.ga.num_kb = op->cv_pad / BK;
    e1.ga.nseg = 3;
    e1.ga.nsplit = 1;
    e1.ep.kind = EPI_SPLIT;
    e1.ep.Mv = op->n_isdf + op->kdef;
    e1.ep.out_hi = op->T_hi;
    e1.ep.out_lo = op->T_lo;
    e1.ep.ldo = op->mu_k;
    e1.tiles_m = op->mu_pad / BM;
    // GEMM2 terms, the Clenshaw rotation of mixed_poly_apply
    CUtensorMap thi, tlo;
    NGW_TRY(make_tmap(&thi, op->T_hi, op->nb_pad, op->mu_k, GBN));
    NGW_TRY(make_tmap(&tlo, op->T_lo, op->nb_pad, op->mu_k, GBN));
    for (int set = 0; set < 2; ++set) {
      int cur = 0, prev = -1;
      for (int t = 0; t < n; ++t) {
        GroupEntry &e = tab[(size_t)G + ((size_t)set * n + t) * G + i];
        std::memset(&e, 0, sizeof(e));
        e.tA_hi = op->tA3hi;
        e.tA_lo = op->tA3lo;
        e.tB_hi = thi;
        e.tB_lo = tlo;
        e.ga.num_kb = op->mu_k / BK;
        e.ga.nseg = 3;
        e.ga.nsplit = 1;
        e.tiles_m = op->cv_pad / BM;
        EpiParams &ep = e.ep;
        ep.kind = EPI_CLENSHAW;
        ep.Mv = op->ncv;
        ep.s = s->d_sqrtR;
        ep.x = op->bb[cur];
        ep.b2 = prev < 0 ? nullptr : op->bb[prev];
        ep.v = op->vperp;
        ep.ldx = op->cv_pad;
        ep.ldv = mem[i].ldv;
        ep.c0 = mem[i].c0;
        ep.beta = 1.0;
        ep.tda = tda;
        ep.lds = op->cv_pad;
        ep.ring = 0;
        if (t < n - 1) {
          const int kk = n - 1 - t;
          const int outb = (prev < 0) ? 1 : 3 - cur - prev;
          ep.gamma = mem[i].g[kk];
          ep.alpha = 2.0 / mem[i].c1;
          ep.out32 = op->bb[outb];
          ep.s_hi = op->S_hi;
          ep.s_lo = op->S_lo;
          prev = cur;
          cur = outb;
        } else {
          ep.gamma = mem[i].g[0];
          ep.alpha = 1.0 / mem[i].c1;
          ep.out64 = set == 0 ? mem[i].out_first : mem[i].out_later;
          if (op->kdef > 0) {
            ep.Up = op->Up;
            ep.xo = op->xo;
            ep.kdef = op->kdef;
          }
        }
      }
    }
  }
  // per-step chain counts and tile ranges
  std::vector<int> hs((size_t)steps * (3 * G + 2));
  P.tiles1.assign(steps, 0);
  P.tiles2.assign(steps, 0);
  P.nv.assign((size_t)steps * G, 0);
  for (int k = 0; k < steps; ++k) {
    int *nvk = hs.data() + (size_t)k * (3 * G + 2), *tb1 = nvk + G, *tb2 = tb1 + G + 1;
    tb1[0] = tb2[0] = 0;
    for (int i = 0; i < G; ++i) {
      const int nk = (k == 0 || !mem[i].nact) ? mem[i].nb : mem[i].nact[k];
      nvk[i] = nk;
      P.nv[(size_t)k * G + i] = nk;
      const int tn = (nk + GBN - 1) / GBN;
      tb1[i + 1] = tb1[i] + tab[i].tiles_m * tn;
      tb2[i + 1] = tb2[i] + tab[(size_t)G + i].tiles_m * tn;
    }
    P.tiles1[k] = tb1[G];
    P.tiles2[k] = tb2[G];
  }
  char *b = static_cast<char *>(buf);
  b = reinterpret_cast<char *>(((uintptr_t)b + 127) & ~(uintptr_t)127);
  P.d_tab = reinterpret_cast<GroupEntry *>(b);
  P.d_steps = reinterpret_cast<int *>(b + tab.size() * sizeof(GroupEntry));
  NGW_CUDA(cudaMemcpyAsync(P.d_tab, tab.data(), tab.size() * sizeof(GroupEntry), cudaMemcpyHostToDevice, st));
  NGW_CUDA(cudaMemcpyAsync(P.d_steps, hs.data(), hs.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  NGW_CUDA(cudaStreamSynchronize(st));
  return NGW_OK;
}

// p(C) v of every member at Lanczos step k (vin[i]: its v, ld mem[i].ldv),
// all on stream st.  Launch-only.
int group_poly_apply(const GroupPlan &P, std::vector<GroupMember> &mem, int k, const double *const *vin,
                     cudaStream_t st) {
  const int G = P.G, n = P.n;
  const int *nvk = P.d_steps + (size_t)k * (3 * G + 2), *tb1 = nvk + G, *tb2 = tb1 + G + 1;
  for (int i = 0; i < G; ++i) {
    const int nk = P.nv[(size_t)k * G + i];
    if (nk > 0) NGW_TRY(mixed_poly_start(mem[i].s, nk, vin[i], mem[i].ldv, mem[i].g[n], P.tda, st));
  }
  if (P.tiles1[k] == 0) return NGW_OK;
  constexpr size_t smem = (size_t)GSTAGES * (BM * BK * 2 + GBN * BK * 2) * 2 + 1024;
  static std::atomic<unsigned long long> attr{0};
  NGW_CUDA(smem_limit_once(k_tc_gemm_grouped, (int)smem, attr));
  int *status = mem[0].s->d_status;
  const int set = k == 0 ? 0 : 1;
  for (int t = 0; t < n; ++t) {
    NGW_CUDA(launch_pdl(k_tc_gemm_grouped, dim3(P.tiles1[k]), dim3(NTHREADS), smem, st,
                        (const GroupEntry *)P.d_tab, tb1, nvk, G, status));
    NGW_CUDA(launch_pdl(k_tc_gemm_grouped, dim3(P.tiles2[k]), dim3(NTHREADS), smem, st,
                        (const GroupEntry *)(P.d_tab + G + ((size_t)set * n + t) * G), tb2, nvk, G, status));
  }
  return NGW_OK;
}

// Monomial (high -> low, reference order) -> Chebyshev coefficients on
// [lo, hi] by interpolation at n+1 Chebyshev nodes (exact for degree n),
// evaluated in long double.
void monomial_to_chebyshev(const double *poly_hl, int n, double lo, double hi, double *g) {
  const long double c0 = 0.5L * ((long double)hi + lo), c1 = 0.5L * ((long double)hi - lo);
  const int N = n + 1;
  std::vector<long double> f(N), t(N);
  const long double PI = 3.141592653589793238462643383279502884L;
  for (int i = 0; i < N; ++i) {
    t[i] = cosl(PI * (i + 0.5L) / N);
    const long double x = c0 + c1 * t[i];
    long double acc = 0.0L;
    for (int k = 0; k <= n; ++k) acc = acc * x + (long double)poly_hl[k];
    f[i] = acc;
  }
  for (int k = 0; k <= n; ++k) {
    long double acc = 0.0L;
    for (int i = 0; i < N; ++i) acc += f[i] * cosl(k * PI * (i + 0.5L) / N);
    acc *= 2.0L / N;
    if (k == 0) acc *= 0.5L;
    g[k] = (double)acc;
  }
}

}  // namespace ngw

// ---------------------------------------------------------------------------
// Per-kernel timing of the two mixed-precision GEMMs on the session stream
// (CUDA events around `reps` back-to-back launches of each), used by the
// benchmark's roofline report.  Operates on the session's own chain buffers.
extern "C" int ngw_profile_mixed_gemms(ngw_session *s, int nb, int reps, double *us_gemm1,
                                       double *us_gemm2) {
  using namespace ngw;
  if (!s || nb <= 0 || reps <= 0 || !us_gemm1 || !us_gemm2) {
    set_error("ngw_profile_mixed_gemms: bad arguments");
    return NGW_ERR_ARG;
  }
  if (!s->mixed) {
    set_error("mixed operator not built (run a mixed-precision solve first)");
    return NGW_ERR_STATE;
  }
  NGW_CUDA(cudaSetDevice(s->device));
  NGW_TRY(mixed_prepare_chains(s, nb, 0, 0, 0));
  MixedOperator *op = s->mixed;
  cudaEvent_t e0, e1, e2;
  NGW_CUDA(cudaEventCreate(&e0));
  NGW_CUDA(cudaEventCreate(&e1));
  NGW_CUDA(cudaEventCreate(&e2));
  NGW_TRY(run_gemm1(s, nb));   // warm
  NGW_TRY(run_gemm2(s, nb, op->bb[0], nullptr, nullptr, 0, 0.0, 1.0, 0.0, 0.0, 0, op->bb[1],
                    nullptr, true));
  NGW_CUDA(cudaEventRecord(e0, s->stream));
  for (int i = 0; i < reps; ++i) NGW_TRY(run_gemm1(s, nb));
  NGW_CUDA(cudaEventRecord(e1, s->stream));
  for (int i = 0; i < reps; ++i)
    NGW_TRY(run_gemm2(s, nb, op->bb[0], nullptr, nullptr, 0, 0.0, 1.0, 0.0, 0.0, 0, op->bb[1],
                      nullptr, true));
  NGW_CUDA(cudaEventRecord(e2, s->stream));
  NGW_CUDA(cudaEventSynchronize(e2));
  float t1 = 0, t2 = 0;
  NGW_CUDA(cudaEventElapsedTime(&t1, e0, e1));
  NGW_CUDA(cudaEventElapsedTime(&t2, e1, e2));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  *us_gemm1 = 1e3 * t1 / reps;
  *us_gemm2 = 1e3 * t2 / reps;
  return check_status(s);
}

// The dense p(C) GEMM of the mixed form (when the session's last plan built
// it): mean device time of one launch for nb chains and its shape.
extern "C" int ngw_profile_dense_gemm(ngw_session *s, int nb, int reps, double *us, int *shape) {
  using namespace ngw;
  if (!s || nb <= 0 || reps <= 0 || !us || !shape) {
    set_error("ngw_profile_dense_gemm: bad arguments");
    return NGW_ERR_ARG;
  }
  if (!s->mixed || !s->mixed->dense_ok || !s->mixed->dense_last) {
    set_error("dense p(C) operator not in use (the last mixed plan used the factored form)");
    return NGW_ERR_STATE;
  }
  NGW_CUDA(cudaSetDevice(s->device));
  NGW_TRY(mixed_prepare_chains(s, nb, 0, 0, 0));
  NGW_TRY(mixed_prepare_dense(s, nb));
  MixedOperator *op = s->mixed;
  PoolTmp tout(s);
  NGW_CUDA(pool_alloc(s, &tout.p, (size_t)s->ncv * nb * 8));
  double *out = static_cast<double *>(tout.p);
  NGW_CUDA(cudaMemsetAsync(op->xo, 0, (size_t)nb * std::max(op->kdef, 1) * 8, s->stream));
  cudaEvent_t e0, e1;
  NGW_CUDA(cudaEventCreate(&e0));
  NGW_CUDA(cudaEventCreate(&e1));
  NGW_TRY(run_dense_gemm(s, nb, out, s->ncv));   // warm
  NGW_CUDA(cudaEventRecord(e0, s->stream));
  for (int i = 0; i < reps; ++i) NGW_TRY(run_dense_gemm(s, nb, out, s->ncv));
  NGW_CUDA(cudaEventRecord(e1, s->stream));
  NGW_CUDA(cudaEventSynchronize(e1));
  float t = 0;
  NGW_CUDA(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *us = 1e3 * t / reps;
  shape[0] = s->ncv;
  shape[1] = nb;
  shape[2] = s->ncv;
  shape[3] = op->BNd;
  shape[4] = op->vard * 16 + op->splitd;
  return check_status(s);
}

// Shapes of the two GEMMs for the roofline (valid M, N, K, N tile, split-K).
extern "C" int ngw_mixed_gemm_shapes(ngw_session *s, int nb, int *shape) {
  using namespace ngw;
  if (!s || !s->mixed || !shape) {
    set_error("mixed operator not built");
    return NGW_ERR_STATE;
  }
  NGW_TRY(mixed_prepare_chains(s, nb, 0, 0, 0));
  MixedOperator *op = s->mixed;
  shape[0] = op->n_isdf + op->kdef; shape[1] = nb; shape[2] = op->ncv; shape[3] = op->BN1;
  shape[4] = op->split1;
  shape[5] = op->ncv; shape[6] = nb; shape[7] = op->n_isdf + op->kdef; shape[8] = op->BN2;
  shape[9] = op->var1; shape[10] = op->var2;
  shape[11] = op->split2; shape[12] = 0;
  return NGW_OK;
}

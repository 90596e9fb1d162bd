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

#include <cmath>
#include <cstring>
#include <mutex>

#include "ngw_internal.h"
#include "tc_gemm.cuh"

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
  // split-K
  float *ws;
  int *counters;
  // EPI_CLENSHAW: rows m = pair index, cols n = chain
  const double *s;       // sqrtR (Mv)
  const float *x;        // b_{k+1}  [n * ldx + m]
  const float *b2;       // b_{k+2}  (nullable)
  const double *v;       // Lanczos vector [n * ldv + m]
  int ldx, ldv;
  double gamma, alpha, c0, beta;
  int tda;
  float *out32;          // b_k (nullable)
  double *out64;         // final p(C) v (nullable)
  bf16 *s_hi, *s_lo;     // split of (R^1/2 or 1) * out  [n * lds + m] (nullable)
  int lds;
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

template <int BN, int STAGES>
__global__ void __launch_bounds__(128, 1)
    k_tc_gemm(const __grid_constant__ CUtensorMap tA_hi, const __grid_constant__ CUtensorMap tA_lo,
              const __grid_constant__ CUtensorMap tB_hi, const __grid_constant__ CUtensorMap tB_lo,
              GemmArgs ga, EpiParams ep, int *status) {
  constexpr uint32_t A_BYTES = BM * BK * 2;
  constexpr uint32_t B_BYTES = BN * BK * 2;
  constexpr uint32_t STAGE_BYTES = A_BYTES + B_BYTES;
  constexpr uint32_t TMEM_COLS = (BN <= 32) ? 32 : (BN <= 64) ? 64 : (BN <= 128) ? 128 : 256;
  constexpr uint32_t IDESC = tc::idesc_bf16_f32(BM, BN);

  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  __shared__ __align__(8) uint64_t full_bar[STAGES];
  __shared__ __align__(8) uint64_t empty_bar[STAGES];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int last_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int split = blockIdx.z;
  const int total_kb = ga.num_kb * ga.nseg;
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
    tc::fence_barrier_init();
    tc::prefetch_tmap(&tA_hi);
    tc::prefetch_tmap(&tB_hi);
  }
  if (warp == 2) {
    tc::tmem_alloc(tc::smem_u32(&tmem_base_sh), TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem_d = tmem_base_sh;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer ----
    for (int i = 0; i < nkb; ++i) {
      const int s = i % STAGES;
      if (i >= STAGES) {
        if (!tc::mbar_wait(tc::smem_u32(&empty_bar[s]), ((i / STAGES) - 1) & 1, status)) break;
      }
      const int kbg = kb_begin + i;
      const int seg = kbg / ga.num_kb;
      const int kb = kbg - seg * ga.num_kb;
      const CUtensorMap *ta = (seg == 2) ? &tA_lo : &tA_hi;
      const CUtensorMap *tb = (seg == 1) ? &tB_lo : &tB_hi;
      const uint32_t bar = tc::smem_u32(&full_bar[s]);
      const uint32_t sa = tc::smem_u32(smem + s * STAGE_BYTES);
      tc::mbar_arrive_expect_tx(bar, STAGE_BYTES);
      tc::tma_load_2d(sa, ta, bar, kb * BK, m0);
      tc::tma_load_2d(sa + A_BYTES, tb, bar, kb * BK, n0);
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    bool ok = true;
    for (int i = 0; i < nkb && ok; ++i) {
      const int s = i % STAGES;
      if (!tc::mbar_wait(tc::smem_u32(&full_bar[s]), (i / STAGES) & 1, status)) {
        ok = false;
        break;
      }
      tc::tc_fence_after();
      const uint32_t sa = tc::smem_u32(smem + s * STAGE_BYTES);
      const uint32_t sb = sa + A_BYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk) {
        const uint64_t ad = tc::smem_desc_sw128(sa + kk * 32);
        const uint64_t bd = tc::smem_desc_sw128(sb + kk * 32);
        tc::mma_bf16(tmem_d, ad, bd, IDESC, (i > 0 || kk > 0) ? 1u : 0u);
      }
      tc::mma_commit(tc::smem_u32(&empty_bar[s]));
    }
    tc::mma_commit(tc::smem_u32(&done_bar));
  }
  __syncwarp();

  // ---- epilogue: all four warps, thread <-> accumulator row ----
  const bool have = tc::mbar_wait(tc::smem_u32(&done_bar), 0, status);
  tc::tc_fence_after();
  const int mloc = warp * 32 + lane;
  const int m = m0 + mloc;
  const uint32_t trow = tmem_d + ((uint32_t)(warp * 32) << 16);

  if (ep.kind == EPI_SPLIT && ga.nsplit > 1) {
    const int tiles_m = gridDim.x;
    const int tile = blockIdx.y * tiles_m + blockIdx.x;
    float *wsl = ep.ws + ((size_t)tile * ga.nsplit + split) * (size_t)(BN * BM);
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      if (have && nkb > 0) {
        tc::tmem_ld16(trow + c, v);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = 0.f;
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) wsl[(size_t)(c + j) * BM + mloc] = v[j];
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      int old = atomicAdd(&ep.counters[tile], 1);
      last_flag = (old == ga.nsplit - 1);
    }
    __syncthreads();
    if (last_flag) {
      __threadfence();
      const float *base = ep.ws + (size_t)tile * ga.nsplit * (size_t)(BN * BM);
      for (int c = 0; c < BN; ++c) {
        const int n = n0 + c;
        float acc = 0.f;
        for (int sp = 0; sp < ga.nsplit; ++sp)
          acc += __ldcg(base + (size_t)sp * (BN * BM) + (size_t)c * BM + mloc);
        if (m < ep.Mv && n < ep.Nv) {
          bf16 hi, lo;
          split_bf16(acc, hi, lo);
          ep.out_hi[(size_t)n * ep.ldo + m] = hi;
          ep.out_lo[(size_t)n * ep.ldo + m] = lo;
        }
      }
      if (threadIdx.x == 0) ep.counters[tile] = 0;
    }
  } else if (ep.kind == EPI_SPLIT) {
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      if (have && nkb > 0) {
        tc::tmem_ld16(trow + c, v);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = 0.f;
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = n0 + c + j;
        if (m < ep.Mv && n < ep.Nv) {
          bf16 hi, lo;
          split_bf16(v[j], hi, lo);
          ep.out_hi[(size_t)n * ep.ldo + m] = hi;
          ep.out_lo[(size_t)n * ep.ldo + m] = lo;
        }
      }
    }
  } else {
    // EPI_CLENSHAW
    const bool mv = m < ep.Mv;
    const double si = mv ? ep.s[m] : 0.0;
    const double s2 = si * si;
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      if (have && nkb > 0) {
        tc::tmem_ld16(trow + c, v);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = 0.f;
      }
#pragma unroll 4
      for (int j = 0; j < 16; ++j) {
        const int n = n0 + c + j;
        if (!mv || n >= ep.Nv) continue;
        const double x = (double)ep.x[(size_t)n * ep.ldx + m];
        const double z = (double)v[j];
        const double y = ep.tda ? (s2 * x + 2.0 * z) : (s2 * s2 * x + 4.0 * si * z);
        double o = ep.alpha * (y - ep.c0 * x);
        if (ep.v) o += ep.gamma * ep.v[(size_t)n * ep.ldv + m];
        if (ep.b2) o -= ep.beta * (double)ep.b2[(size_t)n * ep.ldx + m];
        if (ep.out32) ep.out32[(size_t)n * ep.ldx + m] = (float)o;
        if (ep.out64) ep.out64[(size_t)n * ep.ldv + m] = o;
        if (ep.s_hi) {
          bf16 hi, lo;
          split_bf16((float)(ep.tda ? o : si * o), hi, lo);
          ep.s_hi[(size_t)n * ep.lds + m] = hi;
          ep.s_lo[(size_t)n * ep.lds + m] = lo;
        }
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

template <int BN, int STAGES>
static int launch_tc(const CUtensorMap &a_hi, const CUtensorMap &a_lo, const CUtensorMap &b_hi,
                     const CUtensorMap &b_lo, int tiles_m, int tiles_n, const GemmArgs &ga,
                     const EpiParams &ep, int *status, cudaStream_t st) {
  constexpr size_t smem = (size_t)STAGES * (BM * BK * 2 + BN * BK * 2) + 1024;
  static bool attr = false;
  if (!attr) {
    NGW_CUDA(cudaFuncSetAttribute(k_tc_gemm<BN, STAGES>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  dim3 grid(tiles_m, tiles_n, ga.nsplit);
  k_tc_gemm<BN, STAGES><<<grid, 128, smem, st>>>(a_hi, a_lo, b_hi, b_lo, ga, ep, status);
  NGW_CUDA(cudaGetLastError());
  return NGW_OK;
}

// supported N tiles (multiples of 16, <= 256); chosen per chain count
static const int kBNs[] = {64, 80, 96, 128, 144, 160, 192, 240, 256};

static int dispatch_tc(int BN, const CUtensorMap &a_hi, const CUtensorMap &a_lo,
                       const CUtensorMap &b_hi, const CUtensorMap &b_lo, int tiles_m, int tiles_n,
                       const GemmArgs &ga, const EpiParams &ep, int *status, cudaStream_t st) {
  switch (BN) {
    case 64: return launch_tc<64, 8>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st);
    case 80: return launch_tc<80, 8>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st);
    case 96: return launch_tc<96, 8>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st);
    case 128: return launch_tc<128, 6>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st);
    case 144: return launch_tc<144, 6>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st);
    case 160: return launch_tc<160, 5>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st);
    case 192: return launch_tc<192, 5>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st);
    case 240: return launch_tc<240, 4>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st);
    case 256: return launch_tc<256, 4>(a_hi, a_lo, b_hi, b_lo, tiles_m, tiles_n, ga, ep, status, st);
  }
  set_error("unsupported N tile %d", BN);
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
      bf16 h, l;
      const double x = tile[threadIdx.x][r];
      h = __double2bfloat16(x);
      l = __double2bfloat16(x - (double)__bfloat162float(h));
      hi[(size_t)mu * ldk + cv] = h;
      lo[(size_t)mu * ldk + cv] = l;
    }
  }
}

// D (n_isdf, ncv) FP64 column-major -> A3[cv][mu] hi/lo (row length ldk)
__global__ void k_split_rows(const double *__restrict__ D, int n_isdf, int ncv,
                             bf16 *__restrict__ hi, bf16 *__restrict__ lo, int ldk) {
  const int cv = blockIdx.y;
  for (int mu = blockIdx.x * blockDim.x + threadIdx.x; mu < n_isdf; mu += gridDim.x * blockDim.x) {
    const double x = D[(size_t)cv * n_isdf + mu];
    bf16 h = __double2bfloat16(x);
    bf16 l = __double2bfloat16(x - (double)__bfloat162float(h));
    hi[(size_t)cv * ldk + mu] = h;
    lo[(size_t)cv * ldk + mu] = l;
  }
}

// Clenshaw start: b_n = g * v (FP32) and split((R^1/2 or 1) * b_n)
__global__ void k_cheb_start(const double *__restrict__ v, int ldv, const double *__restrict__ s,
                             int ncv, int nb, double g, int tda, float *__restrict__ bn, int ldx,
                             bf16 *__restrict__ shi, bf16 *__restrict__ slo, int lds) {
  const int j = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncv; i += gridDim.x * blockDim.x) {
    const double b = g * v[(size_t)j * ldv + i];
    bn[(size_t)j * ldx + i] = (float)b;
    const double u = tda ? b : s[i] * b;
    bf16 h, l;
    split_bf16((float)u, h, l);
    shi[(size_t)j * lds + i] = h;
    slo[(size_t)j * lds + i] = l;
  }
}

struct MixedOperator {
  int n_isdf = 0, ncv = 0;
  int mu_pad = 0;     // rows of A1 (multiple of 128)
  int mu_k = 0;       // K of GEMM2 (multiple of 64)
  int cv_pad = 0;     // K of GEMM1 / rows of A3 (multiple of 128)
  bf16 *A1_hi = nullptr, *A1_lo = nullptr, *A3_hi = nullptr, *A3_lo = nullptr;
  CUtensorMap tA1hi, tA1lo, tA3hi, tA3lo;
  size_t op_bytes = 0;
  // chain buffers
  int nb_cap = 0, nb_pad = 0, BN1 = 128, BN2 = 128, split1 = 1;
  bf16 *S_hi = nullptr, *S_lo = nullptr, *T_hi = nullptr, *T_lo = nullptr;
  CUtensorMap tShi, tSlo, tThi, tTlo;
  float *bb[3] = {nullptr, nullptr, nullptr};
  float *ws = nullptr;
  int *counters = nullptr;
  size_t buf_bytes = 0;
};

static int round_up(int a, int b) { return (a + b - 1) / b * b; }

void mixed_free(ngw_session *s) {
  MixedOperator *op = s->mixed;
  if (!op) return;
  void *ptrs[] = {op->A1_hi, op->A1_lo, op->A3_hi, op->A3_lo, op->S_hi, op->S_lo, op->T_hi,
                  op->T_lo,  op->bb[0], op->bb[1], op->bb[2], op->ws,    op->counters};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  s->bytes -= op->op_bytes + op->buf_bytes;
  delete op;
  s->mixed = nullptr;
}

static void free_chain_buffers(ngw_session *s, MixedOperator *op) {
  void *ptrs[] = {op->S_hi, op->S_lo, op->T_hi, op->T_lo, op->bb[0], op->bb[1], op->bb[2],
                  op->ws,   op->counters};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  op->S_hi = op->S_lo = op->T_hi = op->T_lo = nullptr;
  op->bb[0] = op->bb[1] = op->bb[2] = nullptr;
  op->ws = nullptr;
  op->counters = nullptr;
  s->bytes -= op->buf_bytes;
  op->buf_bytes = 0;
  op->nb_cap = 0;
}

// Build A1 = split(C^T-layout) and A3 = split((M C) layout) from the FP64
// pair products already in the session.
int mixed_build_operator(ngw_session *s) {
  mixed_free(s);
  MixedOperator *op = new MixedOperator();
  s->mixed = op;
  op->n_isdf = s->n_isdf;
  op->ncv = s->ncv;
  op->mu_pad = round_up(s->n_isdf, BM);
  op->mu_k = round_up(s->n_isdf, BK);
  op->cv_pad = round_up(s->ncv, BM);
  const size_t a1 = (size_t)op->mu_pad * op->cv_pad * sizeof(bf16);
  const size_t a3 = (size_t)op->cv_pad * op->mu_k * sizeof(bf16);
  NGW_CUDA(cudaMalloc(&op->A1_hi, a1));
  NGW_CUDA(cudaMalloc(&op->A1_lo, a1));
  NGW_CUDA(cudaMalloc(&op->A3_hi, a3));
  NGW_CUDA(cudaMalloc(&op->A3_lo, a3));
  op->op_bytes = 2 * (a1 + a3);
  s->bytes += op->op_bytes;
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
  // D = M * C (FP64, cuBLAS), then split into A3[cv][mu]
  double *D = nullptr;
  NGW_CUDA(cudaMalloc(&D, (size_t)s->n_isdf * s->ncv * sizeof(double)));
  const double one = 1.0, zero = 0.0;
  cublasStatus_t cst = cublasDgemm(s->cublas, CUBLAS_OP_N, CUBLAS_OP_N, s->n_isdf, s->ncv,
                                   s->n_isdf, &one, s->d_M, s->n_isdf, s->d_C, s->n_isdf, &zero,
                                   D, s->n_isdf);
  if (cst != CUBLAS_STATUS_SUCCESS) {
    cudaFree(D);
    set_error("cublasDgemm (M*C) failed %d", (int)cst);
    return NGW_ERR_CUDA;
  }
  {
    int bx = (s->n_isdf + 127) / 128;
    k_split_rows<<<dim3(bx, s->ncv), 128, 0, st>>>(D, s->n_isdf, s->ncv, op->A3_hi, op->A3_lo,
                                                   op->mu_k);
    NGW_CUDA(cudaGetLastError());
  }
  NGW_CUDA(cudaStreamSynchronize(st));
  cudaFree(D);
  NGW_TRY(make_tmap(&op->tA1hi, op->A1_hi, op->mu_pad, op->cv_pad, BM));
  NGW_TRY(make_tmap(&op->tA1lo, op->A1_lo, op->mu_pad, op->cv_pad, BM));
  NGW_TRY(make_tmap(&op->tA3hi, op->A3_hi, op->cv_pad, op->mu_k, BM));
  NGW_TRY(make_tmap(&op->tA3lo, op->A3_lo, op->cv_pad, op->mu_k, BM));
  return NGW_OK;
}

static int pick_bn(int nb) {
  // smallest padding waste, then the larger tile
  int best = 128, best_pad = 1 << 30;
  for (int bn : kBNs) {
    int pad = round_up(nb, bn) - nb;
    if (pad < best_pad || (pad == best_pad && bn > best)) {
      best = bn;
      best_pad = pad;
    }
  }
  return best;
}

int mixed_prepare_chains(ngw_session *s, int nb, int bn1, int bn2, int split1) {
  MixedOperator *op = s->mixed;
  if (!op) {
    set_error("mixed operator not built");
    return NGW_ERR_STATE;
  }
  if (bn1 <= 0) bn1 = pick_bn(nb);
  if (bn2 <= 0) bn2 = pick_bn(nb);
  const int tiles_m1 = op->mu_pad / BM;
  const int tiles_n1 = (nb + bn1 - 1) / bn1;
  if (split1 <= 0) {
    const int total_kb = 3 * (op->cv_pad / BK);
    split1 = 1;
    while (tiles_m1 * tiles_n1 * split1 * 2 <= 148 && split1 * 2 * 4 <= total_kb) split1 *= 2;
  }
  const int nbp = round_up(nb, 256);
  if (op->nb_cap >= nb && op->BN1 == bn1 && op->BN2 == bn2 && op->split1 == split1) return NGW_OK;
  free_chain_buffers(s, op);
  op->BN1 = bn1;
  op->BN2 = bn2;
  op->split1 = split1;
  op->nb_pad = nbp;
  const size_t sbytes = (size_t)nbp * op->cv_pad * sizeof(bf16);
  const size_t tbytes = (size_t)nbp * op->mu_k * sizeof(bf16);
  const size_t bbytes = (size_t)nbp * op->cv_pad * sizeof(float);
  const size_t wsbytes = (size_t)tiles_m1 * ((nbp + bn1 - 1) / bn1) * split1 * bn1 * BM * sizeof(float);
  const size_t cbytes = (size_t)tiles_m1 * ((nbp + bn1 - 1) / bn1) * sizeof(int);
  NGW_CUDA(cudaMalloc(&op->S_hi, sbytes));
  NGW_CUDA(cudaMalloc(&op->S_lo, sbytes));
  NGW_CUDA(cudaMalloc(&op->T_hi, tbytes));
  NGW_CUDA(cudaMalloc(&op->T_lo, tbytes));
  for (int i = 0; i < 3; ++i) NGW_CUDA(cudaMalloc(&op->bb[i], bbytes));
  NGW_CUDA(cudaMalloc(&op->ws, wsbytes));
  NGW_CUDA(cudaMalloc(&op->counters, cbytes));
  op->buf_bytes = 2 * sbytes + 2 * tbytes + 3 * bbytes + wsbytes + cbytes;
  s->bytes += op->buf_bytes;
  NGW_CUDA(cudaMemsetAsync(op->S_hi, 0, sbytes, s->stream));
  NGW_CUDA(cudaMemsetAsync(op->S_lo, 0, sbytes, s->stream));
  NGW_CUDA(cudaMemsetAsync(op->T_hi, 0, tbytes, s->stream));
  NGW_CUDA(cudaMemsetAsync(op->T_lo, 0, tbytes, s->stream));
  NGW_CUDA(cudaMemsetAsync(op->counters, 0, cbytes, s->stream));
  NGW_TRY(make_tmap(&op->tShi, op->S_hi, nbp, op->cv_pad, bn1));
  NGW_TRY(make_tmap(&op->tSlo, op->S_lo, nbp, op->cv_pad, bn1));
  NGW_TRY(make_tmap(&op->tThi, op->T_hi, nbp, op->mu_k, bn2));
  NGW_TRY(make_tmap(&op->tTlo, op->T_lo, nbp, op->mu_k, bn2));
  op->nb_cap = nbp;
  return NGW_OK;
}

// One GEMM1 (T = C_isdf S) with split output into T_hi/T_lo.
static int run_gemm1(ngw_session *s, int nb) {
  MixedOperator *op = s->mixed;
  GemmArgs ga;
  ga.num_kb = op->cv_pad / BK;
  ga.nseg = 3;
  ga.nsplit = op->split1;
  EpiParams ep;
  std::memset(&ep, 0, sizeof(ep));
  ep.kind = EPI_SPLIT;
  ep.Mv = op->n_isdf;
  ep.Nv = nb;
  ep.out_hi = op->T_hi;
  ep.out_lo = op->T_lo;
  ep.ldo = op->mu_k;
  ep.ws = op->ws;
  ep.counters = op->counters;
  const int tiles_m = op->mu_pad / BM;
  const int tiles_n = (nb + op->BN1 - 1) / op->BN1;
  return dispatch_tc(op->BN1, op->tA1hi, op->tA1lo, op->tShi, op->tSlo, tiles_m, tiles_n, ga, ep,
                     s->d_status, s->stream);
}

// One GEMM2 with the Clenshaw epilogue.
static int run_gemm2(ngw_session *s, int nb, const float *x, const float *b2, const double *v,
                     int ldv, double gamma, double alpha, double c0, double beta, int tda,
                     float *out32, double *out64, bool write_split) {
  MixedOperator *op = s->mixed;
  GemmArgs ga;
  ga.num_kb = op->mu_k / BK;
  ga.nseg = 3;
  ga.nsplit = 1;
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
  const int tiles_m = op->cv_pad / BM;
  const int tiles_n = (nb + op->BN2 - 1) / op->BN2;
  return dispatch_tc(op->BN2, op->tA3hi, op->tA3lo, op->tThi, op->tTlo, tiles_m, tiles_n, ga, ep,
                     s->d_status, s->stream);
}

// out64 (ncv x nb, ld ldv) = p(C) v with p given by Chebyshev coefficients
// g[0..n] on [c0 - c1, c0 + c1].  v: FP64 (ld ldv).  Launch-only (no sync),
// so it can be captured in a CUDA graph.
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
  cudaStream_t st = s->stream;
  {
    int bx = (s->ncv + 255) / 256;
    if (bx > 16) bx = 16;
    k_cheb_start<<<dim3(bx, nb), 256, 0, st>>>(v, ldv, s->d_sqrtR, s->ncv, nb, g[n], tda,
                                              op->bb[0], op->cv_pad, op->S_hi, op->S_lo,
                                              op->cv_pad);
    NGW_CUDA(cudaGetLastError());
  }
  // buffers: cur = b_{k+1}, prev = b_{k+2}
  int cur = 0, prev = -1;
  for (int k = n - 1; k >= 1; --k) {
    NGW_TRY(run_gemm1(s, nb));
    // b_k goes to the slot that is neither b_{k+1} nor b_{k+2}
    const int outb = (prev < 0) ? 1 : 3 - cur - prev;
    NGW_TRY(run_gemm2(s, nb, op->bb[cur], prev < 0 ? nullptr : op->bb[prev], v, ldv, g[k],
                      2.0 / c1, c0, 1.0, tda, op->bb[outb], nullptr, true));
    prev = cur;
    cur = outb;
  }
  NGW_TRY(run_gemm1(s, nb));
  NGW_TRY(run_gemm2(s, nb, op->bb[cur], prev < 0 ? nullptr : op->bb[prev], v, ldv, g[0],
                    1.0 / c1, c0, 1.0, tda, nullptr, out64, false));
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
    set_error("mixed operator not built (set precision to mixed and set the operator)");
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

// Shapes of the two GEMMs for the roofline (padded M, N, K and split-K).
extern "C" int ngw_mixed_gemm_shapes(ngw_session *s, int nb, int *shape) {
  using namespace ngw;
  if (!s || !s->mixed || !shape) {
    set_error("mixed operator not built");
    return NGW_ERR_STATE;
  }
  NGW_TRY(mixed_prepare_chains(s, nb, 0, 0, 0));
  MixedOperator *op = s->mixed;
  shape[0] = op->n_isdf; shape[1] = nb; shape[2] = op->ncv; shape[3] = op->BN1; shape[4] = op->split1;
  shape[5] = op->ncv; shape[6] = nb; shape[7] = op->n_isdf; shape[8] = op->BN2;
  return NGW_OK;
}

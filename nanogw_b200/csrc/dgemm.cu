// FP64 GEMM on the FP64 tensor cores (mma.sync m8n8k4 .f64; tcgen05 has no
// FP64 kind, so this is the FP64 tensor path of sm_100a).
//
//   C (m x n) = alpha * op(A) op(B) + beta * C,   column-major, cuBLAS-style
//   op(A) = A (m x k, lda >= m) or A^T (A: k x m, lda >= k), same for B.
//
// It replaces the library DGEMMs of the ISDF kernel build, the fit's P / Q
// products, the Sigma_c start vectors, the deflation projection, the
// eigen-pair Ritz vectors, the exchange / V_xc projections and the kernel
// contraction of k_integrate.
//
// Tiles: 128 x 128 (8 warps as 2 x 4, a 64 x 32 tile per warp) or 64 x 64
// (4 warps as 2 x 2, 32 x 32 per warp) over K steps of 16, staged in shared
// memory by 8-byte cp.async (any alignment and leading dimension) in a
// 4-stage ring; zero fill past the matrix edges.  The operand tiles are laid
// out in shared memory so that each half-warp's fragment loads hit 16
// distinct bank pairs (padding 4 doubles along the contiguous index, or rows
// of 20 doubles).  Shapes whose tile grid would leave most SMs idle split K
// into slices that write partial tiles to a workspace, summed afterwards in
// slice order (deterministic).
#include <algorithm>

#include "ngw_internal.h"

namespace ngw {

namespace {

constexpr int DG_BK = 16;
constexpr int DG_STAGES = 4;
constexpr int DG_PAD = 4;      // doubles of padding on the contiguous index
constexpr int DG_KROW = 20;    // doubles per row when K is the contiguous index

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem, bool pred) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int n = pred ? 8 : 0;   // 0 source bytes: the destination is zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Elements of one operand tile per stage (the larger of the two layouts).
template <int BMN>
__host__ __device__ constexpr int tile_elems() {
  return (DG_BK * (BMN + DG_PAD) > BMN * DG_KROW) ? DG_BK * (BMN + DG_PAD) : BMN * DG_KROW;
}

__device__ __forceinline__ void cp_async16(double *smem, const double *gmem, int src_bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  // src_bytes < 16: the rest of the 16 destination bytes is zero-filled
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}

// Stage the (rows x BK) tile of an operand whose op(X)[r][kk] is X[r + kk*ld]
// (contiguous along r; TR = false) or X[kk + r*ld] (contiguous along kk;
// TR = true).  Shared layout: TR = false -> S[kk][r] with row length
// BMN + PAD; TR = true -> S[r][kk] with row length KROW.  With vec (X
// 16-byte aligned, ld even) pairs of elements along the contiguous index
// move as one 16-byte copy.
template <int BMN, int NT, bool TR>
__device__ __forceinline__ void load_tile(double *S, const double *X, int ld, int r0, int rows, int k0, int K,
                                          bool vec) {
  constexpr int E = BMN * DG_BK;
  if (vec) {
    for (int e = 2 * threadIdx.x; e < E; e += 2 * NT) {
      int r, kk;
      if (!TR) {
        r = e % BMN;
        kk = e / BMN;
      } else {
        kk = e % DG_BK;
        r = e / DG_BK;
      }
      const int gr = r0 + r, gk = k0 + kk;
      int nvalid;   // valid elements of the pair (0, 1, 2)
      const double *src = X;
      if (!TR) {
        nvalid = (gk < K) ? max(0, min(2, rows - gr)) : 0;
        if (nvalid) src = X + (size_t)gk * ld + gr;
      } else {
        nvalid = (gr < rows) ? max(0, min(2, K - gk)) : 0;
        if (nvalid) src = X + (size_t)gr * ld + gk;
      }
      double *dst = TR ? S + r * DG_KROW + kk : S + kk * (BMN + DG_PAD) + r;
      cp_async16(dst, src, 8 * nvalid);
    }
    return;
  }
  for (int e = threadIdx.x; e < E; e += NT) {
    int r, kk;
    if (!TR) {
      r = e % BMN;
      kk = e / BMN;
    } else {
      kk = e % DG_BK;
      r = e / DG_BK;
    }
    const int gr = r0 + r, gk = k0 + kk;
    const bool ok = gr < rows && gk < K;
    const double *src = X;
    if (ok) src = TR ? X + (size_t)gr * ld + gk : X + (size_t)gk * ld + gr;
    double *dst = TR ? S + r * DG_KROW + kk : S + kk * (BMN + DG_PAD) + r;
    cp_async8(dst, src, ok);
  }
}

// fragment value op(X)[r][kk] from the staged tile
template <int BMN, bool TR>
__device__ __forceinline__ double frag(const double *S, int r, int kk) {
  return TR ? S[r * DG_KROW + kk] : S[kk * (BMN + DG_PAD) + r];
}

struct DgemmArgs {
  int m, n, k;
  double alpha, beta;
  const double *A;
  int lda;
  const double *B;
  int ldb;
  double *C;
  int ldc;
  int vecA, vecB;      // 16-byte copies possible (aligned base, even leading dimension)
  int kslices;         // > 1: partial tiles to ws[slice][n][m] (column-major, ld m)
  int kchunk;          // K per slice (multiple of BK)
  double *ws;
};

// TA: op(A) = A^T; TB: op(B) = B^T.  op(B)[kk][j] is B[kk + j*ldb] (TB = false:
// contiguous along kk, the "TR" layout of an operand indexed [j][kk]) or
// B[j + kk*ldb] (TB = true: contiguous along j).
template <int BM, int BN, int WM, int WN, bool TA, bool TB>
__global__ void __launch_bounds__(WM *WN * 32, 1) k_dgemm(DgemmArgs g) {
  constexpr int NT = WM * WN * 32;
  constexpr int TM = BM / WM, TN = BN / WN;         // warp tile
  constexpr int MT = TM / 8, NTL = TN / 8;           // 8 x 8 MMA tiles per warp
  constexpr int SA = tile_elems<BM>(), SB = tile_elems<BN>();
  extern __shared__ double sm[];
  double *sA = sm, *sB = sm + DG_STAGES * SA;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = warp / WN, wn = warp % WN;
  const int grp = lane >> 2, tig = lane & 3;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int slice = blockIdx.z;
  const int kbeg = slice * g.kchunk;
  const int kend = min(g.k, kbeg + g.kchunk);
  const int nkt = kend > kbeg ? (kend - kbeg + DG_BK - 1) / DG_BK : 0;

  double acc[MT][NTL][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NTL; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  // A operand indexed [row m][kk]: TA = false -> A[m + kk*lda] (contiguous along m)
  // B operand indexed [col n][kk]: TB = false -> B[kk + n*ldb] (contiguous along kk)
  auto load_stage = [&](int st, int kt) {
    const int k0 = kbeg + kt * DG_BK;
    load_tile<BM, NT, TA>(sA + st * SA, g.A, g.lda, m0, g.m, k0, kend, g.vecA != 0);
    load_tile<BN, NT, !TB>(sB + st * SB, g.B, g.ldb, n0, g.n, k0, kend, g.vecB != 0);
  };
#pragma unroll
  for (int st = 0; st < DG_STAGES - 1; ++st) {
    if (st < nkt) load_stage(st, st);
    cp_async_commit();
  }
  for (int kt = 0; kt < nkt; ++kt) {
    cp_async_wait<DG_STAGES - 2>();
    __syncthreads();
    // refill the stage consumed in the previous iteration
    const int nxt = kt + DG_STAGES - 1;
    if (nxt < nkt) load_stage(nxt % DG_STAGES, nxt);
    cp_async_commit();
    const double *cA = sA + (kt % DG_STAGES) * SA;
    const double *cB = sB + (kt % DG_STAGES) * SB;
#pragma unroll
    for (int k4 = 0; k4 < DG_BK; k4 += 4) {
      double af[MT], bf[NTL];
#pragma unroll
      for (int i = 0; i < MT; ++i) af[i] = frag<BM, TA>(cA, wm * TM + i * 8 + grp, k4 + tig);
#pragma unroll
      for (int j = 0; j < NTL; ++j) bf[j] = frag<BN, !TB>(cB, wn * TN + j * 8 + grp, k4 + tig);
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NTL; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();
  // epilogue: element (row grp, cols 2 tig, 2 tig + 1) of each 8 x 8 tile
#pragma unroll
  for (int i = 0; i < MT; ++i) {
    const int r = m0 + wm * TM + i * 8 + grp;
    if (r >= g.m) continue;
#pragma unroll
    for (int j = 0; j < NTL; ++j) {
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int c = n0 + wn * TN + j * 8 + 2 * tig + u;
        if (c >= g.n) continue;
        if (g.kslices > 1) {
          g.ws[((size_t)slice * g.n + c) * g.m + r] = acc[i][j][u];
        } else {
          double *cp = g.C + (size_t)c * g.ldc + r;
          const double v = g.alpha * acc[i][j][u];
          *cp = (g.beta == 0.0) ? v : v + g.beta * *cp;
        }
      }
    }
  }
}

// C = alpha * sum_s ws[s] + beta * C, slices summed in order
__global__ void k_dgemm_slices(const double *__restrict__ ws, int S, int m, int n, double alpha, double beta,
                               double *__restrict__ C, int ldc) {
  const size_t total = (size_t)m * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int s = 0; s < S; ++s) t += ws[(size_t)s * total + e];
    const int r = (int)(e % m), c = (int)(e / m);
    double *cp = C + (size_t)c * ldc + r;
    const double v = alpha * t;
    *cp = (beta == 0.0) ? v : v + beta * *cp;
  }
}

template <int BM, int BN, int WM, int WN, bool TA, bool TB>
cudaError_t launch_cfg(const DgemmArgs &a, cudaStream_t st) {
  constexpr int smem = DG_STAGES * (tile_elems<BM>() + tile_elems<BN>()) * 8;
  static std::atomic<unsigned long long> done{0};
  cudaError_t e = smem_limit_once(k_dgemm<BM, BN, WM, WN, TA, TB>, smem, done);
  if (e != cudaSuccess) return e;
  dim3 grid((a.m + BM - 1) / BM, (a.n + BN - 1) / BN, a.kslices);
  k_dgemm<BM, BN, WM, WN, TA, TB><<<grid, WM * WN * 32, smem, st>>>(a);
  return cudaGetLastError();
}

template <int BM, int BN, int WM, int WN>
cudaError_t launch_trans(const DgemmArgs &a, bool ta, bool tb, cudaStream_t st) {
  if (!ta && !tb) return launch_cfg<BM, BN, WM, WN, false, false>(a, st);
  if (ta && !tb) return launch_cfg<BM, BN, WM, WN, true, false>(a, st);
  if (!ta && tb) return launch_cfg<BM, BN, WM, WN, false, true>(a, st);
  return launch_cfg<BM, BN, WM, WN, true, true>(a, st);
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

}  // namespace

size_t dgemm_ws_bytes(int m, int n, int k) {
  // the largest split dgemm() may choose: up to 64 slices
  (void)k;
  return (size_t)64 * m * n * sizeof(double);
}

cudaError_t dgemm(cudaStream_t st, bool ta, bool tb, int m, int n, int k, double alpha, const double *A,
                  int lda, const double *B, int ldb, double beta, double *C, int ldc, double *ws,
                  size_t ws_bytes) {
  if (m <= 0 || n <= 0) return cudaSuccess;
  DgemmArgs a{};
  a.m = m;
  a.n = n;
  a.k = std::max(k, 0);
  a.alpha = alpha;
  a.beta = beta;
  a.A = A;
  a.lda = lda;
  a.B = B;
  a.ldb = ldb;
  a.C = C;
  a.ldc = ldc;
  a.kslices = 1;
  a.kchunk = std::max(a.k, 1);
  a.vecA = ((reinterpret_cast<uintptr_t>(A) & 15) == 0 && (lda & 1) == 0) ? 1 : 0;
  a.vecB = ((reinterpret_cast<uintptr_t>(B) & 15) == 0 && (ldb & 1) == 0) ? 1 : 0;
  const int nsm = sm_count();
  const long long big_tiles = (long long)((m + 127) / 128) * ((n + 127) / 128);
  if (big_tiles >= 2LL * nsm) return launch_trans<128, 128, 2, 4>(a, ta, tb, st);
  // small tile grid: 64 x 64 tiles, and split K when even those leave SMs idle
  const long long tiles = (long long)((m + 63) / 64) * ((n + 63) / 64);
  int S = 1;
  if (ws && a.k >= 8 * DG_BK && tiles < 2LL * nsm) {
    S = (int)std::min<long long>(64, (2LL * nsm + tiles - 1) / tiles);
    S = std::min(S, a.k / (4 * DG_BK));
    while (S > 1 && (size_t)S * m * n * sizeof(double) > ws_bytes) --S;
  }
  if (S > 1) {
    a.kslices = S;
    a.kchunk = ((a.k + S - 1) / S + DG_BK - 1) / DG_BK * DG_BK;
    a.kslices = (a.k + a.kchunk - 1) / a.kchunk;
    a.ws = ws;
    cudaError_t e = launch_trans<64, 64, 2, 2>(a, ta, tb, st);
    if (e != cudaSuccess) return e;
    const size_t total = (size_t)m * n;
    const int blocks = (int)std::min<size_t>((total + 255) / 256, 4096);
    k_dgemm_slices<<<blocks, 256, 0, st>>>(ws, a.kslices, m, n, alpha, beta, C, ldc);
    return cudaGetLastError();
  }
  return launch_trans<64, 64, 2, 2>(a, ta, tb, st);
}

}  // namespace ngw

// Measurement entry (no reference counterpart): C = op(A) op(B) on device
// pointers, for the GEMM tests and the profile of the FP64 tensor path.
extern "C" int ngw_dgemm(int transa, int transb, int m, int n, int k, double alpha, const double *A, int lda,
                         const double *B, int ldb, double beta, double *C, int ldc, double *ws,
                         long long ws_bytes, void *stream) {
  using namespace ngw;
  if (m < 0 || n < 0 || k < 0 || !A || !B || !C || lda < 1 || ldb < 1 || ldc < std::max(1, m) ||
      lda < (transa ? k : m) || ldb < (transb ? n : k) || ws_bytes < 0) {
    set_error("ngw_dgemm: bad arguments");
    return NGW_ERR_ARG;
  }
  NGW_CUDA(dgemm(static_cast<cudaStream_t>(stream), transa != 0, transb != 0, m, n, k, alpha, A, lda, B, ldb,
                 beta, C, ldc, ws, (size_t)ws_bytes));
  return NGW_OK;
}

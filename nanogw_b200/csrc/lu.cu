// LU factorisation with partial pivoting and the solve with many right-hand
// sides, on the device, for the ISDF fit's A Z = B
// (shared/isdf_parallel_sym_UltraLowMem.F90:617/:629, pdgesv).
//
// Factorisation (right-looking, panels of LU_NB columns):
//   1. the panel A[j:n, j:j+NB) is factorised by one CTA: for each column the
//      first row of largest |value| is the pivot (as LAPACK's idamax), the
//      whole row pair is swapped (all n columns), the column is scaled and
//      the panel's remaining columns get the rank-1 update;
//   2. U12 = L11^{-1} A12 by a triangular-solve kernel (one thread per column,
//      L11 in shared memory);
//   3. A22 -= L21 U12 by the FP64 tensor-core GEMM.
// Solve: the row interchanges gathered in one pass (the composed
// permutation), then forward substitution with L and back substitution with U
// in blocks of LU_NB rows: a triangular-solve kernel per diagonal block and
// an FP64 GEMM for the rest of the right-hand side.  Deterministic.
#include <algorithm>
#include <vector>

#include "ngw_internal.h"

namespace ngw {

namespace {

constexpr int LU_NB = 64;
constexpr int LU_PT = 1024;   // threads of the panel kernel

// Panel j0 .. j0+nb-1 of the n x n matrix A (column-major, lda).  ipiv gets
// 0-based pivot rows; info (first singular column + 1) is set when a pivot
// is exactly zero (the factorisation continues, as LAPACK's does).
__global__ void __launch_bounds__(LU_PT) k_lu_panel(double *__restrict__ A, int lda, int n, int j0, int nb,
                                                     int *__restrict__ ipiv, int *__restrict__ info) {
  __shared__ double sv[LU_PT / 32];
  __shared__ int si[LU_PT / 32];
  __shared__ int piv_sh;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int c = j0; c < j0 + nb; ++c) {
    // pivot: the first row of largest |A(r, c)|, r >= c
    double best = -1.0;
    int bi = n;
    for (int r = c + tid; r < n; r += LU_PT) {
      const double v = fabs(A[(size_t)c * lda + r]);
      if (v > best) {
        best = v;
        bi = r;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if (lane == 0) {
      sv[warp] = best;
      si[warp] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      double bv = sv[0];
      int bidx = si[0];
      for (int q = 1; q < LU_PT / 32; ++q)
        if (sv[q] > bv || (sv[q] == bv && si[q] < bidx)) {
          bv = sv[q];
          bidx = si[q];
        }
      if (bidx >= n) bidx = c;
      piv_sh = bidx;
      ipiv[c] = bidx;
      if (bv == 0.0 && *info == 0) *info = c + 1;
    }
    __syncthreads();
    const int p = piv_sh;
    if (p != c)
      for (int q = tid; q < n; q += LU_PT) {
        double *a = A + (size_t)q * lda;
        const double t = a[c];
        a[c] = a[p];
        a[p] = t;
      }
    __syncthreads();
    const double d = A[(size_t)c * lda + c];
    const double inv = d != 0.0 ? 1.0 / d : 0.0;
    for (int r = c + 1 + tid; r < n; r += LU_PT) A[(size_t)c * lda + r] *= inv;
    __syncthreads();
    // rank-1 update of the panel's later columns
    const int ncol = j0 + nb - c - 1;
    const int nrow = n - c - 1;
    for (size_t e = tid; e < (size_t)ncol * nrow; e += LU_PT) {
      const int cc = c + 1 + (int)(e / nrow), r = c + 1 + (int)(e % nrow);
      A[(size_t)cc * lda + r] -= A[(size_t)c * lda + r] * A[(size_t)cc * lda + c];
    }
    __syncthreads();
  }
}

// X (nb x ncol block, leading dimension ldx) = L^{-1} X with L the unit lower
// triangle (lower = true) or U^{-1} X with U the upper triangle, of the
// nb x nb diagonal block T (leading dimension ldt).  One thread per column
// of X, the block of T in shared memory.
template <bool LOWER>
__global__ void __launch_bounds__(128) k_trsm_block(const double *__restrict__ T, int ldt, int nb,
                                                     double *__restrict__ X, int ldx, int ncol) {
  __shared__ double sT[LU_NB * LU_NB];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) sT[e] = T[(size_t)(e / nb) * ldt + (e % nb)];
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  double x[LU_NB];
  double *xc = X + (size_t)col * ldx;
#pragma unroll
  for (int r = 0; r < LU_NB; ++r) x[r] = r < nb ? xc[r] : 0.0;
  if (LOWER) {
#pragma unroll
    for (int r = 0; r < LU_NB; ++r) {
      if (r >= nb) break;
      double t = x[r];
#pragma unroll
      for (int q = 0; q < r; ++q) t -= sT[q * nb + r] * x[q];
      x[r] = t;
    }
  } else {
#pragma unroll
    for (int r = LU_NB - 1; r >= 0; --r) {
      if (r >= nb) continue;
      double t = x[r];
#pragma unroll
      for (int q = r + 1; q < LU_NB; ++q)
        if (q < nb) t -= sT[q * nb + r] * x[q];
      x[r] = t / sT[r * nb + r];
    }
  }
#pragma unroll
  for (int r = 0; r < LU_NB; ++r)
    if (r < nb) xc[r] = x[r];
}

// out(i, c) = B(perm[i], c)
__global__ void k_row_gather(const double *__restrict__ B, int ldb, const int *__restrict__ perm, int n, int ncol,
                             double *__restrict__ out) {
  const size_t total = (size_t)n * ncol;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), c = (int)(e / n);
    out[e] = B[(size_t)c * ldb + perm[i]];
  }
}

}  // namespace

// A (n x n, lda) is overwritten by L\U; hipiv (host, n) gets the 0-based
// pivot rows in order.  NGW_ERR_ARG when a pivot is exactly zero.
int lu_factor(ngw_session *s, int n, double *A, int lda, std::vector<int> &hipiv) {
  int *dpiv = nullptr;
  NGW_TRY(dalloc(s, (void **)&dpiv, (size_t)(n + 1) * 4));
  int *dinfo = dpiv + n;
  int rc = NGW_OK;
  do {
    if (cudaMemsetAsync(dinfo, 0, 4, s->stream) != cudaSuccess) {
      rc = NGW_ERR_CUDA;
      break;
    }
    for (int j = 0; j < n && rc == NGW_OK; j += LU_NB) {
      const int nb = std::min(LU_NB, n - j);
      k_lu_panel<<<1, LU_PT, 0, s->stream>>>(A, lda, n, j, nb, dpiv, dinfo);
      const int rest = n - j - nb;
      if (rest > 0) {
        double *a12 = A + (size_t)(j + nb) * lda + j;
        k_trsm_block<true><<<(rest + 127) / 128, 128, 0, s->stream>>>(A + (size_t)j * lda + j, lda, nb, a12, lda,
                                                                       rest);
        if (dgemm(s->stream, false, false, rest, rest, nb, -1.0, A + (size_t)j * lda + j + nb, lda, a12, lda, 1.0,
                  A + (size_t)(j + nb) * lda + j + nb, lda) != cudaSuccess)
          rc = NGW_ERR_CUDA;
      }
      if (cudaGetLastError() != cudaSuccess) rc = NGW_ERR_CUDA;
    }
    if (rc != NGW_OK) {
      set_error("LU factorisation kernels failed");
      break;
    }
    int hinfo = 0;
    hipiv.assign(n, 0);
    if (cudaMemcpyAsync(hipiv.data(), dpiv, (size_t)n * 4, cudaMemcpyDeviceToHost, s->stream) ||
        cudaMemcpyAsync(&hinfo, dinfo, 4, cudaMemcpyDeviceToHost, s->stream) || cudaStreamSynchronize(s->stream)) {
      set_error("LU factorisation failed to complete");
      rc = NGW_ERR_CUDA;
      break;
    }
    if (hinfo != 0) {
      set_error("LU factorisation: zero pivot in column %d (singular matrix)", hinfo);
      rc = NGW_ERR_ARG;
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, dpiv, (size_t)(n + 1) * 4);
  return rc;
}

// B (n x nrhs, ldb) = A^{-1} B from the factors of lu_factor; work holds
// n x nrhs doubles (the permuted right-hand side is built there and copied
// back into B at the end of the forward pass... solved in place in work,
// then copied to B).
int lu_solve(ngw_session *s, int n, int nrhs, const double *LU, int lda, const std::vector<int> &hipiv, double *B,
             int ldb, double *work) {
  // composed row permutation: row i of P B is row perm[i] of B
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  for (int i = 0; i < n; ++i) std::swap(perm[i], perm[hipiv[i]]);
  int *dperm = nullptr;
  NGW_TRY(dalloc(s, (void **)&dperm, (size_t)n * 4));
  int rc = NGW_OK;
  do {
    if (cudaMemcpyAsync(dperm, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s->stream)) {
      rc = NGW_ERR_CUDA;
      break;
    }
    k_row_gather<<<4096, 256, 0, s->stream>>>(B, ldb, dperm, n, nrhs, work);
    // forward: L y = P b (unit lower), blocks top to bottom
    for (int j = 0; j < n && rc == NGW_OK; j += LU_NB) {
      const int nb = std::min(LU_NB, n - j);
      k_trsm_block<true><<<(nrhs + 127) / 128, 128, 0, s->stream>>>(LU + (size_t)j * lda + j, lda, nb, work + j, n,
                                                                    nrhs);
      const int rest = n - j - nb;
      if (rest > 0 && dgemm(s->stream, false, false, rest, nrhs, nb, -1.0, LU + (size_t)j * lda + j + nb, lda,
                            work + j, n, 1.0, work + j + nb, n) != cudaSuccess)
        rc = NGW_ERR_CUDA;
    }
    // backward: U x = y, blocks bottom to top
    const int last = ((n - 1) / LU_NB) * LU_NB;
    for (int j = last; j >= 0 && rc == NGW_OK; j -= LU_NB) {
      const int nb = std::min(LU_NB, n - j);
      k_trsm_block<false><<<(nrhs + 127) / 128, 128, 0, s->stream>>>(LU + (size_t)j * lda + j, lda, nb, work + j,
                                                                     n, nrhs);
      if (j > 0 && dgemm(s->stream, false, false, j, nrhs, nb, -1.0, LU + (size_t)j * lda, lda, work + j, n, 1.0,
                         work, n) != cudaSuccess)
        rc = NGW_ERR_CUDA;
    }
    if (rc != NGW_OK || cudaGetLastError() != cudaSuccess) {
      set_error("LU solve kernels failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    if (cudaMemcpy2DAsync(B, (size_t)ldb * 8, work, (size_t)n * 8, (size_t)n * 8, nrhs, cudaMemcpyDeviceToDevice,
                          s->stream) != cudaSuccess) {
      set_error("LU solve copy-back failed");
      rc = NGW_ERR_CUDA;
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, dperm, (size_t)n * 4);
  return rc;
}

}  // namespace ngw

// ISDF fit on the device (shared/isdf_parallel_sym_UltraLowMem.F90:439-667, C1):
//   P(mu, r)  = sum_{v <= mv}   psi_v(r_mu) psi_v(r)      (dgemm_hl rank-1 loops :475-480)
//   Q(mu, r)  = sum_{c <= nmem} psi_c(r_mu) psi_c(r)      (:504-509)
//   A = P_intp * Q_intp (Hadamard, N_mu x N_mu)            (:574-576)
//   B = P * Q           (Hadamard, N_mu x N_grid)          (:585-587)
//   A Z = B  (LU with partial pivoting, pdgesv :617/:629); zeta = Z^T.
// P and Q products run on the FP64 tensor-core GEMM, the Hadamard products,
// the row gather and the transpose are kernels of this library, and the LU
// factorisation with partial pivoting and its solve are this library's own
// (lu.cu).
#include <algorithm>
#include <vector>

#include "ngw_internal.h"

namespace ngw {

// psi_intp(mu, b) = psi(intp(mu) - 1, b)   (column-major, ld ngrid / n_isdf)
__global__ void k_gather_rows(const double *__restrict__ psi, int ngrid, const int *__restrict__ intp,
                              int n_isdf, int nmem, double *__restrict__ out) {
  const int b = blockIdx.y;
  for (int mu = blockIdx.x * blockDim.x + threadIdx.x; mu < n_isdf; mu += gridDim.x * blockDim.x)
    out[(size_t)b * n_isdf + mu] = psi[(size_t)b * ngrid + (intp[mu] - 1)];
}

__global__ void k_hadamard(double *__restrict__ x, const double *__restrict__ y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = x[i] * y[i];
}

int lu_factor(ngw_session *s, int n, double *A, int lda, std::vector<int> &hipiv);
int lu_solve(ngw_session *s, int n, int nrhs, const double *LU, int lda, const std::vector<int> &hipiv, double *B,
             int ldb, double *work);

// out (cols x rows) = in^T for a column-major rows x cols matrix, through
// 32 x 32 shared-memory tiles (coalesced reads and writes)
__global__ void k_transpose(const double *__restrict__ in, int rows, int cols, double *__restrict__ out) {
  __shared__ double t[32][33];
  for (int c0 = blockIdx.y * 32; c0 < cols; c0 += gridDim.y * 32)
    for (int r0 = blockIdx.x * 32; r0 < rows; r0 += gridDim.x * 32) {
      for (int q = threadIdx.y; q < 32; q += blockDim.y) {
        const int r = r0 + threadIdx.x, c = c0 + q;
        if (r < rows && c < cols) t[q][threadIdx.x] = in[(size_t)c * rows + r];
      }
      __syncthreads();
      for (int q = threadIdx.y; q < 32; q += blockDim.y) {
        const int c = c0 + threadIdx.x, r = r0 + q;
        if (r < rows && c < cols) out[(size_t)r * cols + c] = t[threadIdx.x][q];
      }
      __syncthreads();
    }
}

void launch_transpose(const double *in, int rows, int cols, double *out, cudaStream_t st) {
  const dim3 grid((unsigned)std::min((rows + 31) / 32, 4096), (unsigned)std::min((cols + 31) / 32, 1024));
  k_transpose<<<grid, dim3(32, 8), 0, st>>>(in, rows, cols, out);
}

int isdf_fit_device(ngw_session *s, int ngrid, int nmem, const double *d_psi, const int *d_intp,
                    int n_isdf, int mv, double *d_psi_intp, double *d_zeta_t) {
  // d_zeta_t receives Z = zeta^T (n_isdf x ngrid, column-major)
  double *P = nullptr, *Q = nullptr, *Ai = nullptr, *Qi = nullptr;
  int rc = NGW_OK;
  const size_t pb = (size_t)n_isdf * ngrid * 8, ab = (size_t)n_isdf * n_isdf * 8;
  do {
    if (dalloc(s, (void **)&Q, pb) || dalloc(s, (void **)&Ai, ab) || dalloc(s, (void **)&Qi, ab)) {
      rc = NGW_ERR_OOM;
      break;
    }
    P = d_zeta_t;   // P is formed in the output buffer, then B = P * Q in place
    k_gather_rows<<<dim3((n_isdf + 255) / 256, nmem), 256, 0, s->stream>>>(d_psi, ngrid, d_intp, n_isdf,
                                                                           nmem, d_psi_intp);
    const double one = 1.0, zero = 0.0;
    // P = psi_intp[:, :mv] psi[:, :mv]^T ; Q = psi_intp psi^T (FP64 tensor-core GEMMs)
    if (dgemm(s->stream, false, true, n_isdf, ngrid, mv, one, d_psi_intp, n_isdf, d_psi, ngrid, zero, P,
              n_isdf) != cudaSuccess ||
        dgemm(s->stream, false, true, n_isdf, ngrid, nmem, one, d_psi_intp, n_isdf, d_psi, ngrid, zero, Q,
              n_isdf) != cudaSuccess ||
        dgemm(s->stream, false, true, n_isdf, n_isdf, mv, one, d_psi_intp, n_isdf, d_psi_intp, n_isdf, zero,
              Ai, n_isdf) != cudaSuccess ||
        dgemm(s->stream, false, true, n_isdf, n_isdf, nmem, one, d_psi_intp, n_isdf, d_psi_intp, n_isdf, zero,
              Qi, n_isdf) != cudaSuccess) {
      set_error("FP64 GEMM (ISDF P/Q products) failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    k_hadamard<<<2048, 256, 0, s->stream>>>(P, Q, (size_t)n_isdf * ngrid);
    k_hadamard<<<256, 256, 0, s->stream>>>(Ai, Qi, (size_t)n_isdf * n_isdf);
    if (cudaGetLastError() != cudaSuccess) {
      set_error("ISDF Hadamard kernels failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    // A Z = B: LU with partial pivoting, then the solve (Q is free again and
    // serves as its workspace)
    std::vector<int> piv;
    rc = lu_factor(s, n_isdf, Ai, n_isdf, piv);
    if (rc == NGW_ERR_ARG)
      set_error("ISDF matrix A is singular (zero pivot): duplicate interpolation points?");
    if (rc != NGW_OK) break;
    rc = lu_solve(s, n_isdf, ngrid, Ai, n_isdf, piv, P, n_isdf, Q);
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, Q, pb);
  dfree(s, Ai, ab);
  dfree(s, Qi, ab);
  return rc;
}

int coulomb_core(ngw_session *s, int ngrid, int n_isdf, const double *dz, const int *dg, int nfft,
                 double h, double trunc, double *dm);
int fxc_core(ngw_session *s, int ngrid, int n_isdf, const double *dz, const double *drho, double h,
             double *dm, double *dfxc);
int check_density(int ngrid, const double *rho, const char *who);

}  // namespace ngw

// Whole ISDF kernel on the device: orbitals on the grid and the (de-duplicated,
// 1-based) interpolation points in; Psi_intp, the Coulomb block and, when rho
// is given, the f_xc block out.  zeta never leaves the device: the fit writes
// zeta^T (N_mu x N_grid), one transpose gives the column layout the FFT-Poisson
// pack reads, and both kernel blocks are built from it.
extern "C" int ngw_build_isdf_kernel(ngw_session *s, int ngrid, int nmem, const double *psi,
                                     const int *grid_idx, int n_isdf, const int *intp, int mv, int nfft,
                                     double h, double trunc, const double *rho, double *psi_intp,
                                     double *mmtrx, double *mxc) {
  using namespace ngw;
  if (!s || ngrid <= 0 || nmem <= 0 || !psi || !grid_idx || n_isdf <= 0 || n_isdf > ngrid || !intp ||
      mv < 1 || mv > nmem || nfft < 4 || (nfft & 1) || h <= 0 || !psi_intp || !mmtrx || (rho && !mxc)) {
    set_error("ngw_build_isdf_kernel: bad arguments");
    return NGW_ERR_ARG;
  }
  for (int i = 0; i < n_isdf; ++i)
    if (intp[i] < 1 || intp[i] > ngrid) {
      set_error("ngw_build_isdf_kernel: point index %d out of range", intp[i]);
      return NGW_ERR_ARG;
    }
  {
    // a repeated point gives two equal rows of A
    std::vector<int> sorted(intp, intp + n_isdf);
    std::sort(sorted.begin(), sorted.end());
    for (int i = 1; i < n_isdf; ++i)
      if (sorted[i] == sorted[i - 1]) {
        set_error("ngw_build_isdf_kernel: grid point %d appears twice among the interpolation points",
                  sorted[i]);
        return NGW_ERR_ARG;
      }
  }
  if (rho)
    if (int e = check_density(ngrid, rho, "ngw_build_isdf_kernel")) return e;
  NGW_CUDA(cudaSetDevice(s->device));
  double *dpsi = nullptr, *dpi = nullptr, *dzt = nullptr, *dz = nullptr, *dm = nullptr, *drho = nullptr,
         *dfxc = nullptr;
  int *dintp = nullptr, *dg = nullptr;
  const size_t psib = (size_t)ngrid * nmem * 8, zb = (size_t)n_isdf * ngrid * 8,
               mb = (size_t)n_isdf * n_isdf * 8, pib = (size_t)n_isdf * nmem * 8;
  int rc = NGW_OK;
  do {
    if (dalloc(s, (void **)&dpsi, psib) || dalloc(s, (void **)&dpi, pib) || dalloc(s, (void **)&dzt, zb) ||
        dalloc(s, (void **)&dm, mb) || dalloc(s, (void **)&dintp, (size_t)n_isdf * 4)) {
      rc = NGW_ERR_OOM;
      break;
    }
    if (cudaMemcpyAsync(dpsi, psi, psib, cudaMemcpyHostToDevice, s->stream) ||
        cudaMemcpyAsync(dintp, intp, (size_t)n_isdf * 4, cudaMemcpyHostToDevice, s->stream)) {
      set_error("copy to device failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    rc = isdf_fit_device(s, ngrid, nmem, dpsi, dintp, n_isdf, mv, dpi, dzt);
    if (rc != NGW_OK) break;
    dfree(s, dpsi, psib);   // orbitals are not needed past the fit
    dpsi = nullptr;
    if (dalloc(s, (void **)&dz, zb) || dalloc(s, (void **)&dg, (size_t)3 * ngrid * 4)) {
      rc = NGW_ERR_OOM;
      break;
    }
    launch_transpose(dzt, n_isdf, ngrid, dz, s->stream);
    if (cudaGetLastError() != cudaSuccess) {
      set_error("zeta transpose failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    if (cudaMemcpyAsync(dg, grid_idx, (size_t)3 * ngrid * 4, cudaMemcpyHostToDevice, s->stream) ||
        cudaStreamSynchronize(s->stream)) {
      set_error("copy to device failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    dfree(s, dzt, zb);
    dzt = nullptr;
    rc = coulomb_core(s, ngrid, n_isdf, dz, dg, nfft, h, trunc, dm);
    if (rc != NGW_OK) break;
    if (cudaMemcpyAsync(psi_intp, dpi, pib, cudaMemcpyDeviceToHost, s->stream) ||
        cudaMemcpyAsync(mmtrx, dm, mb, cudaMemcpyDeviceToHost, s->stream) || cudaStreamSynchronize(s->stream)) {
      set_error("copy back failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    if (rho) {
      if (dalloc(s, (void **)&drho, (size_t)ngrid * 8) || dalloc(s, (void **)&dfxc, (size_t)ngrid * 8)) {
        rc = NGW_ERR_OOM;
        break;
      }
      if (cudaMemcpyAsync(drho, rho, (size_t)ngrid * 8, cudaMemcpyHostToDevice, s->stream)) {
        set_error("copy to device failed");
        rc = NGW_ERR_CUDA;
        break;
      }
      rc = fxc_core(s, ngrid, n_isdf, dz, drho, h, dm, dfxc);
      if (rc != NGW_OK) break;
      if (cudaMemcpyAsync(mxc, dm, mb, cudaMemcpyDeviceToHost, s->stream) || cudaStreamSynchronize(s->stream)) {
        set_error("copy back failed");
        rc = NGW_ERR_CUDA;
        break;
      }
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  if (dpsi) dfree(s, dpsi, psib);
  if (dzt) dfree(s, dzt, zb);
  dfree(s, dpi, pib);
  dfree(s, dz, zb);
  dfree(s, dm, mb);
  dfree(s, dintp, (size_t)n_isdf * 4);
  dfree(s, dg, (size_t)3 * ngrid * 4);
  dfree(s, drho, (size_t)ngrid * 8);
  dfree(s, dfxc, (size_t)ngrid * 8);
  return rc;
}

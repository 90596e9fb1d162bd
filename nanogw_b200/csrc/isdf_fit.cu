// ISDF fit on the device (shared/isdf_parallel_sym_UltraLowMem.F90:439-667, C1):
//   P(mu, r)  = sum_{v <= mv}   psi_v(r_mu) psi_v(r)      (dgemm_hl rank-1 loops :475-480)
//   Q(mu, r)  = sum_{c <= nmem} psi_c(r_mu) psi_c(r)      (:504-509)
//   A = P_intp * Q_intp (Hadamard, N_mu x N_mu)            (:574-576)
//   B = P * Q           (Hadamard, N_mu x N_grid)          (:585-587)
//   A Z = B  (LU with partial pivoting, pdgesv :617/:629); zeta = Z^T.
// P and Q products are cuBLAS DGEMMs, the Hadamard products and the row
// gather are kernels of this library, the LU is cuSOLVER getrf/getrs.
#include <cusolverDn.h>

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

int isdf_fit_device(ngw_session *s, int ngrid, int nmem, const double *d_psi, const int *d_intp,
                    int n_isdf, int mv, double *d_psi_intp, double *d_zeta_t) {
  // d_zeta_t receives Z = zeta^T (n_isdf x ngrid, column-major)
  double *P = nullptr, *Q = nullptr, *Ai = nullptr, *Qi = nullptr, *work = nullptr;
  int *ipiv = nullptr, *info = nullptr;
  cusolverDnHandle_t sol = nullptr;
  void *hv = nullptr;
  int rc = NGW_OK;
  const size_t pb = (size_t)n_isdf * ngrid * 8, ab = (size_t)n_isdf * n_isdf * 8;
  int lwork = 0;
  do {
    if (dalloc(s, (void **)&Q, pb) || dalloc(s, (void **)&Ai, ab) || dalloc(s, (void **)&Qi, ab) ||
        dalloc(s, (void **)&ipiv, (size_t)n_isdf * 4) || dalloc(s, (void **)&info, 4)) {
      rc = NGW_ERR_OOM;
      break;
    }
    P = d_zeta_t;   // P is formed in the output buffer, then B = P * Q in place
    k_gather_rows<<<dim3((n_isdf + 255) / 256, nmem), 256, 0, s->stream>>>(d_psi, ngrid, d_intp, n_isdf,
                                                                           nmem, d_psi_intp);
    const double one = 1.0, zero = 0.0;
    // P = psi_intp[:, :mv] psi[:, :mv]^T ; Q = psi_intp psi^T
    if (cublasDgemm(s->cublas, CUBLAS_OP_N, CUBLAS_OP_T, n_isdf, ngrid, mv, &one, d_psi_intp, n_isdf, d_psi,
                    ngrid, &zero, P, n_isdf) != CUBLAS_STATUS_SUCCESS ||
        cublasDgemm(s->cublas, CUBLAS_OP_N, CUBLAS_OP_T, n_isdf, ngrid, nmem, &one, d_psi_intp, n_isdf, d_psi,
                    ngrid, &zero, Q, n_isdf) != CUBLAS_STATUS_SUCCESS ||
        cublasDgemm(s->cublas, CUBLAS_OP_N, CUBLAS_OP_T, n_isdf, n_isdf, mv, &one, d_psi_intp, n_isdf,
                    d_psi_intp, n_isdf, &zero, Ai, n_isdf) != CUBLAS_STATUS_SUCCESS ||
        cublasDgemm(s->cublas, CUBLAS_OP_N, CUBLAS_OP_T, n_isdf, n_isdf, nmem, &one, d_psi_intp, n_isdf,
                    d_psi_intp, n_isdf, &zero, Qi, n_isdf) != CUBLAS_STATUS_SUCCESS) {
      set_error("cublasDgemm (ISDF P/Q products) failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    k_hadamard<<<2048, 256, 0, s->stream>>>(P, Q, (size_t)n_isdf * ngrid);
    k_hadamard<<<256, 256, 0, s->stream>>>(Ai, Qi, (size_t)n_isdf * n_isdf);
    if ((rc = session_cusolver(s, &hv)) != NGW_OK) break;
    sol = (cusolverDnHandle_t)hv;
    if (cusolverDnDgetrf_bufferSize(sol, n_isdf, n_isdf, Ai, n_isdf, &lwork) != CUSOLVER_STATUS_SUCCESS ||
        dalloc(s, (void **)&work, (size_t)std::max(lwork, 1) * 8)) {
      set_error("getrf workspace failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    if (cusolverDnDgetrf(sol, n_isdf, n_isdf, Ai, n_isdf, work, ipiv, info) != CUSOLVER_STATUS_SUCCESS ||
        cusolverDnDgetrs(sol, CUBLAS_OP_N, n_isdf, ngrid, Ai, n_isdf, ipiv, P, n_isdf, info) !=
            CUSOLVER_STATUS_SUCCESS) {
      set_error("cusolver getrf/getrs failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    int hinfo = 0;
    if (cudaMemcpyAsync(&hinfo, info, 4, cudaMemcpyDeviceToHost, s->stream) ||
        cudaStreamSynchronize(s->stream)) {
      set_error("ISDF solve failed to complete");
      rc = NGW_ERR_CUDA;
      break;
    }
    if (hinfo != 0) {
      set_error("ISDF matrix A is singular (getrf info %d): duplicate interpolation points?", hinfo);
      rc = NGW_ERR_ARG;
      break;
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, Q, pb);
  dfree(s, Ai, ab);
  dfree(s, Qi, ab);
  dfree(s, ipiv, (size_t)n_isdf * 4);
  dfree(s, info, 4);
  if (work) dfree(s, work, (size_t)std::max(lwork, 1) * 8);
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
    const double one = 1.0, zero = 0.0;
    if (cublasDgeam(s->cublas, CUBLAS_OP_T, CUBLAS_OP_T, ngrid, n_isdf, &one, dzt, n_isdf, &zero, dzt, n_isdf,
                    dz, ngrid) != CUBLAS_STATUS_SUCCESS) {
      set_error("cublasDgeam (zeta transpose) failed");
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

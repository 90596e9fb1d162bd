// Bare exchange Sigma_x (SIGMA/fock_exchange.F90z:16-228) and V_xc matrix
// elements (SIGMA/vxc.F90z:147-165, shared/vxcmtxel.F90z) on the device, for
// one spin, one k-point, C1 symmetry, real orbitals, finite system.
//
// Sigma_x: for every (m2 in the Sigma bands, n <= maxv) the pair density
// psi_n psi_m2 goes through the FFT-Poisson solve of poisson.cu, is multiplied
// by psi_n, and one DGEMM projects a chunk of such columns on every psi_m1:
//   K_x(m1, m2) = -(ntrans / hcub) sum_n occ_n <psi_m1 | psi_n V_c[psi_n psi_m2]>
// accumulated over n in increasing order for each m2 (the reference's loop
// order), m1 <= m2, then mirrored.  maxv is the highest state with
// occ > tol_occ = 0.01 (shared/myconstants.F90:51).
// V_xc: v_x = 2 v_x^LDA(rho), v_c = 2 v_c^PZ(rho) (Rydberg,
// shared/xc_module.F90:523-829), V(m1, m2) = ntrans <psi_m1 | v | psi_m2> by
// DGEMM over the grid.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ngw_internal.h"
#include "xc_lda.cuh"

namespace ngw {

int poisson_apply(ngw_session *s, int ngrid, int ncol, const double *drho, const int *dg, int nfft,
                  double h, double trunc, double *dv);
int check_density(int ngrid, const double *rho, const char *who);

// out(:, c) = psi(:, a[c]) * psi(:, b[c])   (1-based bands, ld ngrid)
__global__ void k_grid_pair_cols(const double *__restrict__ psi, int ngrid, const int *__restrict__ a,
                                 const int *__restrict__ b, int ncol, double *__restrict__ out) {
  for (int c = blockIdx.y; c < ncol; c += gridDim.y) {
    const double *pa = psi + (size_t)(a[c] - 1) * ngrid;
    const double *pb = psi + (size_t)(b[c] - 1) * ngrid;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ngrid; i += gridDim.x * blockDim.x)
      out[(size_t)c * ngrid + i] = pa[i] * pb[i];
  }
}

// w(:, c) *= psi(:, a[c])
__global__ void k_grid_mul_band(double *__restrict__ w, const double *__restrict__ psi, int ngrid,
                                const int *__restrict__ a, int ncol) {
  for (int c = blockIdx.y; c < ncol; c += gridDim.y) {
    const double *pa = psi + (size_t)(a[c] - 1) * ngrid;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ngrid; i += gridDim.x * blockDim.x)
      w[(size_t)c * ngrid + i] *= pa[i];
  }
}

// LDA exchange and correlation potentials in Rydberg (vx_get / vxc_get x 2)
__global__ void k_lda_potentials(const double *__restrict__ rho, int n, double *__restrict__ vx,
                                 double *__restrict__ vc) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    vx[i] = 2.0 * slater_vx(rho[i]);
    vc[i] = 2.0 * pz_vc(rho[i]);
  }
}

// w(:, j) = v .* p(:, j)
__global__ void k_grid_scale_cols(const double *__restrict__ p, const double *__restrict__ v, int ngrid,
                                  int ncol, double *__restrict__ w) {
  for (int c = blockIdx.y; c < ncol; c += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ngrid; i += gridDim.x * blockDim.x)
      w[(size_t)c * ngrid + i] = v[i] * p[(size_t)c * ngrid + i];
}

static int check_bands(int nsig, const int *sig, int nmem, const char *who) {
  for (int i = 0; i < nsig; ++i)
    if (sig[i] < 1 || sig[i] > nmem) {
      set_error("%s: band %d out of 1..%d", who, sig[i], nmem);
      return NGW_ERR_ARG;
    }
  return NGW_OK;
}

}  // namespace ngw

using namespace ngw;

extern "C" int ngw_fock_exchange(ngw_session *s, int ngrid, int nmem, const double *psi, const int *grid_idx,
                                 int nfft, double h, double trunc, const double *occ, int nsig,
                                 const int *sig_bands, int ntrans, double *kx) {
  if (!s || ngrid <= 0 || nmem <= 0 || !psi || !grid_idx || nfft < 4 || (nfft & 1) || h <= 0 || !occ ||
      nsig <= 0 || !sig_bands || ntrans < 1 || !kx) {
    set_error("ngw_fock_exchange: bad arguments");
    return NGW_ERR_ARG;
  }
  NGW_TRY(check_bands(nsig, sig_bands, nmem, "ngw_fock_exchange"));
  int maxv = 0;
  for (int i = 0; i < nmem; ++i)
    if (occ[i] > 0.01) maxv = i + 1;
  std::fill(kx, kx + (size_t)nsig * nsig, 0.0);
  if (maxv == 0) return NGW_OK;
  NGW_CUDA(cudaSetDevice(s->device));
  const size_t psib = (size_t)ngrid * nmem * 8;
  const int total = nsig * maxv;
  const int chunk = std::min(total, 256);
  double *dpsi = nullptr, *dps = nullptr, *drho = nullptr, *dv = nullptr, *dg2 = nullptr, *dws = nullptr;
  int *dg = nullptr, *dab = nullptr;
  int rc = NGW_OK;
  const double fac = (double)ntrans / (h * h * h);
  std::vector<double> g((size_t)nsig * chunk);
  std::vector<int> hab(2 * chunk);
  do {
    if (dalloc(s, (void **)&dpsi, psib) || dalloc(s, (void **)&dps, (size_t)ngrid * nsig * 8) ||
        dalloc(s, (void **)&drho, (size_t)ngrid * chunk * 8) || dalloc(s, (void **)&dv, (size_t)ngrid * chunk * 8) ||
        dalloc(s, (void **)&dg2, (size_t)nsig * chunk * 8) || dalloc(s, (void **)&dg, (size_t)3 * ngrid * 4) ||
        dalloc(s, (void **)&dab, (size_t)2 * chunk * 4) ||
        dalloc(s, (void **)&dws, dgemm_ws_bytes(nsig, chunk, ngrid))) {
      rc = NGW_ERR_OOM;
      break;
    }
    if (cudaMemcpyAsync(dpsi, psi, psib, cudaMemcpyHostToDevice, s->stream) ||
        cudaMemcpyAsync(dg, grid_idx, (size_t)3 * ngrid * 4, cudaMemcpyHostToDevice, s->stream)) {
      set_error("copy to device failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    for (int j = 0; j < nsig && rc == NGW_OK; ++j)
      if (cudaMemcpyAsync(dps + (size_t)j * ngrid, dpsi + (size_t)(sig_bands[j] - 1) * ngrid, (size_t)ngrid * 8,
                          cudaMemcpyDeviceToDevice, s->stream)) {
        set_error("band gather failed");
        rc = NGW_ERR_CUDA;
      }
    const int bx = std::min(256, (ngrid + 255) / 256);
    for (int c0 = 0; c0 < total && rc == NGW_OK; c0 += chunk) {
      const int nc = std::min(chunk, total - c0);
      // column c0 + c = (jj, n): n fastest, as the reference's icol
      for (int c = 0; c < nc; ++c) {
        const int icol = c0 + c, jj = icol / maxv, nn = icol % maxv;
        hab[c] = nn + 1;
        hab[chunk + c] = sig_bands[jj];
      }
      if (cudaMemcpyAsync(dab, hab.data(), (size_t)2 * chunk * 4, cudaMemcpyHostToDevice, s->stream)) {
        set_error("copy to device failed");
        rc = NGW_ERR_CUDA;
        break;
      }
      k_grid_pair_cols<<<dim3(bx, ygrid(nc)), 256, 0, s->stream>>>(dpsi, ngrid, dab, dab + chunk, nc, drho);
      if ((rc = poisson_apply(s, ngrid, nc, drho, dg, nfft, h, trunc, dv)) != NGW_OK) break;
      k_grid_mul_band<<<dim3(bx, ygrid(nc)), 256, 0, s->stream>>>(dv, dpsi, ngrid, dab, nc);
      const double one = 1.0, zero = 0.0;
      if (dgemm(s->stream, true, false, nsig, nc, ngrid, one, dps, ngrid, dv, ngrid, zero, dg2, nsig, dws,
                dgemm_ws_bytes(nsig, chunk, ngrid)) != cudaSuccess) {
        set_error("FP64 GEMM (exchange projection) failed");
        rc = NGW_ERR_CUDA;
        break;
      }
      if (cudaMemcpyAsync(g.data(), dg2, (size_t)nsig * nc * 8, cudaMemcpyDeviceToHost, s->stream) ||
          cudaStreamSynchronize(s->stream)) {
        set_error("copy back failed");
        rc = NGW_ERR_CUDA;
        break;
      }
      for (int c = 0; c < nc; ++c) {
        const int icol = c0 + c, jj = icol / maxv, nn = icol % maxv;
        const double w = -fac * occ[nn];
        for (int ii = 0; ii <= jj; ++ii) kx[ii + (size_t)jj * nsig] += g[ii + (size_t)c * nsig] * w;
      }
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, dpsi, psib);
  dfree(s, dps, (size_t)ngrid * nsig * 8);
  dfree(s, drho, (size_t)ngrid * chunk * 8);
  dfree(s, dv, (size_t)ngrid * chunk * 8);
  dfree(s, dg2, (size_t)nsig * chunk * 8);
  dfree(s, dg, (size_t)3 * ngrid * 4);
  dfree(s, dab, (size_t)2 * chunk * 4);
  dfree(s, dws, dgemm_ws_bytes(nsig, chunk, ngrid));
  if (rc != NGW_OK) return rc;
  for (int jj = 0; jj < nsig; ++jj)
    for (int ii = 0; ii < jj; ++ii) kx[jj + (size_t)ii * nsig] = kx[ii + (size_t)jj * nsig];
  return NGW_OK;
}

extern "C" int ngw_vxc_matrix(ngw_session *s, int ngrid, int nmem, const double *psi, const double *rho, int nsig,
                              const int *sig_bands, int ntrans, double *vxc, double *vx) {
  if (!s || ngrid <= 0 || nmem <= 0 || !psi || !rho || nsig <= 0 || !sig_bands || ntrans < 1 || !vxc) {
    set_error("ngw_vxc_matrix: bad arguments");
    return NGW_ERR_ARG;
  }
  NGW_TRY(check_bands(nsig, sig_bands, nmem, "ngw_vxc_matrix"));
  if (int e = check_density(ngrid, rho, "ngw_vxc_matrix")) return e;
  NGW_CUDA(cudaSetDevice(s->device));
  double *dps = nullptr, *drho = nullptr, *dvx = nullptr, *dvc = nullptr, *dw = nullptr, *dmx = nullptr,
         *dmc = nullptr, *dws = nullptr;
  const size_t pb = (size_t)ngrid * nsig * 8, mb = (size_t)nsig * nsig * 8;
  int rc = NGW_OK;
  std::vector<double> mx((size_t)nsig * nsig), mc((size_t)nsig * nsig);
  do {
    if (dalloc(s, (void **)&dps, pb) || dalloc(s, (void **)&dw, pb) || dalloc(s, (void **)&drho, (size_t)ngrid * 8) ||
        dalloc(s, (void **)&dvx, (size_t)ngrid * 8) || dalloc(s, (void **)&dvc, (size_t)ngrid * 8) ||
        dalloc(s, (void **)&dmx, mb) || dalloc(s, (void **)&dmc, mb) ||
        dalloc(s, (void **)&dws, dgemm_ws_bytes(nsig, nsig, ngrid))) {
      rc = NGW_ERR_OOM;
      break;
    }
    for (int j = 0; j < nsig && rc == NGW_OK; ++j)
      if (cudaMemcpyAsync(dps + (size_t)j * ngrid, psi + (size_t)(sig_bands[j] - 1) * ngrid, (size_t)ngrid * 8,
                          cudaMemcpyHostToDevice, s->stream)) {
        set_error("copy to device failed");
        rc = NGW_ERR_CUDA;
      }
    if (rc != NGW_OK) break;
    if (cudaMemcpyAsync(drho, rho, (size_t)ngrid * 8, cudaMemcpyHostToDevice, s->stream)) {
      set_error("copy to device failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    const int bx = std::min(256, (ngrid + 255) / 256);
    k_lda_potentials<<<std::min(1024, (ngrid + 255) / 256), 256, 0, s->stream>>>(drho, ngrid, dvx, dvc);
    const double nt = (double)ntrans, zero = 0.0;
    for (int w = 0; w < 2 && rc == NGW_OK; ++w) {
      k_grid_scale_cols<<<dim3(bx, ygrid(nsig)), 256, 0, s->stream>>>(dps, w == 0 ? dvx : dvc, ngrid, nsig, dw);
      if (dgemm(s->stream, true, false, nsig, nsig, ngrid, nt, dps, ngrid, dw, ngrid, zero, w == 0 ? dmx : dmc,
                nsig, dws, dgemm_ws_bytes(nsig, nsig, ngrid)) != cudaSuccess) {
        set_error("FP64 GEMM (V_xc matrix) failed");
        rc = NGW_ERR_CUDA;
      }
    }
    if (rc != NGW_OK) break;
    if (cudaMemcpyAsync(mx.data(), dmx, mb, cudaMemcpyDeviceToHost, s->stream) ||
        cudaMemcpyAsync(mc.data(), dmc, mb, cudaMemcpyDeviceToHost, s->stream) || cudaStreamSynchronize(s->stream)) {
      set_error("copy back failed");
      rc = NGW_ERR_CUDA;
      break;
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, dps, pb);
  dfree(s, dw, pb);
  dfree(s, drho, (size_t)ngrid * 8);
  dfree(s, dvx, (size_t)ngrid * 8);
  dfree(s, dvc, (size_t)ngrid * 8);
  dfree(s, dmx, mb);
  dfree(s, dmc, mb);
  dfree(s, dws, dgemm_ws_bytes(nsig, nsig, ngrid));
  if (rc != NGW_OK) return rc;
  for (size_t i = 0; i < (size_t)nsig * nsig; ++i) {
    vxc[i] = mx[i] + mc[i];
    if (vx) vx[i] = mx[i];
  }
  return NGW_OK;
}

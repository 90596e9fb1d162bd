// Coulomb block of the ISDF kernel:  M_C = ntrans/hcub * zeta^T (v_c zeta).
//
// v_c zeta_mu is the FFT-Poisson solve of shared/fft_module.F90z:122-177: each
// zeta column is packed into the (zero-padded) FFT box, transformed, multiplied
// by the truncated Coulomb kernel 8 pi (1 - cos(R_t |G|)) / |G|^2
// (8 pi R_t^2 / 2 at G = 0; shared/fft_module.F90z:628-691, R_t = 2 rmax), and
// transformed back.  The box edge is nfft = even(nint(4 rmax / h))
// (shared/parsec_wfn.F90:365-381), the scale 1/nfft^3 (fft_module.F90z:403),
// and the kernel matrix is the GEMM of shared/isdf_parallel_sym_UltraLowMem.F90:865-867.
// Columns are processed in batches: pack / multiply / unpack are kernels of
// this library, the 3-D transforms are batched cuFFT D2Z / Z2D.
#include <cufft.h>

#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "ngw_internal.h"
#include "xc_lda.cuh"

namespace ngw {

__global__ void k_coulomb_table(double *__restrict__ v, int n, double b, double trunc) {
  const int nh = n / 2 + 1;
  const size_t total = (size_t)n * n * nh;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(idx % nh);
    const int bb = (int)((idx / nh) % n);
    const int a = (int)(idx / ((size_t)nh * n));
    const int ja = a < n / 2 ? a : a - n;
    const int jb = bb < n / 2 ? bb : bb - n;
    const int jc = c;
    const double g2 = b * b * ((double)ja * ja + (double)jb * jb + (double)jc * jc);
    double r;
    if (ja == 0 && jb == 0 && jc == 0)
      r = trunc * trunc / 2.0;
    else
      r = (1.0 - cos(trunc * sqrt(g2))) / g2;
    v[idx] = 8.0 * M_PI * r;
  }
}

// box[col][a][b][c] = zeta[col][g] at the grid point's (wrapped) coordinates
__global__ void k_pack(const double *__restrict__ zeta, int ngrid, int ldz,
                       const int *__restrict__ gidx, int n, double *__restrict__ box, int ncol) {
  const int col = blockIdx.y;
  const size_t bsz = (size_t)n * n * n;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngrid; g += gridDim.x * blockDim.x) {
    int a = gidx[3 * g], b = gidx[3 * g + 1], c = gidx[3 * g + 2];
    a = ((a % n) + n) % n;
    b = ((b % n) + n) % n;
    c = ((c % n) + n) % n;
    box[(size_t)col * bsz + ((size_t)a * n + b) * n + c] = zeta[(size_t)col * ldz + g];
  }
  (void)ncol;
}

__global__ void k_unpack(const double *__restrict__ box, int ngrid, const int *__restrict__ gidx,
                         int n, double scale, double *__restrict__ out, int ldo) {
  const int col = blockIdx.y;
  const size_t bsz = (size_t)n * n * n;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngrid; g += gridDim.x * blockDim.x) {
    int a = gidx[3 * g], b = gidx[3 * g + 1], c = gidx[3 * g + 2];
    a = ((a % n) + n) % n;
    b = ((b % n) + n) % n;
    c = ((c % n) + n) % n;
    out[(size_t)col * ldo + g] = box[(size_t)col * bsz + ((size_t)a * n + b) * n + c] * scale;
  }
}

__global__ void k_mul_coulomb(cufftDoubleComplex *__restrict__ f, const double *__restrict__ v,
                              size_t per, int ncol) {
  const size_t total = per * (size_t)ncol;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const double w = v[i % per];
    f[i].x *= w;
    f[i].y *= w;
  }
}


int fft_coulomb_boxes(ngw_session *s, int n, int ncol, double *box, double2 *spec, const double *vtab);

// NGW_FFT=cufft selects cuFFT for the 3-D transforms (timing comparison);
// the default is the library's own FFT.
static bool use_cufft() {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("NGW_FFT");
    v = (e && std::string(e) == "cufft") ? 1 : 0;
  }
  return v == 1;
}

// v_c * rho for ncol columns (ngrid x ncol, column-major, ld ngrid) on the
// device: each column packed into the zero-padded FFT box, D2Z, multiplied by
// the truncated Coulomb kernel, Z2D, unpacked with 1/nfft^3
// (shared/fft_module.F90z:122-177).  Columns go through in batches of boxes
// that stay under ~2 GB.
int poisson_apply(ngw_session *s, int ngrid, int ncol, const double *drho, const int *dg, int nfft,
                  double h, double trunc, double *dv) {
  const int n = nfft;
  const size_t bsz = (size_t)n * n * n;
  const size_t csz = (size_t)n * n * (n / 2 + 1);
  // columns per FFT pass: a 2 GiB box + spectrum budget (NGW_POISSON_BATCH
  // fixes the count: tests of the chunked path at small sizes)
  int batch = (int)std::max<size_t>(1, (size_t)(2ull << 30) / (bsz * 8 + csz * 16));
  if (const char *e = getenv("NGW_POISSON_BATCH")) batch = std::max(1, atoi(e));
  if (batch > ncol) batch = ncol;
  double *box = nullptr, *vtab = nullptr;
  cufftDoubleComplex *spec = nullptr;
  int rc = NGW_OK;
  cufftHandle pf = 0, pb = 0;
  bool have_pf = false, have_pb = false;
  do {
    if (dalloc(s, (void **)&box, bsz * batch * 8) || dalloc(s, (void **)&spec, csz * batch * 16) ||
        dalloc(s, (void **)&vtab, csz * 8)) {
      rc = NGW_ERR_OOM;
      break;
    }
    const double b = 2.0 * M_PI / ((double)n * h);
    k_coulomb_table<<<1024, 256, 0, s->stream>>>(vtab, n, b, trunc);
    if (!use_cufft()) {
      // the library's own batched 3-D FFT (fft3d.cu)
      const double scale = 1.0 / ((double)n * (double)n * (double)n);
      int bx = (ngrid + 255) / 256;
      if (bx > 256) bx = 256;
      for (int c0 = 0; c0 < ncol && rc == NGW_OK; c0 += batch) {
        const int nc = std::min(batch, ncol - c0);
        cudaMemsetAsync(box, 0, bsz * nc * 8, s->stream);
        k_pack<<<dim3(bx, nc), 256, 0, s->stream>>>(drho + (size_t)c0 * ngrid, ngrid, ngrid, dg, n, box, nc);
        rc = fft_coulomb_boxes(s, n, nc, box, reinterpret_cast<double2 *>(spec), vtab);
        if (rc != NGW_OK) break;
        k_unpack<<<dim3(bx, nc), 256, 0, s->stream>>>(box, ngrid, dg, n, scale, dv + (size_t)c0 * ngrid, ngrid);
      }
      if (rc == NGW_OK && cudaGetLastError() != cudaSuccess) {
        set_error("Poisson kernels failed to launch");
        rc = NGW_ERR_CUDA;
      }
      break;
    }
    int dims[3] = {n, n, n};
    if (cufftPlanMany(&pf, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, batch) != CUFFT_SUCCESS) {
      set_error("cufftPlanMany D2Z failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    have_pf = true;
    if (cufftPlanMany(&pb, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, batch) != CUFFT_SUCCESS) {
      set_error("cufftPlanMany Z2D failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    have_pb = true;
    cufftSetStream(pf, s->stream);
    cufftSetStream(pb, s->stream);
    const double scale = 1.0 / ((double)n * (double)n * (double)n);
    for (int c0 = 0; c0 < ncol && rc == NGW_OK; c0 += batch) {
      const int nc = std::min(batch, ncol - c0);
      cudaMemsetAsync(box, 0, bsz * batch * 8, s->stream);
      int bx = (ngrid + 255) / 256;
      if (bx > 256) bx = 256;
      k_pack<<<dim3(bx, nc), 256, 0, s->stream>>>(drho + (size_t)c0 * ngrid, ngrid, ngrid, dg, n, box, nc);
      if (cufftExecD2Z(pf, box, spec) != CUFFT_SUCCESS) {
        set_error("cufftExecD2Z failed");
        rc = NGW_ERR_CUDA;
        break;
      }
      k_mul_coulomb<<<2048, 256, 0, s->stream>>>(spec, vtab, csz, batch);
      if (cufftExecZ2D(pb, spec, box) != CUFFT_SUCCESS) {
        set_error("cufftExecZ2D failed");
        rc = NGW_ERR_CUDA;
        break;
      }
      k_unpack<<<dim3(bx, nc), 256, 0, s->stream>>>(box, ngrid, dg, n, scale, dv + (size_t)c0 * ngrid, ngrid);
    }
    if (rc != NGW_OK) break;
    if (cudaGetLastError() != cudaSuccess) {
      set_error("Poisson kernels failed to launch");
      rc = NGW_ERR_CUDA;
      break;
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  if (have_pf) cufftDestroy(pf);
  if (have_pb) cufftDestroy(pb);
  dfree(s, box, bsz * batch * 8);
  dfree(s, spec, csz * batch * 16);
  dfree(s, vtab, csz * 8);
  return rc;
}

// M = (ntrans / hcub) zeta^T (v_c zeta) from a device-resident zeta
// (ngrid x n_isdf, column-major) and grid coordinates (3 x ngrid).
int coulomb_core(ngw_session *s, int ngrid, int n_isdf, const double *dz, const int *dg, int nfft,
                 double h, double trunc, double *dm) {
  double *dvz = nullptr, *dws = nullptr;
  int rc = NGW_OK;
  do {
    if (dalloc(s, (void **)&dvz, (size_t)ngrid * n_isdf * 8)) {
      rc = NGW_ERR_OOM;
      break;
    }
    if ((rc = poisson_apply(s, ngrid, n_isdf, dz, dg, nfft, h, trunc, dvz)) != NGW_OK) break;
    const double nf = 1.0 / (h * h * h);
    const double zero = 0.0;
    const size_t wsb = (size_t)8 * n_isdf * n_isdf * 8;   // up to 8 K slices
    if (dalloc(s, (void **)&dws, wsb)) {
      rc = NGW_ERR_OOM;
      break;
    }
    if (dgemm(s->stream, true, false, n_isdf, n_isdf, ngrid, nf, dz, ngrid, dvz, ngrid, zero, dm, n_isdf, dws,
              wsb) != cudaSuccess) {
      set_error("FP64 GEMM (zeta^T v zeta) failed");
      rc = NGW_ERR_CUDA;
      break;
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, dvz, (size_t)ngrid * n_isdf * 8);
  dfree(s, dws, (size_t)8 * n_isdf * n_isdf * 8);
  return rc;
}

}  // namespace ngw

using namespace ngw;

extern "C" int ngw_build_coulomb_kernel(ngw_session *s, int ngrid, int n_isdf, const double *zeta,
                                        const int *grid_idx, int nfft, double h, double trunc,
                                        double *mmtrx) {
  if (!s || ngrid <= 0 || n_isdf <= 0 || !zeta || !grid_idx || nfft < 4 || (nfft & 1) || h <= 0 ||
      !mmtrx) {
    set_error("ngw_build_coulomb_kernel: bad arguments");
    return NGW_ERR_ARG;
  }
  NGW_CUDA(cudaSetDevice(s->device));
  double *dz = nullptr, *dm = nullptr;
  int *dg = nullptr;
  int rc = NGW_OK;
  do {
    if (dalloc(s, (void **)&dz, (size_t)ngrid * n_isdf * 8) ||
        dalloc(s, (void **)&dm, (size_t)n_isdf * n_isdf * 8) || dalloc(s, (void **)&dg, (size_t)3 * ngrid * 4)) {
      rc = NGW_ERR_OOM;
      break;
    }
    if (cudaMemcpyAsync(dz, zeta, (size_t)ngrid * n_isdf * 8, cudaMemcpyHostToDevice, s->stream) ||
        cudaMemcpyAsync(dg, grid_idx, (size_t)3 * ngrid * 4, cudaMemcpyHostToDevice, s->stream)) {
      set_error("copy to device failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    rc = coulomb_core(s, ngrid, n_isdf, dz, dg, nfft, h, trunc, dm);
    if (rc != NGW_OK) break;
    if (cudaMemcpyAsync(mmtrx, dm, (size_t)n_isdf * n_isdf * 8, cudaMemcpyDeviceToHost, s->stream) ||
        cudaStreamSynchronize(s->stream)) {
      set_error("copy back failed");
      rc = NGW_ERR_CUDA;
      break;
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, dz, (size_t)ngrid * n_isdf * 8);
  dfree(s, dm, (size_t)n_isdf * n_isdf * 8);
  dfree(s, dg, (size_t)3 * ngrid * 4);
  return rc;
}

// ---------------------------------------------------------------------------
// f_xc block of the ISDF kernel:  M_xc = ntrans/hcub * zeta^T (f_xc * zeta)
// (shared/isdf_parallel_sym_UltraLowMem.F90:809-839).  f_xc is the
// unpolarised LDA kernel of shared/xc_module.F90:853-893 (fxc_get, kflag 1/2):
// 2 * (f_x + f_c) in Ry bohr^3, with f_x the analytic Slater exchange kernel
// and f_c libxc's finite difference of the Perdew-Zunger potential
// (LIB/libxc/src/lda.c:153-182, delta_rho = 1e-8, centred unless rho < 2 delta).
namespace ngw {

__global__ void k_fxc_lda(const double *__restrict__ rho, int n, double *__restrict__ fxc) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double r = rho[i];
    const double eps_x = -0.75 * cbrt(3.0 / M_PI) * cbrt(r);
    const double fx = 4.0 / 9.0 * eps_x / r;
    const double dr = 1e-8;
    double fc;
    if (r < 2.0 * dr) fc = (pz_vc(r + dr) - pz_vc(r)) / dr;
    else fc = (pz_vc(r + dr) - pz_vc(r - dr)) / (2.0 * dr);
    fxc[i] = (fx + fc) * 2.0;
  }
}

__global__ void k_scale_cols_by(const double *__restrict__ z, const double *__restrict__ f, int n,
                                int ncol, double *__restrict__ out) {
  const int col = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[(size_t)col * n + i] = f[i] * z[(size_t)col * n + i];
}


// M_xc = (ntrans / hcub) zeta^T (f_xc * zeta) from device-resident zeta and rho.
int fxc_core(ngw_session *s, int ngrid, int n_isdf, const double *dz, const double *drho, double h,
             double *dm, double *dfxc) {
  double *dfz = nullptr, *dws = nullptr;
  const size_t zb = (size_t)ngrid * n_isdf * 8, wsb = (size_t)8 * n_isdf * n_isdf * 8;
  int rc = NGW_OK;
  do {
    if (dalloc(s, (void **)&dfz, zb) || dalloc(s, (void **)&dws, wsb)) {
      rc = NGW_ERR_OOM;
      break;
    }
    k_fxc_lda<<<std::min(1024, (ngrid + 255) / 256), 256, 0, s->stream>>>(drho, ngrid, dfxc);
    k_scale_cols_by<<<dim3(std::min(256, (ngrid + 255) / 256), n_isdf), 256, 0, s->stream>>>(
        dz, dfxc, ngrid, n_isdf, dfz);
    const double nf = 1.0 / (h * h * h), zero = 0.0;
    if (dgemm(s->stream, true, false, n_isdf, n_isdf, ngrid, nf, dz, ngrid, dfz, ngrid, zero, dm, n_isdf, dws,
              wsb) != cudaSuccess) {
      set_error("FP64 GEMM (zeta^T f zeta) failed");
      rc = NGW_ERR_CUDA;
      break;
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, dfz, zb);
  dfree(s, dws, wsb);
  return rc;
}

int check_density(int ngrid, const double *rho, const char *who) {
  for (int i = 0; i < ngrid; ++i)
    if (!(rho[i] > 0.0) || !std::isfinite(rho[i])) {
      set_error("%s: density must be positive and finite (point %d)", who, i);
      return NGW_ERR_NONFINITE;
    }
  return NGW_OK;
}

}  // namespace ngw

extern "C" int ngw_build_fxc_kernel(ngw_session *s, int ngrid, int n_isdf, const double *zeta,
                                    const double *rho, double h, double *mxc, double *fxc_out) {
  using namespace ngw;
  if (!s || ngrid <= 0 || n_isdf <= 0 || !zeta || !rho || h <= 0 || !mxc) {
    set_error("ngw_build_fxc_kernel: bad arguments");
    return NGW_ERR_ARG;
  }
  if (int e = check_density(ngrid, rho, "ngw_build_fxc_kernel")) return e;
  NGW_CUDA(cudaSetDevice(s->device));
  double *dz = nullptr, *drho = nullptr, *dfxc = nullptr, *dm = nullptr;
  const size_t zb = (size_t)ngrid * n_isdf * 8;
  int rc = NGW_OK;
  do {
    if (dalloc(s, (void **)&dz, zb) || dalloc(s, (void **)&drho, (size_t)ngrid * 8) ||
        dalloc(s, (void **)&dfxc, (size_t)ngrid * 8) || dalloc(s, (void **)&dm, (size_t)n_isdf * n_isdf * 8)) {
      rc = NGW_ERR_OOM;
      break;
    }
    if (cudaMemcpyAsync(dz, zeta, zb, cudaMemcpyHostToDevice, s->stream) ||
        cudaMemcpyAsync(drho, rho, (size_t)ngrid * 8, cudaMemcpyHostToDevice, s->stream)) {
      set_error("copy to device failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    rc = fxc_core(s, ngrid, n_isdf, dz, drho, h, dm, dfxc);
    if (rc != NGW_OK) break;
    if (cudaMemcpyAsync(mxc, dm, (size_t)n_isdf * n_isdf * 8, cudaMemcpyDeviceToHost, s->stream) ||
        (fxc_out && cudaMemcpyAsync(fxc_out, dfxc, (size_t)ngrid * 8, cudaMemcpyDeviceToHost, s->stream)) ||
        cudaStreamSynchronize(s->stream)) {
      set_error("copy back failed");
      rc = NGW_ERR_CUDA;
      break;
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, dz, zb);
  dfree(s, drho, (size_t)ngrid * 8);
  dfree(s, dfxc, (size_t)ngrid * 8);
  dfree(s, dm, (size_t)n_isdf * n_isdf * 8);
  return rc;
}

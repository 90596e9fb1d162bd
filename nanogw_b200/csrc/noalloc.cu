// QP Newton solve for callers that cannot allocate device memory.
//
// Some host programs cannot call cudaMalloc when they need a QP energy: a
// Fortran driver that hands device memory out of its own pool, code that runs
// while a stream is being captured into a CUDA graph, or a process whose
// allocator has reserved all free device memory.  This entry point solves the
// same problem as ngw_qp_newton but takes device pointers for every input and
// output and keeps the spline workspace (4 * nen doubles per QP state) in a
// fixed file-scope device array, so it allocates nothing.
//
// Limits and sharing: the array holds NGW_NOALLOC_MAX_DOUBLES doubles (2 MiB),
// so nqp * 4 * nen must not exceed that; larger requests are rejected.  Every
// call on a device uses the same array and it keeps the previous call's
// contents (each solve overwrites every entry it reads before reading it, so
// nothing needs clearing); two calls whose kernels overlap on the GPU (for
// example on two streams) race on it.  The first call on each device looks up
// the array's device address with cudaGetSymbolAddress; make that first call
// before any stream capture.
#include <mutex>

#include "ngw_internal.h"

#define NGW_NOALLOC_MAX_DOUBLES (1 << 18)

namespace ngw {

// the kernel of the regular entry point (kernels_core.cu)
__global__ void k_qp_newton(int nqp, int nen, const double *__restrict__ sig,
                            const double *__restrict__ e1, const double *__restrict__ e0,
                            double deltae, const double *__restrict__ sigx,
                            const double *__restrict__ vxc, double xacc, double *__restrict__ eqp,
                            double *__restrict__ zfac, int *__restrict__ ierr,
                            double *__restrict__ work);

static __device__ __align__(256) double g_newton_scratch[NGW_NOALLOC_MAX_DOUBLES];

// device address of g_newton_scratch, looked up once per device and kept for
// the life of the process: after cudaDeviceReset (or anything else that
// destroys and recreates the device's primary context) the cached address is
// stale, so a process that resets a device must not call
// ngw_qp_newton_noalloc on it again
static double *scratch_address(int device, int *rc) {
  static std::mutex mu;
  static double *addr[64] = {nullptr};
  std::lock_guard<std::mutex> lk(mu);
  if (device < 0 || device >= 64) {
    set_error("device %d out of range", device);
    *rc = NGW_ERR_ARG;
    return nullptr;
  }
  if (!addr[device]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_newton_scratch);
    if (e != cudaSuccess) {
      set_error("cudaGetSymbolAddress(newton scratch) failed: %s", cudaGetErrorString(e));
      *rc = NGW_ERR_CUDA;
      return nullptr;
    }
    addr[device] = static_cast<double *>(p);
  }
  *rc = NGW_OK;
  return addr[device];
}

}  // namespace ngw

extern "C" int ngw_qp_newton_noalloc(int nqp, int nen, const double *sigma_c_ev,
                                     const double *e1_ev, const double *e0_ev, double deltae_ev,
                                     const double *sigx_ev, const double *vxc_ev, double xacc_ev,
                                     double *eqp_ev, double *zfac, int *ierr, void *stream) {
  using namespace ngw;
  if (nqp <= 0 || nen < 4 || !sigma_c_ev || !e1_ev || !e0_ev || !sigx_ev || !vxc_ev || !eqp_ev ||
      !zfac || !ierr) {
    set_error("ngw_qp_newton_noalloc: bad arguments");
    return NGW_ERR_ARG;
  }
  if ((long long)nqp * 4 * nen > NGW_NOALLOC_MAX_DOUBLES) {
    set_error("ngw_qp_newton_noalloc: nqp * 4 * nen = %lld exceeds the fixed workspace of %d doubles",
              (long long)nqp * 4 * nen, NGW_NOALLOC_MAX_DOUBLES);
    return NGW_ERR_BUDGET;
  }
  int dev = 0;
  NGW_CUDA(cudaGetDevice(&dev));
  int rc = NGW_OK;
  double *work = scratch_address(dev, &rc);
  if (rc != NGW_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_qp_newton<<<(nqp + 31) / 32, 32, 0, st>>>(nqp, nen, sigma_c_ev, e1_ev, e0_ev, deltae_ev, sigx_ev,
                                              vxc_ev, xacc_ev, eqp_ev, zfac, ierr, work);
  NGW_CUDA(cudaGetLastError());
  return NGW_OK;
}

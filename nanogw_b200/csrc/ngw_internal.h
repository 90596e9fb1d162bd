// Internal declarations shared by the ngw_b200 translation units.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cublas_v2.h>
#include <atomic>
#include <shared_mutex>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/ngw_b200.h"

namespace ngw {

void set_error(const char *fmt, ...);

// gridDim.y / gridDim.z are limited to 65535: kernels indexed by pair or chain
// in y take min(n, 65535) blocks there and stride over the rest.
inline unsigned ygrid(long long n) { return n < 1 ? 1u : (n < 65535 ? (unsigned)n : 65535u); }

#define NGW_CUDA(call)                                                           \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      ::ngw::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,               \
                       cudaGetErrorString(e_));                                  \
      return (e_ == cudaErrorMemoryAllocation) ? NGW_ERR_OOM : NGW_ERR_CUDA;     \
    }                                                                            \
  } while (0)

#define NGW_CUBLAS(call)                                                         \
  do {                                                                           \
    cublasStatus_t st_ = (call);                                                 \
    if (st_ != CUBLAS_STATUS_SUCCESS) {                                          \
      ::ngw::set_error("%s:%d %s: cublas status %d", __FILE__, __LINE__, #call,  \
                       (int)st_);                                                \
      return NGW_ERR_CUDA;                                                       \
    }                                                                            \
  } while (0)

#define NGW_TRY(call)                                                            \
  do {                                                                           \
    int r_ = (call);                                                             \
    if (r_ != NGW_OK) return r_;                                                 \
  } while (0)

// Device buffer owned by a session (bytes tracked for admission / reporting).
struct DBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

// Status word the kernels write when a bounded wait gives up or an index
// check fails; read back after every synchronising call.  DEV_TIMEOUT comes
// from a tensor-core GEMM's mbarrier wait: the CTA gave up while TMA copies or
// MMAs of its own may still have been in flight, so the session is refused
// further work.  DEV_BARRIER_TIMEOUT comes from a grid barrier of a kernel
// with nothing asynchronous in flight, which every CTA left cleanly.
enum DevStatus : int { DEV_OK = 0, DEV_TIMEOUT = 1, DEV_BOUNDS = 2, DEV_BARRIER_TIMEOUT = 3 };

struct MixedOperator;   // tcgen05 operand set (gemm_tc.cu)

}  // namespace ngw

struct ngw_session {
  int device = 0;
  cudaStream_t stream = nullptr;
  cublasHandle_t cublas = nullptr;
  int precision = NGW_PREC_FP64;
  size_t bytes = 0;
  // operator
  int n_isdf = 0, nmem = 0, ncv = 0;
  double *d_psi = nullptr;     // (n_isdf, nmem) column-major
  double *d_M = nullptr;       // (n_isdf, n_isdf)
  double *d_Mxc = nullptr;     // optional
  int *d_cvpair = nullptr;     // (2, ncv) 1-based
  double *d_sqrtR = nullptr;   // (ncv)
  double *d_C = nullptr;       // (n_isdf, ncv) pair products (FP64)
  bool have_isdf = false, have_pairs = false, have_C = false;
  ngw::MixedOperator *mixed = nullptr;
  int *d_status = nullptr;     // device status word
  // top eigenpairs of C (FP64 Lanczos, full reorthogonalisation) for deflation
  std::vector<double> eig_vals, eig_res;   // Ritz values (descending) and residual bounds
  double *eig_U = nullptr;                  // (ncv, eig_k) Ritz vectors
  size_t eig_U_bytes = 0;
  int eig_k = 0, eig_tda = -1;
  // CUDA graphs of the per-block Sigma_c region, keyed by shapes + pointers
  struct GraphEntry {
    std::vector<unsigned long long> key;
    cudaGraphExec_t exec = nullptr;
    int seen = 0;
  };
  std::vector<GraphEntry> graphs;
  // bumped whenever a device buffer that captured graphs may reference is
  // freed or reallocated; part of every graph key
  unsigned long long gen = 0;
  // the mixed operator's values are stale (new Psi_intp / M / pairs of the
  // same shapes were uploaded into the existing buffers)
  bool mixed_dirty = false;
  void *cublas_ws = nullptr;
  void *cusolver = nullptr;    // cusolverDnHandle_t, created on first use
  bool use_graphs = true;
  // set when a GEMM's bounded wait timed out: the session refuses further
  // work (NGW_ERR_STATE) and has to be destroyed and created again
  bool poisoned = false;
  // scratch (grown on demand)
  std::vector<ngw::DBuf> scratch;
  std::vector<void *> owned;
};

namespace ngw {

// allocation helpers (track session bytes)
cudaError_t pool_alloc(ngw_session *s, void **p, size_t bytes);
void pool_free(ngw_session *s, void *p);

// Per-device lock that keeps the autotuner's timings clean: a Sigma_c solve
// holds it shared from the launch of its device region until its results
// are on the host; the autotuner holds it exclusively, so it times its
// candidates without other sessions' solves running beside them.
std::shared_mutex &gpu_quiet_lock(int device);

// Raises a kernel's dynamic shared-memory limit to `bytes` on the current
// device, once per device (the attribute is per device; `done` holds one bit
// per device already set).  Safe to call from several threads.
template <class Kernel>
inline cudaError_t smem_limit_once(Kernel kernel, int bytes, std::atomic<unsigned long long> &done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}
int dalloc(ngw_session *s, void **p, size_t bytes);
void dfree(ngw_session *s, void *p, size_t bytes);
int scratch(ngw_session *s, int slot, size_t bytes, void **p);
int check_status(ngw_session *s);
// Device buffers of the operator / chains / scratch are about to change: wait
// for the stream, drop every captured graph and advance the generation.
void bump_generation(ngw_session *s);
// session's cuSOLVER dense handle on the session stream (created on first use)
int session_cusolver(ngw_session *s, void **handle);

// ---- grouped mixed-precision p(C) v across molecules (gemm_tc.cu) ----
struct GroupEntry;           // one problem of a grouped tcgen05 GEMM launch (device table)
struct GroupMember {         // one molecule of the group
  ngw_session *s;
  const double *g;           // Chebyshev coefficients g[0..n]
  double c0, c1;             // the Chebyshev interval [c0 - c1, c0 + c1]
  int ldv;                   // leading dimension of v / out64 (ncv)
  double *out_first;         // out64 of the step-0 product
  double *out_later;         // out64 of the later products
  int nb;                    // chains at step 0
  const int *nact;           // chains still running at step k (nullptr: nb every step)
};
struct GroupPlan {           // device tables of a group (built by group_build)
  int G = 0, n = 0, tda = 0, steps = 0;
  GroupEntry *d_tab = nullptr;
  int *d_steps = nullptr;
  std::vector<int> tiles1, tiles2;   // launch sizes per step
  std::vector<int> nv;               // [steps][G] chains per member
};
size_t group_bytes(int G, int n, int steps);
int group_build(std::vector<GroupMember> &mem, int n, int tda, int steps, void *buf, cudaStream_t st,
                GroupPlan &P);
int group_poly_apply(const GroupPlan &P, std::vector<GroupMember> &mem, int k, const double *const *vin,
                     cudaStream_t st);

// ---- FP64 GEMM on the FP64 tensor cores (dgemm.cu) ----
// C = alpha op(A) op(B) + beta C, column-major (cuBLAS conventions).  With a
// workspace (ws, ws_bytes) shapes with a small tile grid split K into slices
// summed in order; without one they run unsplit.  Launch-only: safe inside
// stream capture once the kernel has run outside one.
cudaError_t dgemm(cudaStream_t st, bool ta, bool tb, int m, int n, int k, double alpha, const double *A,
                  int lda, const double *B, int ldb, double beta, double *C, int ldc, double *ws = nullptr,
                  size_t ws_bytes = 0);
// workspace that lets dgemm() choose any split for an m x n result
size_t dgemm_ws_bytes(int m, int n, int k);

// ---- FP64 path kernels (kernels_core.cu) ----
void launch_pair_gather_f64(const double *psi, int n_isdf, const int *cvpair, int ncv,
                            double *C, cudaStream_t st);
void launch_pair_gather_cols(const double *psi, int n_isdf, const int *b1, const int *b2,
                             int n, double *out, cudaStream_t st);
void launch_scale_rows(const double *s, const double *x, int ldx, double *y, int ldy,
                       int ncv, int nb, int tamm_d, cudaStream_t st);
void launch_matvec_combine(const double *s, const double *h, const double *z, double *y,
                           const double *vec, int ncv, int nb, int tamm_d, int horner_k,
                           double pk, double pk1, double *hs_next, cudaStream_t st);
void launch_copy_cols(const double *x, int ldx, double *y, int ldy, int n, int nb,
                      cudaStream_t st);
void launch_lanczos_init(const double *v0, int ld, const double *v0_norm, double *vec,
                         double *hs, const double *s, int ncv, int nb, int tamm_d,
                         double *b_elmt, int niter, const int *len, int *clen, cudaStream_t st);
void launch_lanczos_first(double *w, const double *v, int ncv, int nb, double *a, double *b,
                          int niter, int *clen, double eps, cudaStream_t st);
void launch_lanczos_step(double *w, double *v, const double *t, int ncv, int nb, int k,
                         double *a, double *b, int niter, const double *s, double *hs,
                         int tamm_d, int prescale_next, int *clen, double eps, cudaStream_t st);
// one molecule's chains in a grouped Lanczos-step launch
struct LanczosGroupEntry {
  double *w, *v;
  const double *t;
  double *a, *b;
  const double *s;
  int *clen;
  double eps;
  int ncv, niter, prescale_next, pad;
};
void launch_lanczos_step_grouped(const LanczosGroupEntry *tab, const int *cb, int G, int k, int total,
                                 cudaStream_t st);
void launch_lanczos_reorth_step(double *w, double *v, const double *t, int ncv, int nb, int k, double *a,
                                double *b, int niter, const double *s, double *hs, int tamm_d,
                                int prescale_next, int *clen, double eps, double *basis, long long ldb,
                                cudaStream_t st);
void launch_basis_init(const double *vec, int ncv, int nb, double *basis, long long ldb, cudaStream_t st);
void launch_lanczos_prescale(double *w, double *v, int ncv, int nb, int k, const double *b,
                             int niter, const double *s, double *hs, int tamm_d, const int *clen,
                             cudaStream_t st);
void launch_contfrac(const double *a, const double *b, int niter, int nb, const double *zz,
                     int nz, double *spectra, const int *clen, cudaStream_t st);
void launch_sigma_spectra(const double *a, const double *b, int niter, int nchain,
                          const double *e1, const int *chain_band, const int *chain_qp,
                          const double *zz0, double de, int nen, double ecuts, int nval,
                          double *S, const int *clen, cudaStream_t st);
void launch_sigma_reduce(const double *S, const double *pnorm2, const double *e1,
                         const int *chain_band, const double *zz0, double de, int nen,
                         double ecuts, int nval, int nbsum, int nqp, int tamm_d,
                         double *sigma, int accumulate, const int *slot, cudaStream_t st);
void launch_norms(const double *P, int ncv, int nb, const double *s, int tamm_d, double *P_out,
                  double *pnorm2, cudaStream_t st);
void launch_qp_newton_ws(int nqp, int nen, const double *sig, const double *e1, const double *e0,
                         double deltae, const double *sigx, const double *vxc, double xacc,
                         double *eqp, double *zfac, int *ierr, double *work, cudaStream_t st);
void launch_sqrt_vec(const double *x, double *y, int n, cudaStream_t st);
void launch_k_combine(const double *M, const double *Mxc, int n, int kflag, double *out,
                      cudaStream_t st);

}  // namespace ngw

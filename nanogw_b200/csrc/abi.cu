// C ABI of ngw_b200: sessions, the ISDF operator, matvec / polynomial matvec,
// Lanczos spectra, Sigma_c driver, k_integrate and the QP Newton solve.
// FP64 GEMMs of the plain path go through cuBLAS (library GEMMs); every other
// step is a kernel of this library.
#include <algorithm>
#include <chrono>
#include <string>
#include <cstdarg>
#include <cstring>
#include <cmath>
#include <vector>

#include <cusolverDn.h>

#include "ngw_internal.h"

namespace ngw {

int mixed_build_operator(ngw_session *s, int kdef, int tda);
int mixed_kdef(ngw_session *s);
int mixed_set_deflation_values(ngw_session *s, const double *pvals);
int compute_top_eigs(ngw_session *s, int tamm_d, int kmax, int msteps);
void extern_mixed_tune(ngw_session *s, int *tune);
int mixed_prepare_chains(ngw_session *s, int nb, int bn1, int bn2, int split1);
bool mixed_dense_ready(ngw_session *s, const double *g, int n, double c0, double c1);
void mixed_dense_mark(ngw_session *s, bool used);
int mixed_dense_build(ngw_session *s, const double *g, int n, double c0, double c1);
int mixed_dense_apply(ngw_session *s, int nb, const double *v, int ldv, double *out64);
int mixed_prepare_dense(ngw_session *s, int nb);
int mixed_poly_apply(ngw_session *s, int nb, const double *v, int ldv, const double *g, int n,
                     double c0, double c1, int tda, double *out64);
void mixed_free(ngw_session *s);
void monomial_to_chebyshev(const double *poly_hl, int n, double lo, double hi, double *g);


static thread_local char g_err[1024] = {0};

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

// Device memory comes from the device's stream-ordered pool on the session
// stream (its release threshold is raised at session creation, so freed
// blocks stay cached for the next request).  A free is ordered after the
// work already queued on the session stream and, unlike cudaFree, does not
// wait for the whole device: sessions serving requests side by side do not
// stall each other.  An allocation waits for the session stream, so the
// block is ready for use on any stream when pool_alloc returns.
cudaError_t pool_alloc(ngw_session *s, void **p, size_t bytes) {
  *p = nullptr;
  cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  return e;
}

void pool_free(ngw_session *s, void *p) {
  if (p) cudaFreeAsync(p, s->stream);
}

std::shared_mutex &gpu_quiet_lock(int device) {
  static std::shared_mutex locks[64];
  return locks[device & 63];
}

int dalloc(ngw_session *s, void **p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = pool_alloc(s, p, bytes);
  if (e != cudaSuccess) {
    set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    *p = nullptr;
    return NGW_ERR_OOM;
  }
  s->bytes += bytes;
  return NGW_OK;
}

void dfree(ngw_session *s, void *p, size_t bytes) {
  if (!p) return;
  pool_free(s, p);
  s->bytes -= bytes;
}

// Named scratch slots, grown on demand and kept for the session's lifetime.
int scratch(ngw_session *s, int slot, size_t bytes, void **p) {
  if ((int)s->scratch.size() <= slot) s->scratch.resize(slot + 1);
  DBuf &b = s->scratch[slot];
  if (b.bytes < bytes) {
    bump_generation(s);
    if (b.p) {
      NGW_CUDA(cudaStreamSynchronize(s->stream));
      dfree(s, b.p, b.bytes);
      b.p = nullptr;
      b.bytes = 0;
    }
    NGW_TRY(dalloc(s, &b.p, bytes));
    b.bytes = bytes;
  }
  *p = b.p;
  return NGW_OK;
}

int check_status(ngw_session *s) {
  int h = 0;
  NGW_CUDA(cudaMemcpyAsync(&h, s->d_status, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  if (h != DEV_OK) {
    int z = 0;
    cudaMemcpy(s->d_status, &z, sizeof(int), cudaMemcpyHostToDevice);
    if (h == DEV_TIMEOUT) {
      // a GEMM CTA gave up with its own copies possibly in flight: the
      // kernel's state is not defined afterwards, so the session stops here
      s->poisoned = true;
      set_error("device status %d: a tensor-core GEMM's bounded wait timed out; the session refuses "
                "further work (destroy and create it again)", h);
      return NGW_ERR_TIMEOUT;
    }
    if (h == DEV_BARRIER_TIMEOUT) {
      set_error("device status %d: a grid barrier's bounded wait timed out", h);
      return NGW_ERR_TIMEOUT;
    }
    set_error("device status %d (index check)", h);
    return NGW_ERR_CUDA;
  }
  return NGW_OK;
}

void bump_generation(ngw_session *s) {
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (auto &g : s->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  s->graphs.clear();
  ++s->gen;
}

int session_cusolver(ngw_session *s, void **handle) {
  if (!s->cusolver) {
    cusolverDnHandle_t h = nullptr;
    if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) {
      set_error("cusolverDnCreate failed");
      return NGW_ERR_CUDA;
    }
    s->cusolver = h;
  }
  if (cusolverDnSetStream((cusolverDnHandle_t)s->cusolver, s->stream) != CUSOLVER_STATUS_SUCCESS) {
    set_error("cusolverDnSetStream failed");
    return NGW_ERR_CUDA;
  }
  *handle = s->cusolver;
  return NGW_OK;
}

static bool all_finite(const double *x, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(x[i])) return false;
  return true;
}

// slots of session scratch
enum {
  SL_IN = 0, SL_OUT, SL_HS, SL_T1, SL_T2, SL_Z, SL_VEC, SL_WVEC, SL_TMP, SL_A, SL_B, SL_ZZ,
  SL_SPEC, SL_CMN, SL_CM, SL_P, SL_P2, SL_PN2, SL_PN, SL_CHB, SL_CHQ, SL_E1, SL_ZZ0, SL_SIG,
  SL_KR, SL_KC, SL_KM, SL_B1, SL_B2, SL_QPW, SL_QPIO, SL_SPECS, SL_CLEN, SL_LEN, SL_SLOT, SL_BASIS,
  SL_DGWS, SL_GROUP, SL_LGROUP, SL_NUM
};

// ---------------------------------------------------------------------------
// FP64 matvec on device buffers.  hs = (R^1/2 or 1) * x must already be in
// place; y = H x; optional Horner step against vec; optional next hs.
static int matvec_f64_dev(ngw_session *s, int nb, double *hs, double *y, const double *vec,
                          int tamm_d, int horner_k, double pk, double pk1, double *hs_next) {
  double *t1, *t2, *z;
  NGW_TRY(scratch(s, SL_T1, (size_t)s->n_isdf * nb * 8, (void **)&t1));
  NGW_TRY(scratch(s, SL_T2, (size_t)s->n_isdf * nb * 8, (void **)&t2));
  NGW_TRY(scratch(s, SL_Z, (size_t)s->ncv * nb * 8, (void **)&z));
  const double one = 1.0, zero = 0.0;
  // tmp_vec = Cmtrx * Hvec          (apply_matvec_lowcomsym.F90:228-229)
  NGW_CUBLAS(cublasDgemm(s->cublas, CUBLAS_OP_N, CUBLAS_OP_N, s->n_isdf, nb, s->ncv, &one, s->d_C,
                         s->n_isdf, hs, s->ncv, &zero, t1, s->n_isdf));
  // MC_vec = Mmtrx * tmp_vec         (:283-284)
  NGW_CUBLAS(cublasDgemm(s->cublas, CUBLAS_OP_N, CUBLAS_OP_N, s->n_isdf, nb, s->n_isdf, &one,
                         s->d_M, s->n_isdf, t1, s->n_isdf, &zero, t2, s->n_isdf));
  // CMC_vec = Cmtrx^T * MC_vec       (:365-366)
  NGW_CUBLAS(cublasDgemm(s->cublas, CUBLAS_OP_T, CUBLAS_OP_N, s->ncv, nb, s->n_isdf, &one, s->d_C,
                         s->n_isdf, t2, s->n_isdf, &zero, z, s->ncv));
  launch_matvec_combine(s->d_sqrtR, hs, z, y, vec, s->ncv, nb, tamm_d, horner_k, pk, pk1, hs_next,
                        s->stream);
  NGW_CUDA(cudaGetLastError());
  return NGW_OK;
}

int matvec_f64_dev_pub(ngw_session *s, int nb, double *hs, double *y, int tamm_d) {
  return matvec_f64_dev(s, nb, hs, y, nullptr, tamm_d, 0, 0.0, 0.0, nullptr);
}

// out = p(H) vec by Horner (FP64), vec/out: (ncv, nb); hs scratch holds
// (R^1/2) vec on entry and is clobbered.
static int poly_f64_dev(ngw_session *s, int nb, const double *poly, int npoly, const double *vec,
                        double *hs, double *out) {
  for (int k = 1; k <= npoly; ++k) {
    double *hn = (k < npoly) ? hs : nullptr;
    NGW_TRY(matvec_f64_dev(s, nb, hs, out, vec, 0, k, poly[k - 1], poly[k], hn));
  }
  return NGW_OK;
}

struct PolyPlan {
  int tamm_d = 0;
  int npoly = 0;
  std::vector<double> poly;   // high -> low
  std::vector<double> cheb;   // Chebyshev coefficients (mixed)
  double c0 = 0, c1 = 1;
  int kdef = 0;               // deflated eigenpairs (mixed)
  bool dense = false;         // mixed: p(C) through the dense operator H (one GEMM per product)
};

// t = p(H) vec  (or A vec with TDA) on device, in the session's precision.
static int apply_poly(ngw_session *s, const PolyPlan &pp, int nb, const double *vec, double *hs,
                      double *t) {
  if (s->precision == NGW_PREC_MIXED) {
    if (pp.tamm_d) {
      // A = R + 2 C^T M C as the degree-1 Chebyshev series x on [c0-c1, c0+c1]
      const double g[2] = {pp.c0, pp.c1};
      return mixed_poly_apply(s, nb, vec, s->ncv, g, 1, pp.c0, pp.c1, 1, t);
    }
    if (pp.dense) return mixed_dense_apply(s, nb, vec, s->ncv, t);
    return mixed_poly_apply(s, nb, vec, s->ncv, pp.cheb.data(), pp.npoly, pp.c0, pp.c1, 0, t);
  }
  if (pp.tamm_d) return matvec_f64_dev(s, nb, hs, t, vec, 1, 0, 0.0, 0.0, nullptr);
  return poly_f64_dev(s, nb, pp.poly.data(), pp.npoly, vec, hs, t);
}

// Lanczos recurrence for nb chains whose normalised start vectors are set up
// by launch_lanczos_init.  Leaves a, b (niter x nb).  clen: per-chain lengths
// (set by launch_lanczos_init, lowered by the convergence mask eps);
// nact[k] (optional): chains still scheduled at step k -- the chains are
// ordered longest first, so step k's matvecs and updates cover chains
// 0 .. nact[k]-1 only.
static int lanczos_dev(ngw_session *s, const PolyPlan &pp, int nb, int niter, double *V,
                       double *W, double *hs, double *tmp, double *a, double *b, int *clen,
                       double eps, const std::vector<int> *nact, double *basis = nullptr,
                       long long ldb = 0) {
  // the scaled copy hs feeds only the FP64 path's first DGEMM
  double *hsn = (s->precision == NGW_PREC_MIXED) ? nullptr : hs;
  auto active = [&](int k) { return nact ? (*nact)[k] : nb; };
  if (basis) launch_basis_init(V, s->ncv, nb, basis, ldb, s->stream);
  // wvec = p(H) vec
  NGW_TRY(apply_poly(s, pp, nb, V, hs, W));
  if (basis) {
    // first step with Gram-Schmidt against v_0, rescale into v_1
    launch_lanczos_reorth_step(W, V, nullptr, s->ncv, nb, 0, a, b, niter, s->d_sqrtR, hsn, pp.tamm_d,
                               niter >= 2 ? 1 : 0, clen, eps, basis, ldb, s->stream);
  } else {
    launch_lanczos_first(W, V, s->ncv, nb, a, b, niter, clen, eps, s->stream);
    if (niter >= 2)
      launch_lanczos_prescale(W, V, s->ncv, active(1), 1, b, niter, s->d_sqrtR, hsn, pp.tamm_d, clen,
                              s->stream);
  }
  double *vec = W, *wvec = V;   // roles after the swap
  for (int k = 1; k < niter; ++k) {
    const int nk = active(k);
    if (nk <= 0) break;
    NGW_TRY(apply_poly(s, pp, nk, vec, hs, tmp));
    if (basis)
      launch_lanczos_reorth_step(wvec, vec, tmp, s->ncv, nk, k, a, b, niter, s->d_sqrtR, hsn, pp.tamm_d,
                                 (k + 1 < niter) ? 1 : 0, clen, eps, basis, ldb, s->stream);
    else
      launch_lanczos_step(wvec, vec, tmp, s->ncv, nk, k, a, b, niter, s->d_sqrtR, hsn, pp.tamm_d,
                          (k + 1 < niter) ? 1 : 0, clen, eps, s->stream);
    if (k + 1 < niter) {
      double *t = vec;
      vec = wvec;
      wvec = t;
    }
  }
  NGW_CUDA(cudaGetLastError());
  return NGW_OK;
}

// NGW_TIMING=1: host wall-clock of the phases of a call on stderr (the
// stream is synchronised at each mark, so only for diagnosis).
struct PhaseTimer {
  ngw_session *s;
  bool on;
  std::chrono::steady_clock::time_point t;
  std::string line;
  explicit PhaseTimer(ngw_session *s_) : s(s_) {
    const char *e = getenv("NGW_TIMING");
    on = e && e[0] == '1';
    if (on) {
      cudaStreamSynchronize(s->stream);
      t = std::chrono::steady_clock::now();
    }
  }
  void mark(const char *name) {
    if (!on) return;
    cudaStreamSynchronize(s->stream);
    const auto now = std::chrono::steady_clock::now();
    char buf[96];
    snprintf(buf, sizeof(buf), " %s=%.2fms", name, std::chrono::duration<double, std::milli>(now - t).count());
    line += buf;
    t = now;
  }
  ~PhaseTimer() {
    if (on) fprintf(stderr, "ngw timing:%s\n", line.c_str());
  }
};

static int need_op(ngw_session *s) {
  if (!s) {
    set_error("null session");
    return NGW_ERR_ARG;
  }
  if (s->poisoned) {
    set_error("a tensor-core GEMM of this session timed out earlier; destroy and create the session again");
    return NGW_ERR_STATE;
  }
  if (!s->have_isdf || !s->have_pairs) {
    set_error("ISDF operator or pair list not set");
    return NGW_ERR_STATE;
  }
  if (!s->have_C) {
    launch_pair_gather_f64(s->d_psi, s->n_isdf, s->d_cvpair, s->ncv, s->d_C, s->stream);
    NGW_CUDA(cudaGetLastError());
    s->have_C = true;
  }
  return NGW_OK;
}

static double poly_eval(const std::vector<double> &p, double x) {
  long double acc = 0.0L;
  for (double c : p) acc = acc * x + (long double)c;
  return (double)acc;
}

// Mixed-precision plan: Chebyshev interval and deflated eigenpairs.
// Eigenpairs of the operator (C, or A with TDA) come from an FP64 Lanczos run
// with full reorthogonalisation (cached per operator).  Top eigenpairs are
// deflated while |p(lambda_k)| exceeds 4x the largest |p| on [0, 1.05
// lambda_{k+1}] (the reference's fit leaves that range), so the Clenshaw
// recurrence only ever sees a spectrum on which p is bounded.
// Dense or factored p(C) for a solve of `steps` products on nb chains: the
// dense operator costs about 2 sqrt(p) FP64 GEMMs of N_cv^3 multiply-adds to
// form (Paterson-Stockmeyer; nothing when it is already built for this
// polynomial) and 2 N_cv^2 split-BF16 ones per chain
// and product; the factored form 4 p (N_mu + k) N_cv per chain and product in
// 2 p launches.  Rates: the FP64 tensor-core GEMM ~25 TFLOP/s, the dense
// split-BF16 GEMM ~0.9 PFLOP/s executed (x3 products), the factored pair
// ~0.6 PFLOP/s executed plus ~5 us per launch.  NGW_DENSE=0 / 1 overrides
// (1 within the memory cap: N_cv <= 16384).
static bool want_dense(ngw_session *s, const PolyPlan &pp, int steps, int nb) {
  if (pp.tamm_d || pp.npoly < 2) return false;
  const double N = s->ncv, mu = s->n_isdf + pp.kdef, p = pp.npoly;
  if (N > 16384) return false;
  if (const char *e = getenv("NGW_DENSE")) {
    if (e[0] == '0') return false;
    if (e[0] == '1') return true;
  }
  if (steps < 1 || nb < 1) return false;
  const bool built = mixed_dense_ready(s, pp.cheb.data(), pp.npoly, pp.c0, pp.c1);
  const int m = std::max(2, (int)std::ceil(std::sqrt(p + 1.0)));
  const double products = (m - 1) + pp.npoly / m;
  const double form = built ? 0.0 : 2.0 * products * N * N * N / 25e12;
  const double dense_step = 3.0 * 2.0 * N * N * nb / 0.9e15 + 10e-6;
  const double fact_step = p * (3.0 * 4.0 * mu * N * nb / 0.6e15 + 10e-6);
  return form + steps * dense_step < steps * fact_step;
}

static int plan_mixed(ngw_session *s, PolyPlan &pp, double lo_in, double hi_in, int steps, int nb) {
  const int tda = pp.tamm_d;
  PhaseTimer tm(s);
  if (hi_in > lo_in) {
    pp.c0 = 0.5 * (hi_in + lo_in);
    pp.c1 = 0.5 * (hi_in - lo_in);
    pp.kdef = 0;
  } else {
    if (s->eig_tda != tda) NGW_TRY(compute_top_eigs(s, tda, 64, 240));
    tm.mark("eigenpairs");
    const std::vector<double> &r = s->eig_vals, &res = s->eig_res;
    const int mm = (int)r.size();
    int k = 0;
    if (!tda) {
      // typical |p| on the spectrum: median over the Ritz values
      std::vector<double> pv(mm);
      for (int i = 0; i < mm; ++i) pv[i] = std::fabs(poly_eval(pp.poly, r[i]));
      std::vector<double> srt(pv);
      std::nth_element(srt.begin(), srt.begin() + mm / 2, srt.end());
      const double typical = std::max(srt[mm / 2], 1e-300);
      // deflate while the Clenshaw interval [0, 1.05 lambda_k] would hold
      // values of |p| more than 8x the typical one
      auto interval_max = [&](double h) {
        double m = 0.0;
        for (int i = 0; i <= 4000; ++i) m = std::max(m, std::fabs(poly_eval(pp.poly, h * i / 4000.0)));
        return m;
      };
      while (k < std::min(s->eig_k, mm - 1) && interval_max(1.05 * (r[k] + res[k])) > 8.0 * typical &&
             res[k] < 1e-6 * std::fabs(r[0]))
        ++k;
    }
    const double top = (k < mm) ? r[k] + res[k] : 0.0;
    const double hi = std::max(1.05 * top, 1e-12);
    pp.c0 = 0.5 * hi;
    pp.c1 = 0.5 * hi;
    pp.kdef = k;
  }
  if (!tda) {
    pp.cheb.resize(pp.npoly + 1);
    monomial_to_chebyshev(pp.poly.data(), pp.npoly, pp.c0 - pp.c1, pp.c0 + pp.c1, pp.cheb.data());
  }
  tm.mark("interval");
  if (!s->mixed || s->mixed_dirty || mixed_kdef(s) != pp.kdef)
    NGW_TRY(mixed_build_operator(s, pp.kdef, tda));
  tm.mark("split_operator");
  std::vector<double> pv(pp.kdef);
  for (int j = 0; j < pp.kdef; ++j) pv[j] = tda ? s->eig_vals[j] : poly_eval(pp.poly, s->eig_vals[j]);
  NGW_TRY(mixed_set_deflation_values(s, pv.data()));
  pp.dense = want_dense(s, pp, steps, nb);
  if (pp.dense) NGW_TRY(mixed_dense_build(s, pp.cheb.data(), pp.npoly, pp.c0, pp.c1));
  mixed_dense_mark(s, pp.dense);
  tm.mark("dense_operator");
  return NGW_OK;
}

static int make_plan(ngw_session *s, PolyPlan &pp, const double *poly, int npoly, int tamm_d,
                     double lo, double hi, int steps = 1, int nb = 1) {
  pp.tamm_d = tamm_d;
  if (!tamm_d) {
    if (!poly || npoly < 1) {
      set_error("polynomial of degree >= 1 required");
      return NGW_ERR_ARG;
    }
    pp.npoly = npoly;
    pp.poly.assign(poly, poly + npoly + 1);
    if (!all_finite(poly, npoly + 1)) {
      set_error("non-finite polynomial coefficient");
      return NGW_ERR_NONFINITE;
    }
  } else {
    pp.npoly = 1;
    pp.poly = {1.0, 0.0};
  }
  if (s->precision == NGW_PREC_MIXED) NGW_TRY(plan_mixed(s, pp, lo, hi, steps, nb));
  return NGW_OK;
}

// Run `region` (launches only, no host synchronisation or allocation) on the
// session stream, through a CUDA graph once the same key has been seen before.
template <class F>
static int run_graphed(ngw_session *s, const std::vector<unsigned long long> &key, F region) {
  if (!s->use_graphs) return region();
  ngw_session::GraphEntry *e = nullptr;
  for (auto &g : s->graphs)
    if (g.key == key) e = &g;
  if (!e) {
    if (s->graphs.size() >= 8) {
      if (s->graphs.front().exec) cudaGraphExecDestroy(s->graphs.front().exec);
      s->graphs.erase(s->graphs.begin());
    }
    s->graphs.push_back(ngw_session::GraphEntry());
    e = &s->graphs.back();
    e->key = key;
  }
  if (e->exec) {
    NGW_CUDA(cudaGraphLaunch(e->exec, s->stream));
    return NGW_OK;
  }
  if (e->seen == 0) {   // first time: run eagerly (sizes every scratch buffer)
    e->seen = 1;
    return region();
  }
  cudaGraph_t graph = nullptr;
  NGW_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  int rc = region();
  cudaError_t ce = cudaStreamEndCapture(s->stream, &graph);
  if (rc != NGW_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (ce != cudaSuccess) {
    set_error("graph capture failed: %s", cudaGetErrorString(ce));
    return NGW_ERR_CUDA;
  }
  ce = cudaGraphInstantiate(&e->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) {
    e->exec = nullptr;
    set_error("graph instantiate failed: %s", cudaGetErrorString(ce));
    return NGW_ERR_CUDA;
  }
  NGW_CUDA(cudaGraphLaunch(e->exec, s->stream));
  return NGW_OK;
}

static unsigned long long dbits(double x) {
  unsigned long long u;
  std::memcpy(&u, &x, 8);
  return u;
}

// ---------------------------------------------------------------------------
// Sigma_c driver (SIGMA/calculate_sigma_lanczos_lowcomsym.F90z:516-779), split
// into the host preparation, one device region per chain block (run through
// the graph cache) and the download, so that a batch of sessions can record
// their regions as branches of one graph.
struct SigmaJob {
  ngw_session *s = nullptr;
  const ngw_sigma_params *p = nullptr;
  const double *e1 = nullptr;
  int nbsum = 0, ncv = 0, n = 0, nen = 0, niter = 0, tamm_d = 0, nq_blk = 0, nb_max = 0;
  PolyPlan pp;
  double de = 0.0;
  double *de1, *zz0, *sig, *cmn, *cm, *P, *P2, *pn2, *pn, *V, *W, *hs, *tmp, *a, *b, *S;
  double *basis = nullptr;     // Krylov bases (reorth): chain j at basis + j * ldb
  long long ldb = 0;
  double *dgws = nullptr;      // split-K workspace of the start-vector GEMMs
  size_t dgws_bytes = 0;
  int *chb, *chq, *clen, *dlen, *dslot;
  // current block
  int q0 = 0, nq = 0, nb = 0;
  const int *len = nullptr;
  std::vector<int> hb, hq, hl, hslot, order, nact;
};

static int sigma_prepare(SigmaJob &J, ngw_session *s, const ngw_sigma_params *p, const double *e1) {
  NGW_TRY(need_op(s));
  if (!p || !e1 || p->nen < 2 || p->niter < 1 || p->nqp < 1 || !p->qp_bands || p->nval < 1 ||
      p->nval >= s->nmem) {
    set_error("ngw_sigma_lanczos: bad arguments");
    return NGW_ERR_ARG;
  }
  const int nbsum = p->nbands_sum > 0 ? p->nbands_sum : s->nmem;
  if (nbsum > s->nmem) {
    set_error("nbands_sum > nmem");
    return NGW_ERR_ARG;
  }
  for (int i = 0; i < p->nqp; ++i)
    if (p->qp_bands[i] < 1 || p->qp_bands[i] > s->nmem) {
      set_error("qp band %d out of range", p->qp_bands[i]);
      return NGW_ERR_ARG;
    }
  if (p->chain_niter)
    for (int i = 0; i < p->nqp * nbsum; ++i)
      if (p->chain_niter[i] < 1 || p->chain_niter[i] > p->niter) {
        set_error("chain_niter[%d] = %d out of 1..niter", i, p->chain_niter[i]);
        return NGW_ERR_ARG;
      }
  if (!(p->early_exit_eps >= 0.0)) {
    set_error("early_exit_eps must be >= 0");
    return NGW_ERR_ARG;
  }
  if (!all_finite(e1, s->nmem)) {
    set_error("non-finite energies");
    return NGW_ERR_NONFINITE;
  }
  NGW_CUDA(cudaSetDevice(s->device));
  J.s = s;
  J.p = p;
  J.e1 = e1;
  J.nbsum = nbsum;
  J.ncv = s->ncv;
  J.n = s->n_isdf;
  J.nen = p->nen;
  J.niter = p->niter;
  J.tamm_d = p->tamm_d ? 1 : 0;
  // Chebyshev interval of the mixed form: from the operator's eigenpairs
  // unless given (cheb_lo < cheb_hi)
  NGW_TRY(make_plan(s, J.pp, p->polynomial, p->npoly, J.tamm_d, p->cheb_lo, p->cheb_hi, p->niter,
                    p->nqp * nbsum));
  // chain blocking: whole QP states per block
  J.nq_blk = p->nqp;
  if (p->block_chains > 0) J.nq_blk = std::max(1, std::min(p->nqp, p->block_chains / nbsum));
  if (p->reorth) {
    // the Krylov bases of a block's chains must fit the cap: fewer QP states
    // per block when they do not
    if (p->niter > 6000) {
      set_error("reorth: niter %d > 6000", p->niter);
      return NGW_ERR_ARG;
    }
    size_t freeb = 0, totb = 0;
    NGW_CUDA(cudaMemGetInfo(&freeb, &totb));
    double cap = 0.4 * (double)freeb;
    if (const char *e = getenv("NGW_REORTH_MAX_GB")) cap = atof(e) * 1073741824.0;
    const double per_state = (double)nbsum * (p->niter + 1) * (double)s->ncv * 8.0;
    const int fit = (int)std::min<double>(p->nqp, std::floor(cap / per_state));
    if (fit < 1) {
      set_error("reorth: the Krylov bases of one QP state (%.3g bytes) exceed the cap (%.3g bytes)",
                per_state, cap);
      return NGW_ERR_BUDGET;
    }
    J.nq_blk = std::min(J.nq_blk, fit);
  }
  const int nb_max = J.nq_blk * nbsum, ncv = J.ncv, n = J.n, nen = J.nen, niter = J.niter;
  J.nb_max = nb_max;
  NGW_TRY(scratch(s, SL_E1, (size_t)s->nmem * 8, (void **)&J.de1));
  NGW_TRY(scratch(s, SL_ZZ0, (size_t)p->nqp * 8, (void **)&J.zz0));
  NGW_TRY(scratch(s, SL_SIG, (size_t)p->nqp * nen * 16, (void **)&J.sig));
  NGW_TRY(scratch(s, SL_CMN, (size_t)n * nb_max * 8, (void **)&J.cmn));
  NGW_TRY(scratch(s, SL_CM, (size_t)n * nb_max * 8, (void **)&J.cm));
  NGW_TRY(scratch(s, SL_P, (size_t)ncv * nb_max * 8, (void **)&J.P));
  NGW_TRY(scratch(s, SL_P2, (size_t)ncv * nb_max * 8, (void **)&J.P2));
  NGW_TRY(scratch(s, SL_PN2, (size_t)nb_max * 8, (void **)&J.pn2));
  NGW_TRY(scratch(s, SL_PN, (size_t)nb_max * 8, (void **)&J.pn));
  NGW_TRY(scratch(s, SL_WVEC, (size_t)ncv * nb_max * 8, (void **)&J.W));
  NGW_TRY(scratch(s, SL_HS, (size_t)ncv * nb_max * 8, (void **)&J.hs));
  NGW_TRY(scratch(s, SL_TMP, (size_t)ncv * nb_max * 8, (void **)&J.tmp));
  NGW_TRY(scratch(s, SL_A, (size_t)niter * nb_max * 8, (void **)&J.a));
  NGW_TRY(scratch(s, SL_B, (size_t)niter * nb_max * 8, (void **)&J.b));
  NGW_TRY(scratch(s, SL_SPECS, (size_t)(nen + 1) * nb_max * 16, (void **)&J.S));
  NGW_TRY(scratch(s, SL_CHB, (size_t)2 * nb_max * 4, (void **)&J.chb));
  NGW_TRY(scratch(s, SL_CHQ, (size_t)2 * nb_max * 4, (void **)&J.chq));
  NGW_TRY(scratch(s, SL_VEC, (size_t)ncv * nb_max * 8, (void **)&J.V));
  NGW_TRY(scratch(s, SL_CLEN, (size_t)nb_max * 4, (void **)&J.clen));
  NGW_TRY(scratch(s, SL_LEN, (size_t)nb_max * 4, (void **)&J.dlen));
  NGW_TRY(scratch(s, SL_SLOT, (size_t)nb_max * 4, (void **)&J.dslot));
  J.dgws_bytes = (size_t)4 * n * nb_max * 8;   // up to 4 K slices of the N_mu x chains product
  NGW_TRY(scratch(s, SL_DGWS, J.dgws_bytes, (void **)&J.dgws));
  if (p->reorth) {
    J.ldb = (long long)(niter + 1) * ncv;
    NGW_TRY(scratch(s, SL_BASIS, (size_t)nb_max * (size_t)J.ldb * 8, (void **)&J.basis));
  }
  if (s->precision == NGW_PREC_MIXED) {
    NGW_TRY(mixed_prepare_chains(s, nb_max, 0, 0, 0));
    if (J.pp.dense) NGW_TRY(mixed_prepare_dense(s, nb_max));
  }
  NGW_CUDA(cudaMemcpyAsync(J.de1, e1, (size_t)s->nmem * 8, cudaMemcpyHostToDevice, s->stream));
  // energy grid origin per QP state: en0 = e1(m) - deltae/2, step deltae/(nen-1)
  std::vector<double> hz0(p->nqp);
  for (int i = 0; i < p->nqp; ++i) hz0[i] = e1[p->qp_bands[i] - 1] - p->deltae * 0.5;
  J.de = p->deltae / (double)(nen - 1);
  NGW_CUDA(cudaMemcpyAsync(J.zz0, hz0.data(), (size_t)p->nqp * 8, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  J.hb.assign(2 * nb_max, 0);
  J.hq.assign(2 * nb_max, 0);
  J.hl.assign(nb_max, 0);
  J.hslot.assign(nb_max, 0);
  J.order.assign(nb_max, 0);
  return NGW_OK;
}

// Chain tables of the block starting at QP state q0.  Chain o = (iq, n) of the
// block, o = iq*nbsum + n-1: band1 = m (QP band), band2 = n.  With per-chain
// lengths the chains run longest first (stable order): position j holds chain
// order[j], slot[o] is o's position, nact[k] the chains still running at step k.
static int sigma_block_setup(SigmaJob &J, int q0) {
  ngw_session *s = J.s;
  const ngw_sigma_params *p = J.p;
  const int nbsum = J.nbsum, niter = J.niter;
  J.q0 = q0;
  J.nq = std::min(J.nq_blk, p->nqp - q0);
  const int nb = J.nb = J.nq * nbsum;
  for (int o = 0; o < nb; ++o) J.order[o] = o;
  const int *len = J.len = p->chain_niter ? p->chain_niter + (size_t)q0 * nbsum : nullptr;
  if (len)
    std::stable_sort(J.order.begin(), J.order.begin() + nb, [&](int x, int y) { return len[x] > len[y]; });
  for (int j = 0; j < nb; ++j) {
    const int o = J.order[j], iq = o / nbsum, jn = o % nbsum;
    J.hb[j] = p->qp_bands[q0 + iq];
    J.hb[nb + j] = jn + 1;
    J.hq[j] = q0 + iq;
    J.hl[j] = len ? len[o] : niter;
    J.hslot[o] = j;
  }
  J.nact.assign(niter, nb);
  if (len)
    for (int k = 0; k < niter; ++k) {
      int c = 0;
      while (c < nb && J.hl[c] > k) ++c;
      J.nact[k] = c;
    }
  NGW_CUDA(cudaMemcpyAsync(J.chb, J.hb.data(), (size_t)2 * nb * 4, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(J.chq, J.hq.data(), (size_t)nb * 4, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(J.dlen, J.hl.data(), (size_t)nb * 4, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(J.dslot, J.hslot.data(), (size_t)nb * 4, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  return NGW_OK;
}

// The device work of one block, launch-only (graph-capturable), in three
// parts: start vectors and chain set-up, the Lanczos recurrence, spectra and
// the Sigma_c sum.
static int sigma_start(SigmaJob &J) {
  ngw_session *s = J.s;
  const int n = J.n, ncv = J.ncv, nb = J.nb, niter = J.niter, tamm_d = J.tamm_d;
  const double one = 1.0, zero = 0.0;
  // start vectors  P = sqrtR * C^T M (psi_m psi_n)   (F90z:578-709), FP64
  launch_pair_gather_cols(s->d_psi, n, J.chb, J.chb + nb, nb, J.cmn, s->stream);
  NGW_CUDA(dgemm(s->stream, false, false, n, nb, n, one, s->d_M, n, J.cmn, n, zero, J.cm, n, J.dgws,
                 J.dgws_bytes));
  NGW_CUDA(dgemm(s->stream, true, false, ncv, nb, n, one, s->d_C, n, J.cm, n, zero, J.P, ncv, J.dgws,
                 J.dgws_bytes));
  launch_norms(J.P, ncv, nb, s->d_sqrtR, tamm_d, J.P2, J.pn2, s->stream);
  NGW_CUDA(cudaMemsetAsync(J.a, 0, (size_t)niter * nb * 8, s->stream));
  NGW_CUDA(cudaMemsetAsync(J.b, 0, (size_t)niter * nb * 8, s->stream));
  // pnorm = sqrt(pnorm2), v0 = P / pnorm   (F90z:707-709, lanczos_spectra_lowcomsym.F90:68-70)
  launch_sqrt_vec(J.pn2, J.pn, nb, s->stream);
  launch_lanczos_init(J.P2, ncv, J.pn, J.V, J.hs, s->d_sqrtR, ncv, nb, tamm_d, J.b, niter, J.dlen, J.clen,
                      s->stream);
  NGW_CUDA(cudaGetLastError());
  return NGW_OK;
}

static int sigma_end(SigmaJob &J) {
  ngw_session *s = J.s;
  const ngw_sigma_params *p = J.p;
  const int nb = J.nb, niter = J.niter, tamm_d = J.tamm_d;
  launch_sigma_spectra(J.a, J.b, niter, nb, J.de1, J.chb + nb, J.chq, J.zz0, J.de, J.nen, p->ecuts, p->nval,
                       J.S, J.clen, s->stream);
  launch_sigma_reduce(J.S, J.pn2, J.de1, J.chb + nb, J.zz0 + J.q0, J.de, J.nen, p->ecuts, p->nval, J.nbsum,
                      J.nq, tamm_d, J.sig + (size_t)2 * J.q0 * J.nen, 0, J.dslot, s->stream);
  NGW_CUDA(cudaGetLastError());
  return NGW_OK;
}

static int sigma_region(SigmaJob &J) {
  NGW_TRY(sigma_start(J));
  NGW_TRY(lanczos_dev(J.s, J.pp, J.nb, J.niter, J.V, J.W, J.hs, J.tmp, J.a, J.b, J.clen, J.p->early_exit_eps,
                      J.len ? &J.nact : nullptr, J.basis, J.ldb));
  return sigma_end(J);
}

// The Lanczos recurrences of several molecules (mixed precision) in lock
// step, their p(C) v products through grouped GEMM launches (one GEMM1 and
// one GEMM2 launch per Clenshaw term for all molecules still running), the
// per-chain updates per molecule.  Same arithmetic per chain as lanczos_dev
// with the grouped tiles.  Launch-only; everything on stream st.
// Tables of the grouped Lanczos-step launches (steps >= 1): the members'
// vector roles follow the swaps of lanczos_grouped.
struct LanczosGroupTables {
  std::vector<LanczosGroupEntry> tab;   // [steps][G]
  std::vector<int> cb;                  // [steps][G + 1] chain begins
  std::vector<int> tot;                 // chains per launch
  const LanczosGroupEntry *d_tab = nullptr;
  const int *d_cb = nullptr;
};

static void lanczos_group_tables(std::vector<SigmaJob> &jobs, const GroupPlan &P, LanczosGroupTables &T) {
  const int G = (int)jobs.size(), steps = P.steps;
  T.tab.assign((size_t)steps * G, LanczosGroupEntry{});
  T.cb.assign((size_t)steps * (G + 1), 0);
  T.tot.assign(steps, 0);
  std::vector<double *> vec(G), wvec(G);
  for (int i = 0; i < G; ++i) {
    vec[i] = jobs[i].W;
    wvec[i] = jobs[i].V;
  }
  for (int k = 1; k < steps; ++k) {
    int *cbk = T.cb.data() + (size_t)k * (G + 1);
    for (int i = 0; i < G; ++i) {
      SigmaJob &J = jobs[i];
      const int nk = std::max(0, P.nv[(size_t)k * G + i]);
      LanczosGroupEntry &e = T.tab[(size_t)k * G + i];
      e.w = wvec[i];
      e.v = vec[i];
      e.t = J.tmp;
      e.a = J.a;
      e.b = J.b;
      e.s = J.s->d_sqrtR;
      e.clen = J.clen;
      e.eps = J.p->early_exit_eps;
      e.ncv = J.ncv;
      e.niter = J.niter;
      e.prescale_next = (k + 1 < J.niter) ? 1 : 0;
      cbk[i + 1] = cbk[i] + nk;
      if (nk > 0 && k + 1 < J.niter) std::swap(vec[i], wvec[i]);
    }
    T.tot[k] = cbk[G];
  }
}

static int lanczos_grouped(std::vector<SigmaJob> &jobs, std::vector<GroupMember> &mem, const GroupPlan &P,
                           cudaStream_t st, const LanczosGroupTables *LT = nullptr) {
  const int G = (int)jobs.size();
  std::vector<double *> vec(G), wvec(G);
  std::vector<const double *> vin(G);
  for (int i = 0; i < G; ++i) vin[i] = jobs[i].V;
  NGW_TRY(group_poly_apply(P, mem, 0, vin.data(), st));   // W = p(H) V
  for (int i = 0; i < G; ++i) {
    SigmaJob &J = jobs[i];
    ngw_session *s = J.s;
    const double eps = J.p->early_exit_eps;
    if (J.basis) {
      launch_lanczos_reorth_step(J.W, J.V, nullptr, s->ncv, J.nb, 0, J.a, J.b, J.niter, s->d_sqrtR, nullptr, 0,
                                 J.niter >= 2 ? 1 : 0, J.clen, eps, J.basis, J.ldb, st);
    } else {
      launch_lanczos_first(J.W, J.V, s->ncv, J.nb, J.a, J.b, J.niter, J.clen, eps, st);
      if (J.niter >= 2)
        launch_lanczos_prescale(J.W, J.V, s->ncv, P.nv[(size_t)1 * G + i], 1, J.b, J.niter, s->d_sqrtR, nullptr,
                                0, J.clen, st);
    }
    vec[i] = J.W;
    wvec[i] = J.V;
  }
  for (int k = 1; k < P.steps; ++k) {
    bool any = false;
    for (int i = 0; i < G; ++i) {
      vin[i] = vec[i];
      any = any || P.nv[(size_t)k * G + i] > 0;
    }
    if (!any) break;
    NGW_TRY(group_poly_apply(P, mem, k, vin.data(), st));   // tmp = p(H) vec
    if (LT)   // every member's step in one launch
      launch_lanczos_step_grouped(LT->d_tab + (size_t)k * G, LT->d_cb + (size_t)k * (G + 1), G, k, LT->tot[k], st);
    for (int i = 0; i < G; ++i) {
      SigmaJob &J = jobs[i];
      const int nk = P.nv[(size_t)k * G + i];
      if (nk <= 0) continue;
      if (LT) {
        if (k + 1 < J.niter) std::swap(vec[i], wvec[i]);
        continue;
      }
      ngw_session *s = J.s;
      const double eps = J.p->early_exit_eps;
      if (J.basis)
        launch_lanczos_reorth_step(wvec[i], vec[i], J.tmp, s->ncv, nk, k, J.a, J.b, J.niter, s->d_sqrtR, nullptr,
                                   0, (k + 1 < J.niter) ? 1 : 0, J.clen, eps, J.basis, J.ldb, st);
      else
        launch_lanczos_step(wvec[i], vec[i], J.tmp, s->ncv, nk, k, J.a, J.b, J.niter, s->d_sqrtR, nullptr, 0,
                            (k + 1 < J.niter) ? 1 : 0, J.clen, eps, st);
      if (k + 1 < J.niter) std::swap(vec[i], wvec[i]);
    }
  }
  NGW_CUDA(cudaGetLastError());
  return NGW_OK;
}

// Graph key of the current block: every shape, scalar and device address the
// region's launches capture.
static void sigma_key(const SigmaJob &J, std::vector<unsigned long long> &key) {
  ngw_session *s = J.s;
  const ngw_sigma_params *p = J.p;
  const unsigned long long head[] = {
      (unsigned long long)s->precision, (unsigned long long)J.nb, (unsigned long long)J.niter,
      (unsigned long long)J.pp.npoly, (unsigned long long)J.tamm_d, (unsigned long long)J.nen,
      (unsigned long long)p->nval, (unsigned long long)J.nbsum, (unsigned long long)J.nq,
      (unsigned long long)J.q0, (unsigned long long)J.pp.kdef, dbits(p->ecuts), dbits(J.de),
      dbits(J.pp.c0), dbits(J.pp.c1), s->gen, dbits(p->early_exit_eps), (unsigned long long)J.pp.dense,
      (unsigned long long)(J.len != nullptr), (unsigned long long)(uintptr_t)J.basis,
      (unsigned long long)J.ldb};
  key.insert(key.end(), std::begin(head), std::end(head));
  if (J.len) key.insert(key.end(), J.nact.begin(), J.nact.end());
  for (double c : J.pp.poly) key.push_back(dbits(c));
  for (double c : J.pp.cheb) key.push_back(dbits(c));
  for (const void *ptr : {(const void *)J.cmn, (const void *)J.cm, (const void *)J.P, (const void *)J.P2,
                          (const void *)J.pn2, (const void *)J.pn, (const void *)J.V, (const void *)J.W,
                          (const void *)J.hs, (const void *)J.tmp, (const void *)J.a, (const void *)J.b,
                          (const void *)J.S, (const void *)J.chb, (const void *)J.chq, (const void *)J.de1,
                          (const void *)J.zz0, (const void *)J.sig, (const void *)s->mixed,
                          (const void *)J.clen, (const void *)J.dlen, (const void *)J.dslot, (const void *)J.dgws})
    key.push_back((unsigned long long)(uintptr_t)ptr);
  if (s->mixed) {
    int tune[6];
    extern_mixed_tune(s, tune);
    for (int t : tune) key.push_back((unsigned long long)t);
  }
}

// alpha / beta of the current block back in chain order
static int sigma_block_ab(SigmaJob &J, double *alpha, double *beta) {
  ngw_session *s = J.s;
  for (int w = 0; w < 2; ++w) {
    double *dst = w == 0 ? alpha : beta;
    if (!dst) continue;
    std::vector<double> h((size_t)J.niter * J.nb);
    NGW_CUDA(cudaMemcpyAsync(h.data(), w == 0 ? J.a : J.b, (size_t)J.niter * J.nb * 8,
                             cudaMemcpyDeviceToHost, s->stream));
    NGW_CUDA(cudaStreamSynchronize(s->stream));
    for (int o = 0; o < J.nb; ++o)
      std::memcpy(dst + ((size_t)J.q0 * J.nbsum + o) * J.niter, h.data() + (size_t)J.hslot[o] * J.niter,
                  (size_t)J.niter * 8);
  }
  return NGW_OK;
}

static int sigma_finish(SigmaJob &J, double *sigma_c) {
  ngw_session *s = J.s;
  NGW_CUDA(cudaMemcpyAsync(sigma_c, J.sig, (size_t)J.p->nqp * J.nen * 16, cudaMemcpyDeviceToHost, s->stream));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  return check_status(s);
}

}  // namespace ngw

using namespace ngw;

extern "C" {


int ngw_version(void) { return 100; }

const char *ngw_last_error(void) { return g_err; }

int ngw_session_create(int device, ngw_session **out) {
  if (!out) {
    set_error("null out pointer");
    return NGW_ERR_ARG;
  }
  *out = nullptr;
  int ndev = 0;
  NGW_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) {
    set_error("device %d out of range (%d devices)", device, ndev);
    return NGW_ERR_ARG;
  }
  NGW_CUDA(cudaSetDevice(device));
  {
    // keep freed pool memory cached in this process (not returned at each sync)
    cudaMemPool_t pool;
    uint64_t keep = UINT64_MAX;
    NGW_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    NGW_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  ngw_session *s = new ngw_session();
  s->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    set_error("cudaStreamCreate: %s", cudaGetErrorString(e));
    delete s;
    return NGW_ERR_CUDA;
  }
  if (cublasCreate(&s->cublas) != CUBLAS_STATUS_SUCCESS) {
    set_error("cublasCreate failed");
    cudaStreamDestroy(s->stream);
    delete s;
    return NGW_ERR_CUDA;
  }
  cublasSetStream(s->cublas, s->stream);
  cublasSetMathMode(s->cublas, CUBLAS_DEFAULT_MATH);
  // a fixed cuBLAS workspace lets its GEMMs be captured in CUDA graphs
  if (dalloc(s, &s->cublas_ws, 64ull << 20) != NGW_OK) {
    ngw_session_destroy(s);
    return NGW_ERR_OOM;
  }
  cublasSetWorkspace(s->cublas, s->cublas_ws, 64ull << 20);
  if (dalloc(s, (void **)&s->d_status, sizeof(int)) != NGW_OK) {
    ngw_session_destroy(s);
    return NGW_ERR_OOM;
  }
  cudaMemset(s->d_status, 0, sizeof(int));
  *out = s;
  return NGW_OK;
}

void ngw_session_destroy(ngw_session *s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (auto &g : s->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (s->stream) {   // frees are queued on the session stream, before it goes
    mixed_free(s);
    for (auto &b : s->scratch) pool_free(s, b.p);
    pool_free(s, s->cublas_ws);
    void *ptrs[] = {s->d_psi, s->d_M, s->d_Mxc, s->d_cvpair, s->d_sqrtR, s->d_C, s->d_status, s->eig_U};
    for (void *p : ptrs) pool_free(s, p);
    cudaStreamSynchronize(s->stream);
  }
  if (s->cublas) cublasDestroy(s->cublas);
  if (s->cusolver) cusolverDnDestroy((cusolverDnHandle_t)s->cusolver);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

void *ngw_session_stream(ngw_session *s) { return s ? (void *)s->stream : nullptr; }

long long ngw_session_bytes(ngw_session *s) { return s ? (long long)s->bytes : 0; }

int ngw_set_precision(ngw_session *s, int mode) {
  if (!s || (mode != NGW_PREC_FP64 && mode != NGW_PREC_MIXED)) {
    set_error("bad precision mode %d", mode);
    return NGW_ERR_ARG;
  }
  NGW_CUDA(cudaSetDevice(s->device));
  s->precision = mode;
  return NGW_OK;
}

int ngw_set_isdf(ngw_session *s, int n_isdf, int nmem, const double *psi_intp, const double *mmtrx,
                 const double *mxc) {
  if (!s || n_isdf <= 0 || nmem <= 0 || !psi_intp || !mmtrx) {
    set_error("ngw_set_isdf: bad arguments");
    return NGW_ERR_ARG;
  }
  if (!all_finite(psi_intp, (size_t)n_isdf * nmem) || !all_finite(mmtrx, (size_t)n_isdf * n_isdf) ||
      (mxc && !all_finite(mxc, (size_t)n_isdf * n_isdf))) {
    set_error("ngw_set_isdf: non-finite input");
    return NGW_ERR_NONFINITE;
  }
  NGW_CUDA(cudaSetDevice(s->device));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  // Same shapes: the new values go into the existing buffers, so captured
  // graphs (which hold buffer addresses) stay valid; every value derived from
  // the operator (pair products, eigenpairs, split-BF16 operands) is rebuilt.
  const bool same = s->have_isdf && s->n_isdf == n_isdf && s->nmem == nmem &&
                    (mxc != nullptr) == (s->d_Mxc != nullptr);
  if (!same) {
    bump_generation(s);
    mixed_free(s);
    if (s->d_psi) dfree(s, s->d_psi, (size_t)s->n_isdf * s->nmem * 8);
    if (s->d_M) dfree(s, s->d_M, (size_t)s->n_isdf * s->n_isdf * 8);
    if (s->d_Mxc) dfree(s, s->d_Mxc, (size_t)s->n_isdf * s->n_isdf * 8);
    if (s->d_C) dfree(s, s->d_C, (size_t)s->n_isdf * s->ncv * 8);
    s->d_psi = s->d_M = s->d_Mxc = s->d_C = nullptr;
    s->n_isdf = n_isdf;
    s->nmem = nmem;
    NGW_TRY(dalloc(s, (void **)&s->d_psi, (size_t)n_isdf * nmem * 8));
    NGW_TRY(dalloc(s, (void **)&s->d_M, (size_t)n_isdf * n_isdf * 8));
    if (mxc) NGW_TRY(dalloc(s, (void **)&s->d_Mxc, (size_t)n_isdf * n_isdf * 8));
    if (s->have_pairs) NGW_TRY(dalloc(s, (void **)&s->d_C, (size_t)n_isdf * s->ncv * 8));
  } else {
    s->mixed_dirty = true;
  }
  s->have_C = false;
  s->eig_tda = -1;
  NGW_CUDA(cudaMemcpyAsync(s->d_psi, psi_intp, (size_t)n_isdf * nmem * 8, cudaMemcpyHostToDevice,
                           s->stream));
  NGW_CUDA(cudaMemcpyAsync(s->d_M, mmtrx, (size_t)n_isdf * n_isdf * 8, cudaMemcpyHostToDevice,
                           s->stream));
  if (mxc)
    NGW_CUDA(cudaMemcpyAsync(s->d_Mxc, mxc, (size_t)n_isdf * n_isdf * 8, cudaMemcpyHostToDevice,
                             s->stream));
  s->have_isdf = true;
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  return NGW_OK;
}

int ngw_set_pairs(ngw_session *s, int ncv, const int *cvpair, const double *sqrtR) {
  if (!s || ncv <= 0 || !cvpair || !sqrtR) {
    set_error("ngw_set_pairs: bad arguments");
    return NGW_ERR_ARG;
  }
  if (s->have_isdf) {
    for (int i = 0; i < 2 * ncv; ++i) {
      if (cvpair[i] < 1 || cvpair[i] > s->nmem) {
        set_error("ngw_set_pairs: band index %d out of 1..%d", cvpair[i], s->nmem);
        return NGW_ERR_ARG;
      }
    }
  }
  if (!all_finite(sqrtR, ncv)) {
    set_error("ngw_set_pairs: non-finite sqrtR");
    return NGW_ERR_NONFINITE;
  }
  NGW_CUDA(cudaSetDevice(s->device));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  const bool same = s->have_pairs && s->ncv == ncv && (!s->have_isdf || s->d_C);
  if (!same) {
    bump_generation(s);
    mixed_free(s);
    if (s->d_cvpair) dfree(s, s->d_cvpair, (size_t)2 * s->ncv * 4);
    if (s->d_sqrtR) dfree(s, s->d_sqrtR, (size_t)s->ncv * 8);
    if (s->d_C) dfree(s, s->d_C, (size_t)s->n_isdf * s->ncv * 8);
    s->d_C = nullptr;
    s->ncv = ncv;
    NGW_TRY(dalloc(s, (void **)&s->d_cvpair, (size_t)2 * ncv * 4));
    NGW_TRY(dalloc(s, (void **)&s->d_sqrtR, (size_t)ncv * 8));
    if (s->have_isdf) NGW_TRY(dalloc(s, (void **)&s->d_C, (size_t)s->n_isdf * ncv * 8));
  } else {
    s->mixed_dirty = true;
  }
  s->have_C = false;
  s->eig_tda = -1;
  NGW_CUDA(cudaMemcpyAsync(s->d_cvpair, cvpair, (size_t)2 * ncv * 4, cudaMemcpyHostToDevice,
                           s->stream));
  NGW_CUDA(cudaMemcpyAsync(s->d_sqrtR, sqrtR, (size_t)ncv * 8, cudaMemcpyHostToDevice, s->stream));
  s->have_pairs = true;
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  return NGW_OK;
}

int ngw_matvec_isdf(ngw_session *s, const double *vec, double *hvec, int ld, int blksz,
                    int tamm_d) {
  NGW_TRY(need_op(s));
  if (!vec || !hvec || blksz <= 0 || ld < s->ncv) {
    set_error("ngw_matvec_isdf: bad arguments");
    return NGW_ERR_ARG;
  }
  NGW_CUDA(cudaSetDevice(s->device));
  const int ncv = s->ncv, nb = blksz;
  double *din, *dout, *hs;
  NGW_TRY(scratch(s, SL_IN, (size_t)ncv * nb * 8, (void **)&din));
  NGW_TRY(scratch(s, SL_OUT, (size_t)ncv * nb * 8, (void **)&dout));
  NGW_TRY(scratch(s, SL_HS, (size_t)ncv * nb * 8, (void **)&hs));
  NGW_CUDA(cudaMemcpy2DAsync(din, (size_t)ncv * 8, vec, (size_t)ld * 8, (size_t)ncv * 8, nb,
                             cudaMemcpyHostToDevice, s->stream));
  if (s->precision == NGW_PREC_MIXED) {
    // one matvec in mixed precision: the degree-1 series p(x) = x
    PolyPlan pp;
    const double px[2] = {1.0, 0.0};
    NGW_TRY(make_plan(s, pp, px, 1, tamm_d ? 1 : 0, 0.0, 0.0));
    NGW_TRY(mixed_prepare_chains(s, nb, 0, 0, 0));
    const double g[2] = {pp.c0, pp.c1};
    NGW_TRY(mixed_poly_apply(s, nb, din, ncv, g, 1, pp.c0, pp.c1, tamm_d ? 1 : 0, dout));
  } else {
    launch_scale_rows(s->d_sqrtR, din, ncv, hs, ncv, ncv, nb, tamm_d, s->stream);
    NGW_TRY(matvec_f64_dev(s, nb, hs, dout, din, tamm_d, 0, 0.0, 0.0, nullptr));
  }
  NGW_CUDA(cudaMemcpy2DAsync(hvec, (size_t)ld * 8, dout, (size_t)ncv * 8, (size_t)ncv * 8, nb,
                             cudaMemcpyDeviceToHost, s->stream));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  return check_status(s);
}

int ngw_polynomial_matvec_isdf(ngw_session *s, const double *polynomial, int npoly,
                               const double *vec, double *hvec, int ld, int blksz) {
  NGW_TRY(need_op(s));
  if (!vec || !hvec || blksz <= 0 || ld < s->ncv || !polynomial || npoly < 1) {
    set_error("ngw_polynomial_matvec_isdf: bad arguments");
    return NGW_ERR_ARG;
  }
  NGW_CUDA(cudaSetDevice(s->device));
  const int ncv = s->ncv, nb = blksz;
  double *din, *dout, *hs;
  NGW_TRY(scratch(s, SL_IN, (size_t)ncv * nb * 8, (void **)&din));
  NGW_TRY(scratch(s, SL_OUT, (size_t)ncv * nb * 8, (void **)&dout));
  NGW_TRY(scratch(s, SL_HS, (size_t)ncv * nb * 8, (void **)&hs));
  NGW_CUDA(cudaMemcpy2DAsync(din, (size_t)ncv * 8, vec, (size_t)ld * 8, (size_t)ncv * 8, nb,
                             cudaMemcpyHostToDevice, s->stream));
  // the explicit Horner form of the reference, always in FP64
  launch_scale_rows(s->d_sqrtR, din, ncv, hs, ncv, ncv, nb, 0, s->stream);
  NGW_TRY(poly_f64_dev(s, nb, polynomial, npoly, din, hs, dout));
  NGW_CUDA(cudaMemcpy2DAsync(hvec, (size_t)ld * 8, dout, (size_t)ncv * 8, (size_t)ncv * 8, nb,
                             cudaMemcpyDeviceToHost, s->stream));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  return check_status(s);
}

int ngw_lanczos_spectra_isdf(ngw_session *s, const double *v0, const double *v0_norm, int ld,
                             const double *zz, int nz, int niter, const double *polynomial,
                             int npoly, int blksz, int tamm_d, double *spectra, double *alpha,
                             double *beta) {
  return ngw_lanczos_spectra_isdf_masked(s, v0, v0_norm, ld, zz, nz, niter, polynomial, npoly, blksz,
                                         tamm_d, nullptr, 0.0, spectra, alpha, beta);
}

int ngw_lanczos_spectra_isdf_masked(ngw_session *s, const double *v0, const double *v0_norm, int ld,
                                    const double *zz, int nz, int niter, const double *polynomial,
                                    int npoly, int blksz, int tamm_d, const int *chain_niter,
                                    double early_exit_eps, double *spectra, double *alpha,
                                    double *beta) {
  NGW_TRY(need_op(s));
  if (!v0 || !v0_norm || !zz || !spectra || nz <= 0 || niter <= 0 || blksz <= 0 || ld < s->ncv ||
      !(early_exit_eps >= 0.0)) {
    set_error("ngw_lanczos_spectra_isdf: bad arguments");
    return NGW_ERR_ARG;
  }
  if (chain_niter)
    for (int j = 0; j < blksz; ++j)
      if (chain_niter[j] < 1 || chain_niter[j] > niter) {
        set_error("chain_niter[%d] = %d out of 1..niter", j, chain_niter[j]);
        return NGW_ERR_ARG;
      }
  NGW_CUDA(cudaSetDevice(s->device));
  const int ncv = s->ncv, nb = blksz;
  PolyPlan pp;
  NGW_TRY(make_plan(s, pp, polynomial, npoly, tamm_d, 0.0, 0.0, niter, blksz));
  double *dv0, *V, *W, *hs, *tmp, *a, *b, *dzz, *dspec, *dnorm;
  NGW_TRY(scratch(s, SL_IN, (size_t)ncv * nb * 8, (void **)&dv0));
  NGW_TRY(scratch(s, SL_VEC, (size_t)ncv * nb * 8, (void **)&V));
  NGW_TRY(scratch(s, SL_WVEC, (size_t)ncv * nb * 8, (void **)&W));
  NGW_TRY(scratch(s, SL_HS, (size_t)ncv * nb * 8, (void **)&hs));
  NGW_TRY(scratch(s, SL_TMP, (size_t)ncv * nb * 8, (void **)&tmp));
  NGW_TRY(scratch(s, SL_A, (size_t)niter * nb * 8, (void **)&a));
  NGW_TRY(scratch(s, SL_B, (size_t)niter * nb * 8, (void **)&b));
  NGW_TRY(scratch(s, SL_ZZ, (size_t)nz * nb * 16, (void **)&dzz));
  NGW_TRY(scratch(s, SL_SPEC, (size_t)nz * nb * 16, (void **)&dspec));
  NGW_TRY(scratch(s, SL_PN, (size_t)nb * 8, (void **)&dnorm));
  int *clen = nullptr, *dlen = nullptr;
  NGW_TRY(scratch(s, SL_CLEN, (size_t)nb * 4, (void **)&clen));
  if (chain_niter) {
    NGW_TRY(scratch(s, SL_LEN, (size_t)nb * 4, (void **)&dlen));
    NGW_CUDA(cudaMemcpyAsync(dlen, chain_niter, (size_t)nb * 4, cudaMemcpyHostToDevice, s->stream));
  }
  if (s->precision == NGW_PREC_MIXED) {
    NGW_TRY(mixed_prepare_chains(s, nb, 0, 0, 0));
    if (pp.dense) NGW_TRY(mixed_prepare_dense(s, nb));
  }
  NGW_CUDA(cudaMemcpy2DAsync(dv0, (size_t)ncv * 8, v0, (size_t)ld * 8, (size_t)ncv * 8, nb,
                             cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(dnorm, v0_norm, (size_t)nb * 8, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(dzz, zz, (size_t)nz * nb * 16, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemsetAsync(b, 0, (size_t)niter * nb * 8, s->stream));
  NGW_CUDA(cudaMemsetAsync(a, 0, (size_t)niter * nb * 8, s->stream));
  launch_lanczos_init(dv0, ncv, dnorm, V, hs, s->d_sqrtR, ncv, nb, tamm_d, b, niter, dlen, clen,
                      s->stream);
  NGW_TRY(lanczos_dev(s, pp, nb, niter, V, W, hs, tmp, a, b, clen, early_exit_eps, nullptr));
  launch_contfrac(a, b, niter, nb, dzz, nz, dspec, clen, s->stream);
  NGW_CUDA(cudaGetLastError());
  NGW_CUDA(cudaMemcpyAsync(spectra, dspec, (size_t)nz * nb * 16, cudaMemcpyDeviceToHost, s->stream));
  if (alpha)
    NGW_CUDA(cudaMemcpyAsync(alpha, a, (size_t)niter * nb * 8, cudaMemcpyDeviceToHost, s->stream));
  if (beta)
    NGW_CUDA(cudaMemcpyAsync(beta, b, (size_t)niter * nb * 8, cudaMemcpyDeviceToHost, s->stream));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  return check_status(s);
}

int ngw_k_integrate_isdf(ngw_session *s, int kflag, const int *rows, int nrow, const int *cols,
                         int ncol, double *kmat) {
  if (!s || !s->have_isdf) {
    set_error("ISDF operator not set");
    return NGW_ERR_STATE;
  }
  if (!rows || !cols || !kmat || nrow <= 0 || ncol <= 0 || kflag < 0 || kflag > 2) {
    set_error("ngw_k_integrate_isdf: bad arguments");
    return NGW_ERR_ARG;
  }
  if (kflag > 0 && !s->d_Mxc) {
    set_error("kflag > 0 needs the f_xc kernel block");
    return NGW_ERR_STATE;
  }
  for (int i = 0; i < 2 * nrow; ++i)
    if (rows[i] < 1 || rows[i] > s->nmem) { set_error("row band out of range"); return NGW_ERR_ARG; }
  for (int i = 0; i < 2 * ncol; ++i)
    if (cols[i] < 1 || cols[i] > s->nmem) { set_error("col band out of range"); return NGW_ERR_ARG; }
  NGW_CUDA(cudaSetDevice(s->device));
  const int n = s->n_isdf;
  std::vector<int> r1(nrow), r2(nrow), c1(ncol), c2(ncol);
  for (int i = 0; i < nrow; ++i) { r1[i] = rows[2 * i]; r2[i] = rows[2 * i + 1]; }
  for (int i = 0; i < ncol; ++i) { c1[i] = cols[2 * i]; c2[i] = cols[2 * i + 1]; }
  int *db;
  double *cr, *cc, *km, *tmp, *out;
  NGW_TRY(scratch(s, SL_B1, (size_t)2 * (nrow + ncol) * 4, (void **)&db));
  NGW_TRY(scratch(s, SL_KR, (size_t)n * nrow * 8, (void **)&cr));
  NGW_TRY(scratch(s, SL_KC, (size_t)n * ncol * 8, (void **)&cc));
  NGW_TRY(scratch(s, SL_KM, (size_t)n * n * 8, (void **)&km));
  NGW_TRY(scratch(s, SL_T1, (size_t)n * nrow * 8, (void **)&tmp));
  NGW_TRY(scratch(s, SL_OUT, (size_t)nrow * ncol * 8, (void **)&out));
  NGW_CUDA(cudaMemcpyAsync(db, r1.data(), nrow * 4, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(db + nrow, r2.data(), nrow * 4, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(db + 2 * nrow, c1.data(), ncol * 4, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(db + 2 * nrow + ncol, c2.data(), ncol * 4, cudaMemcpyHostToDevice, s->stream));
  launch_pair_gather_cols(s->d_psi, n, db, db + nrow, nrow, cr, s->stream);
  launch_pair_gather_cols(s->d_psi, n, db + 2 * nrow, db + 2 * nrow + ncol, ncol, cc, s->stream);
  launch_k_combine(s->d_M, s->d_Mxc, n, kflag, km, s->stream);
  const double one = 1.0, zero = 0.0;
  NGW_CUDA(dgemm(s->stream, false, false, n, nrow, n, one, km, n, cr, n, zero, tmp, n));
  NGW_CUDA(dgemm(s->stream, true, false, nrow, ncol, n, one, tmp, n, cc, n, zero, out, nrow));
  NGW_CUDA(cudaMemcpyAsync(kmat, out, (size_t)nrow * ncol * 8, cudaMemcpyDeviceToHost, s->stream));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  return check_status(s);
}

int ngw_sigma_lanczos(ngw_session *s, const ngw_sigma_params *p, const double *e1,
                      double *sigma_c, double *alpha, double *beta) {
  if (!s) {
    set_error("ngw_sigma_lanczos: null session");
    return NGW_ERR_ARG;
  }
  PhaseTimer tm(s);
  SigmaJob J;
  NGW_TRY(sigma_prepare(J, s, p, e1));
  tm.mark("plan");
  std::shared_lock<std::shared_mutex> busy(gpu_quiet_lock(s->device));   // no tuning meanwhile
  for (int q0 = 0; q0 < p->nqp; q0 += J.nq_blk) {
    NGW_TRY(sigma_block_setup(J, q0));
    std::vector<unsigned long long> key;
    sigma_key(J, key);
    tm.mark("block_setup");
    NGW_TRY(run_graphed(s, key, [&]() { return sigma_region(J); }));
    tm.mark("region");
    NGW_TRY(sigma_block_ab(J, alpha, beta));
  }
  return sigma_finish(J, sigma_c);
}

int ngw_sigma_lanczos_batch(ngw_session *const *sessions, int count, const ngw_sigma_params *params,
                            const double *const *e1, double *const *sigma_c) {
  if (!sessions || count < 1 || !params || !e1 || !sigma_c) {
    set_error("ngw_sigma_lanczos_batch: bad arguments");
    return NGW_ERR_ARG;
  }
  for (int i = 0; i < count; ++i) {
    if (!sessions[i] || !e1[i] || !sigma_c[i]) {
      set_error("ngw_sigma_lanczos_batch: entry %d is null", i);
      return NGW_ERR_ARG;
    }
    if (sessions[i]->device != sessions[0]->device) {
      set_error("ngw_sigma_lanczos_batch: sessions on different devices");
      return NGW_ERR_ARG;
    }
    for (int k = 0; k < i; ++k)
      if (sessions[k] == sessions[i]) {
        set_error("ngw_sigma_lanczos_batch: session %d appears twice", i);
        return NGW_ERR_ARG;
      }
  }
  std::vector<SigmaJob> jobs(count);
  for (int i = 0; i < count; ++i) {
    NGW_TRY(sigma_prepare(jobs[i], sessions[i], &params[i], e1[i]));
    if (jobs[i].nq_blk < params[i].nqp) {
      set_error("ngw_sigma_lanczos_batch: entry %d needs %d chain blocks (one per entry allowed)", i,
                (params[i].nqp + jobs[i].nq_blk - 1) / jobs[i].nq_blk);
      return NGW_ERR_ARG;
    }
    NGW_TRY(sigma_block_setup(jobs[i], 0));
  }
  ngw_session *s0 = sessions[0];
  // Entries run as graph branches on their own streams with their tuned
  // tiles (the default: measured fastest, the branches of small molecules
  // overlap on the GPU).  NGW_BATCH_MODE=grouped_small groups the small
  // mixed-precision molecules (N_cv <= 8192, N_mu <= 512, not TDA, one
  // polynomial degree, factored p(C): entries whose plan chose the dense
  // operator stay branches), NGW_BATCH_MODE=grouped every eligible molecule: their
  // Lanczos recurrences in lock step on one stream, each Clenshaw term of
  // their p(C) v one grouped GEMM1 and one grouped GEMM2 launch over all of
  // them, one grouped step launch per Lanczos step, the other entries as
  // branches beside the group.
  int mode = 1;   // 0 small only, 1 none, 2 every eligible entry
  if (const char *e = getenv("NGW_BATCH_MODE")) {
    if (std::string(e) == "grouped_small") mode = 0;
    if (std::string(e) == "grouped") mode = 2;
  }
  std::vector<int> grp, br;
  for (int i = 0; i < count; ++i) {
    const SigmaJob &J = jobs[i];
    const bool eligible = mode != 1 && sessions[i]->precision == NGW_PREC_MIXED && !J.tamm_d && !J.pp.dense &&
                          (int)J.pp.cheb.size() == J.pp.npoly + 1 &&
                          (grp.empty() || J.pp.npoly == jobs[grp[0]].pp.npoly) &&
                          (mode == 2 || (J.ncv <= 8192 && J.n <= 512));
    (eligible ? grp : br).push_back(i);
  }
  if (grp.size() < 2) {
    br.insert(br.end(), grp.begin(), grp.end());
    std::sort(br.begin(), br.end());
    grp.clear();
  }
  const int G = (int)grp.size();
  std::vector<SigmaJob> gjobs;
  for (int i : grp) gjobs.push_back(jobs[i]);
  std::vector<std::vector<int>> nact(G);
  std::vector<GroupMember> mem(G);
  GroupPlan P;
  LanczosGroupTables LT;
  bool any_reorth = false;
  ngw_session *sg = G ? sessions[grp[0]] : nullptr;   // the group runs on this session's stream
  std::vector<unsigned long long> key = {0xBA7C5ull, (unsigned long long)count, (unsigned long long)G};
  if (G) {
    int steps = 0;
    for (auto &J : gjobs) steps = std::max(steps, J.niter);
    for (int i = 0; i < G; ++i) {
      SigmaJob &J = gjobs[i];
      nact[i].assign(steps, 0);
      for (int k = 0; k < J.niter; ++k) nact[i][k] = J.len ? J.nact[k] : J.nb;
      mem[i] = GroupMember{J.s, J.pp.cheb.data(), J.pp.c0, J.pp.c1, J.ncv, J.W, J.tmp, J.nb, nact[i].data()};
    }
    const int n = gjobs[0].pp.npoly;
    void *buf = nullptr;
    NGW_TRY(scratch(sg, SL_GROUP, group_bytes(G, n, steps), &buf));
    NGW_TRY(group_build(mem, n, 0, steps, buf, sg->stream, P));
    // one Lanczos-step launch per step for all members (none reorthogonalises)
    for (auto &J : gjobs) any_reorth = any_reorth || J.basis != nullptr;
    if (!any_reorth) {
      lanczos_group_tables(gjobs, P, LT);
      const size_t tb = LT.tab.size() * sizeof(LanczosGroupEntry), cbb = LT.cb.size() * sizeof(int);
      void *lbuf = nullptr;
      NGW_TRY(scratch(sg, SL_LGROUP, tb + cbb + 256, &lbuf));
      LT.d_tab = static_cast<const LanczosGroupEntry *>(lbuf);
      LT.d_cb = reinterpret_cast<const int *>(static_cast<char *>(lbuf) + tb);
      NGW_CUDA(cudaMemcpyAsync(lbuf, LT.tab.data(), tb, cudaMemcpyHostToDevice, sg->stream));
      NGW_CUDA(cudaMemcpyAsync(static_cast<char *>(lbuf) + tb, LT.cb.data(), cbb, cudaMemcpyHostToDevice,
                               sg->stream));
      NGW_CUDA(cudaStreamSynchronize(sg->stream));
    }
    key.push_back((unsigned long long)(uintptr_t)buf);
    key.push_back((unsigned long long)(uintptr_t)LT.d_tab);
  }
  for (int i = 0; i < count; ++i) {
    key.push_back((unsigned long long)(uintptr_t)sessions[i]);
    key.push_back((unsigned long long)(uintptr_t)sessions[i]->cublas_ws);
    sigma_key(jobs[i], key);
  }
  // the group on sg's stream and every other entry on its own stream, all
  // forked from and joined back into session 0's stream
  std::vector<cudaEvent_t> ev(count + 2, nullptr);
  for (auto &e : ev) NGW_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  std::vector<cudaStream_t> saved(count);
  for (int i = 0; i < count; ++i) saved[i] = sessions[i]->stream;
  cudaStream_t gst = sg ? sg->stream : nullptr;
  for (int i : grp) sessions[i]->stream = gst;      // every launch of the group on one stream
  auto region = [&]() -> int {
    NGW_CUDA(cudaEventRecord(ev[count], s0->stream));
    if (G) {
      if (gst != s0->stream) NGW_CUDA(cudaStreamWaitEvent(gst, ev[count], 0));
      for (auto &J : gjobs) NGW_TRY(sigma_start(J));
      NGW_TRY(lanczos_grouped(gjobs, mem, P, gst, any_reorth ? nullptr : &LT));
      for (auto &J : gjobs) NGW_TRY(sigma_end(J));
      if (gst != s0->stream) {
        NGW_CUDA(cudaEventRecord(ev[count + 1], gst));
        NGW_CUDA(cudaStreamWaitEvent(s0->stream, ev[count + 1], 0));
      }
    }
    for (int i : br) {
      ngw_session *si = sessions[i];
      if (si->stream != s0->stream) NGW_CUDA(cudaStreamWaitEvent(si->stream, ev[count], 0));
      NGW_TRY(sigma_region(jobs[i]));
      if (si->stream != s0->stream) {
        NGW_CUDA(cudaEventRecord(ev[i], si->stream));
        NGW_CUDA(cudaStreamWaitEvent(s0->stream, ev[i], 0));
      }
    }
    return NGW_OK;
  };
  int rc;
  {
    std::shared_lock<std::shared_mutex> busy(gpu_quiet_lock(s0->device));   // no tuning meanwhile
    rc = run_graphed(s0, key, region);
    if (rc == NGW_OK && cudaStreamSynchronize(s0->stream) != cudaSuccess) {
      set_error("ngw_sigma_lanczos_batch: %s", cudaGetErrorString(cudaGetLastError()));
      rc = NGW_ERR_CUDA;
    }
  }
  for (int i = 0; i < count; ++i) sessions[i]->stream = saved[i];
  for (auto &e : ev) cudaEventDestroy(e);
  NGW_TRY(rc);
  for (int i = 0; i < count; ++i) NGW_TRY(sigma_finish(jobs[i], sigma_c[i]));
  return NGW_OK;
}

int ngw_qp_newton(ngw_session *s, int nqp, int nen, const double *sigma_c_ev, const double *e1_ev,
                  const double *e0_ev, double deltae_ev, const double *sigx_ev,
                  const double *vxc_ev, double xacc_ev, double *eqp_ev, double *zfac, int *ierr) {
  if (!s || nqp <= 0 || nen < 4 || !sigma_c_ev || !e1_ev || !e0_ev || !sigx_ev || !vxc_ev ||
      !eqp_ev || !zfac || !ierr) {
    set_error("ngw_qp_newton: bad arguments");
    return NGW_ERR_ARG;
  }
  NGW_CUDA(cudaSetDevice(s->device));
  double *dsig, *io, *w;
  NGW_TRY(scratch(s, SL_SIG, (size_t)nqp * nen * 16, (void **)&dsig));
  NGW_TRY(scratch(s, SL_QPIO, (size_t)nqp * 6 * 8 + (size_t)nqp * 4, (void **)&io));
  NGW_TRY(scratch(s, SL_QPW, (size_t)nqp * 4 * nen * 8, (void **)&w));
  double *d_e1 = io, *d_e0 = io + nqp, *d_sx = io + 2 * nqp, *d_vx = io + 3 * nqp;
  double *d_eq = io + 4 * nqp, *d_z = io + 5 * nqp;
  int *d_err = reinterpret_cast<int *>(io + 6 * nqp);
  NGW_CUDA(cudaMemcpyAsync(dsig, sigma_c_ev, (size_t)nqp * nen * 16, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(d_e1, e1_ev, nqp * 8, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(d_e0, e0_ev, nqp * 8, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(d_sx, sigx_ev, nqp * 8, cudaMemcpyHostToDevice, s->stream));
  NGW_CUDA(cudaMemcpyAsync(d_vx, vxc_ev, nqp * 8, cudaMemcpyHostToDevice, s->stream));
  launch_qp_newton_ws(nqp, nen, dsig, d_e1, d_e0, deltae_ev, d_sx, d_vx, xacc_ev, d_eq, d_z, d_err,
                      w, s->stream);
  NGW_CUDA(cudaGetLastError());
  NGW_CUDA(cudaMemcpyAsync(eqp_ev, d_eq, nqp * 8, cudaMemcpyDeviceToHost, s->stream));
  NGW_CUDA(cudaMemcpyAsync(zfac, d_z, nqp * 8, cudaMemcpyDeviceToHost, s->stream));
  NGW_CUDA(cudaMemcpyAsync(ierr, d_err, nqp * 4, cudaMemcpyDeviceToHost, s->stream));
  NGW_CUDA(cudaStreamSynchronize(s->stream));
  return check_status(s);
}

}  // extern "C"

extern "C" int ngw_operator_eigenpairs(ngw_session *s, int tamm_d, int msteps, int kmax, double *vals,
                                       double *res, int *count) {
  using namespace ngw;
  if (!vals || !res || !count || msteps < 1 || kmax < 1 || (tamm_d != 0 && tamm_d != 1)) {
    set_error("ngw_operator_eigenpairs: bad arguments");
    return NGW_ERR_ARG;
  }
  NGW_TRY(need_op(s));   // the FP64 pair products are gathered on first use
  NGW_TRY(compute_top_eigs(s, tamm_d, kmax, msteps));
  const int k = std::min(kmax, (int)s->eig_vals.size());
  for (int i = 0; i < k; ++i) {
    vals[i] = s->eig_vals[i];
    res[i] = s->eig_res[i];
  }
  *count = k;
  // the mixed-precision plan recomputes its own eigenpairs (and operator)
  s->eig_tda = -1;
  s->mixed_dirty = true;
  return NGW_OK;
}

// FP64 kernels of the ISDF-Lanczos GW path: pair gather, the matvec's
// diagonal combine + Horner step, the Lanczos recurrence (one CTA per chain,
// warp-shuffle reductions), the continued fraction, the Sigma_c accumulation
// and the QP Newton solve.  All vectors are column blocks (ncv, nb) with the
// pair index fastest, i.e. one chain's vector is contiguous.
#include "ngw_internal.h"

#include <algorithm>
#include <cmath>

namespace ngw {

static inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// pair products C(mu, icv) = psi(mu, c) * psi(mu, v)
// (shared/apply_matvec_lowcomsym.F90:209-210, hadamard_prod_mat_sym.cpp:3-17)
// 128-bit loads along mu when n_isdf is even (columns stay 16-byte aligned).
__global__ void k_pair_gather_f64(const double *__restrict__ psi, int n_isdf,
                                  const int *__restrict__ cvpair, int ncv,
                                  double *__restrict__ C) {
  for (int cv = blockIdx.y; cv < ncv; cv += gridDim.y) {
    const int v = cvpair[2 * cv] - 1, c = cvpair[2 * cv + 1] - 1;
    const double *pv = psi + (size_t)v * n_isdf;
    const double *pc = psi + (size_t)c * n_isdf;
    double *out = C + (size_t)cv * n_isdf;
    if ((n_isdf & 1) == 0) {
      const int n2 = n_isdf >> 1;
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += gridDim.x * blockDim.x) {
        double2 a = reinterpret_cast<const double2 *>(pc)[i];
        double2 b = reinterpret_cast<const double2 *>(pv)[i];
        reinterpret_cast<double2 *>(out)[i] = make_double2(a.x * b.x, a.y * b.y);
      }
    } else {
      for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_isdf; i += gridDim.x * blockDim.x)
        out[i] = pc[i] * pv[i];
    }
  }
}

void launch_pair_gather_f64(const double *psi, int n_isdf, const int *cvpair, int ncv,
                            double *C, cudaStream_t st) {
  if (ncv <= 0) return;
  int threads = 128;
  int bx = cdiv((n_isdf + 1) / 2, threads);
  if (bx > 8) bx = 8;
  dim3 grid(bx, ygrid(ncv));
  k_pair_gather_f64<<<grid, threads, 0, st>>>(psi, n_isdf, cvpair, ncv, C);
}

// out(:, j) = psi(:, b1(j)) * psi(:, b2(j))  (start vectors C_mn, k_integrate)
__global__ void k_pair_gather_cols(const double *__restrict__ psi, int n_isdf,
                                   const int *__restrict__ b1, const int *__restrict__ b2, int n,
                                   double *__restrict__ out) {
  for (int j = blockIdx.y; j < n; j += gridDim.y) {
    const double *p1 = psi + (size_t)(b1[j] - 1) * n_isdf;
    const double *p2 = psi + (size_t)(b2[j] - 1) * n_isdf;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_isdf; i += gridDim.x * blockDim.x)
      out[(size_t)j * n_isdf + i] = p1[i] * p2[i];
  }
}

void launch_pair_gather_cols(const double *psi, int n_isdf, const int *b1, const int *b2, int n,
                             double *out, cudaStream_t st) {
  if (n <= 0) return;
  int bx = cdiv(n_isdf, 128);
  if (bx > 8) bx = 8;
  k_pair_gather_cols<<<dim3(bx, ygrid(n)), 128, 0, st>>>(psi, n_isdf, b1, b2, n, out);
}

// ---------------------------------------------------------------------------
// y = sqrtR * x  (or a copy with TDA)   apply_matvec_lowcomsym.F90:112-128
__global__ void k_scale_rows(const double *__restrict__ s, const double *__restrict__ x, int ldx,
                             double *__restrict__ y, int ldy, int ncv, int nb, int tamm_d) {
  for (int j = blockIdx.y; j < nb; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncv; i += gridDim.x * blockDim.x) {
      double v = x[(size_t)j * ldx + i];
      y[(size_t)j * ldy + i] = tamm_d ? v : s[i] * v;
    }
}

void launch_scale_rows(const double *s, const double *x, int ldx, double *y, int ldy, int ncv,
                       int nb, int tamm_d, cudaStream_t st) {
  if (nb <= 0) return;
  int bx = cdiv(ncv, 256);
  if (bx > 16) bx = 16;
  k_scale_rows<<<dim3(bx, ygrid(nb)), 256, 0, st>>>(s, x, ldx, y, ldy, ncv, nb, tamm_d);
}

__global__ void k_copy_cols(const double *__restrict__ x, int ldx, double *__restrict__ y, int ldy,
                            int n, int nb) {
  for (int j = blockIdx.y; j < nb; j += gridDim.y)
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
      y[(size_t)j * ldy + i] = x[(size_t)j * ldx + i];
}

void launch_copy_cols(const double *x, int ldx, double *y, int ldy, int n, int nb,
                      cudaStream_t st) {
  if (nb <= 0) return;
  int bx = cdiv(n, 256);
  if (bx > 16) bx = 16;
  k_copy_cols<<<dim3(bx, ygrid(nb)), 256, 0, st>>>(x, ldx, y, ldy, n, nb);
}

// Diagonal combine of the ISDF matvec (apply_matvec_lowcomsym.F90:396-412)
//   non-TDA: y = sqrtR^3 * h + 4 sqrtR * z      (h = sqrtR * x)
//   TDA:     y = sqrtR^2 * h + 2 z              (h = x)
// followed by the Horner step (apply_matvec_lowcomsym.F90:504-511)
//   k == 1: y = p_k * y + p_{k+1} * vec ;  k > 1: y = y + p_{k+1} * vec
// and, for the next Horner matvec, hs = sqrtR * y (TDA: y).
__global__ void k_matvec_combine(const double *__restrict__ s, const double *__restrict__ h,
                                 const double *__restrict__ z, double *__restrict__ y,
                                 const double *__restrict__ vec, int ncv, int nb, int tamm_d,
                                 int horner_k, double pk, double pk1, double *__restrict__ hs) {
  for (int j = blockIdx.y; j < nb; j += gridDim.y) {
    const size_t base = (size_t)j * ncv;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncv; i += gridDim.x * blockDim.x) {
      const double si = s[i];
      double r;
      if (tamm_d) {
        r = (si * si) * h[base + i];
        r = r + 2.0 * z[base + i];
      } else {
        r = (si * si * si) * h[base + i];
        r = r + 4.0 * si * z[base + i];
      }
      if (horner_k == 1) {
        r = pk * r + pk1 * vec[base + i];
      } else if (horner_k > 1) {
        r = r + pk1 * vec[base + i];
      }
      y[base + i] = r;
      if (hs) hs[base + i] = tamm_d ? r : si * r;
    }
  }
}

void launch_matvec_combine(const double *s, const double *h, const double *z, double *y,
                           const double *vec, int ncv, int nb, int tamm_d, int horner_k,
                           double pk, double pk1, double *hs_next, cudaStream_t st) {
  if (nb <= 0) return;
  int bx = cdiv(ncv, 256);
  if (bx > 16) bx = 16;
  k_matvec_combine<<<dim3(bx, ygrid(nb)), 256, 0, st>>>(s, h, z, y, vec, ncv, nb, tamm_d, horner_k,
                                                 pk, pk1, hs_next);
}

// ---------------------------------------------------------------------------
// block reduction helper (sum of one double per thread; result to all threads)
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = (l < NT / 32) ? sh[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (l == 0) sh[32] = t;
  }
  __syncthreads();
  return sh[32];
}

constexpr int LNT = 256;

// vec = v0 / v0_norm ; b(1) = 1 ; hs = sqrtR * vec (TDA: vec)
// (lanczos_spectra_lowcomsym.F90:68-72).  clen (optional) receives each
// chain's length: len[j] (per-chain lengths) or niter, clamped to 1..niter.
// The step kernels leave a chain alone from step clen[j] on, and lower clen[j]
// when its recurrence breaks down (convergence mask, below).
__global__ void k_lanczos_init(const double *__restrict__ v0, int ld,
                               const double *__restrict__ v0_norm, double *__restrict__ vec,
                               double *__restrict__ hs, const double *__restrict__ s, int ncv,
                               int tamm_d, double *__restrict__ b_elmt, int niter,
                               const int *__restrict__ len, int *__restrict__ clen) {
  const int j = blockIdx.x;
  const double nrm = v0_norm[j];
  for (int i = threadIdx.x; i < ncv; i += blockDim.x) {
    double v = v0[(size_t)j * ld + i] / nrm;
    vec[(size_t)j * ncv + i] = v;
    hs[(size_t)j * ncv + i] = tamm_d ? v : s[i] * v;
  }
  if (threadIdx.x == 0) {
    b_elmt[(size_t)j * niter] = 1.0;
    if (clen) clen[j] = len ? min(max(len[j], 1), niter) : niter;
  }
}

void launch_lanczos_init(const double *v0, int ld, const double *v0_norm, double *vec, double *hs,
                         const double *s, int ncv, int nb, int tamm_d, double *b_elmt, int niter,
                         const int *len, int *clen, cudaStream_t st) {
  if (nb <= 0) return;
  k_lanczos_init<<<nb, LNT, 0, st>>>(v0, ld, v0_norm, vec, hs, s, ncv, tamm_d, b_elmt, niter, len,
                                     clen);
}

// Rescale for the next step and hand the next matvec its input:
//   w = w / b_k ; v = -v * b_k ; (swap: the caller exchanges the roles)
//   hs = sqrtR * w  (w is the next "vec")          lanczos_spectra_lowcomsym.F90:121-128
__device__ __forceinline__ void prescale_chain(double *w, double *v, int ncv, double bk,
                                               const double *s, double *hs, int tamm_d) {
  for (int i = threadIdx.x; i < ncv; i += blockDim.x) {
    double wi = w[i] / bk;
    w[i] = wi;
    v[i] = -v[i] * bk;
    if (hs) hs[i] = tamm_d ? wi : s[i] * wi;
  }
}

// a(1) = <w, v> ; w = w - a(1) v ; b(2) = ||w||   (lanczos_spectra_lowcomsym.F90:104-116)
// Convergence mask (eps > 0): the chain stops when |b(k)| < eps, as the
// single-vector reference does (shared/lanczos_spectra.f90:24,58: its later
// a/b stay unset; here they stay 0 and the continued fraction ends at clen).
__global__ void k_lanczos_first(double *__restrict__ w, const double *__restrict__ v, int ncv,
                                double *__restrict__ a, double *__restrict__ b, int niter,
                                int *__restrict__ clen, double eps) {
  __shared__ double sh[33];
  const int j = blockIdx.x;
  const int L = clen ? clen[j] : niter;
  double *wj = w + (size_t)j * ncv;
  const double *vj = v + (size_t)j * ncv;
  double acc = 0.0;
  for (int i = threadIdx.x; i < ncv; i += blockDim.x) acc += wj[i] * vj[i];
  const double a1 = block_sum<LNT>(acc, sh);
  acc = 0.0;
  for (int i = threadIdx.x; i < ncv; i += blockDim.x) {
    double wi = wj[i] - a1 * vj[i];
    wj[i] = wi;
    acc += wi * wi;
  }
  const double bb = block_sum<LNT>(acc, sh);
  if (threadIdx.x == 0) {
    a[(size_t)j * niter] = a1;
    if (L >= 2) {
      const double b2 = sqrt(bb);
      b[(size_t)j * niter + 1] = b2;
      if (clen && eps > 0.0 && b2 < eps) clen[j] = 1;
    }
  }
}

void launch_lanczos_first(double *w, const double *v, int ncv, int nb, double *a, double *b,
                          int niter, int *clen, double eps, cudaStream_t st) {
  if (nb <= 0) return;
  k_lanczos_first<<<nb, LNT, 0, st>>>(w, v, ncv, a, b, niter, clen, eps);
}

__global__ void k_lanczos_prescale(double *__restrict__ w, double *__restrict__ v, int ncv, int k,
                                   const double *__restrict__ b, int niter,
                                   const double *__restrict__ s, double *__restrict__ hs,
                                   int tamm_d, const int *__restrict__ clen) {
  const int j = blockIdx.x;
  if (clen && k >= clen[j]) return;     // finished or stopped chain
  const double bk = b[(size_t)j * niter + k];
  prescale_chain(w + (size_t)j * ncv, v + (size_t)j * ncv, ncv, bk, s,
                 hs ? hs + (size_t)j * ncv : nullptr, tamm_d);
}

void launch_lanczos_prescale(double *w, double *v, int ncv, int nb, int k, const double *b,
                             int niter, const double *s, double *hs, int tamm_d, const int *clen,
                             cudaStream_t st) {
  if (nb <= 0) return;
  k_lanczos_prescale<<<nb, LNT, 0, st>>>(w, v, ncv, k, b, niter, s, hs, tamm_d, clen);
}

// Step k (0-based, k >= 1):  w = w + t ; a(k) = <w, v> ;
//   if k+1 < niter: w = w - a(k) v ; b(k+1) = ||w||    (lanczos_spectra_lowcomsym.F90:153-164)
// and, when prescale_next, the next step's rescale (w /= b(k+1), v = -v b(k+1), hs).
// One CTA runs chain j.
__device__ __forceinline__ void lanczos_step_chain(double *__restrict__ w, double *__restrict__ v,
                                                   const double *__restrict__ t, int ncv, int k,
                                                   double *__restrict__ a, double *__restrict__ b, int niter,
                                                   const double *__restrict__ s, double *__restrict__ hs,
                                                   int tamm_d, int prescale_next, int *__restrict__ clen,
                                                   double eps, int j) {
  __shared__ double sh[33];
  const int L = clen ? clen[j] : niter;
  if (k >= L) return;                    // finished or stopped chain: vectors left as they are
  double *wj = w + (size_t)j * ncv;
  double *vj = v + (size_t)j * ncv;
  const double *tj = t + (size_t)j * ncv;
  double acc = 0.0;
  for (int i = threadIdx.x; i < ncv; i += blockDim.x) {
    double wi = wj[i] + tj[i];
    wj[i] = wi;
    acc += wi * vj[i];
  }
  const double ak = block_sum<LNT>(acc, sh);
  if (threadIdx.x == 0) a[(size_t)j * niter + k] = ak;
  if (k + 1 < L) {
    acc = 0.0;
    for (int i = threadIdx.x; i < ncv; i += blockDim.x) {
      double wi = wj[i] - ak * vj[i];
      wj[i] = wi;
      acc += wi * wi;
    }
    const double bk1 = sqrt(block_sum<LNT>(acc, sh));
    const bool stop = clen && eps > 0.0 && bk1 < eps;
    if (threadIdx.x == 0) {
      b[(size_t)j * niter + k + 1] = bk1;
      if (stop) clen[j] = k + 1;
    }
    if (prescale_next && !stop)
      prescale_chain(wj, vj, ncv, bk1, s, hs ? hs + (size_t)j * ncv : nullptr, tamm_d);
  }
}

__global__ void k_lanczos_step(double *__restrict__ w, double *__restrict__ v,
                               const double *__restrict__ t, int ncv, int k,
                               double *__restrict__ a, double *__restrict__ b, int niter,
                               const double *__restrict__ s, double *__restrict__ hs, int tamm_d,
                               int prescale_next, int *__restrict__ clen, double eps) {
  lanczos_step_chain(w, v, t, ncv, k, a, b, niter, s, hs, tamm_d, prescale_next, clen, eps, blockIdx.x);
}

// The step of several molecules' chains in one launch (mixed precision, no
// scaled copy): block b runs chain b - cb[g] of entry g, cb[g] <= b < cb[g+1].
__global__ void __launch_bounds__(LNT)
    k_lanczos_step_grouped(const LanczosGroupEntry *__restrict__ tab, const int *__restrict__ cb, int G, int k) {
  __shared__ int sg;
  if (threadIdx.x == 0) {
    int g = 0;
    while (g + 1 < G && (int)blockIdx.x >= cb[g + 1]) ++g;
    sg = g;
  }
  __syncthreads();
  const LanczosGroupEntry &e = tab[sg];
  lanczos_step_chain(e.w, e.v, e.t, e.ncv, k, e.a, e.b, e.niter, e.s, nullptr, 0, e.prescale_next, e.clen, e.eps,
                     (int)blockIdx.x - cb[sg]);
}

void launch_lanczos_step_grouped(const LanczosGroupEntry *tab, const int *cb, int G, int k, int total,
                                 cudaStream_t st) {
  if (total <= 0) return;
  k_lanczos_step_grouped<<<total, LNT, 0, st>>>(tab, cb, G, k);
}

// The same step with the chain's elements held in registers (EPT per thread,
// element i = threadIdx.x + e * LNT, the order of the three-pass form, so
// both block sums and every result are bit-identical to it): t, w, v are read
// once and w, v (and hs) written once, instead of three passes over the
// vectors.  For ncv <= EPT * LNT.
template <int EPT>
__global__ void __launch_bounds__(LNT)
    k_lanczos_step_reg(double *__restrict__ w, double *__restrict__ v, const double *__restrict__ t, int ncv,
                       int k, double *__restrict__ a, double *__restrict__ b, int niter,
                       const double *__restrict__ s, double *__restrict__ hs, int tamm_d, int prescale_next,
                       int *__restrict__ clen, double eps) {
  __shared__ double sh[33];
  const int j = blockIdx.x;
  const int L = clen ? clen[j] : niter;
  if (k >= L) return;
  double *wj = w + (size_t)j * ncv;
  double *vj = v + (size_t)j * ncv;
  const double *tj = t + (size_t)j * ncv;
  double wr[EPT], vr[EPT];
  double acc = 0.0;
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int i = threadIdx.x + e * LNT;
    wr[e] = 0.0;
    vr[e] = 0.0;
    if (i < ncv) {
      wr[e] = wj[i] + tj[i];
      vr[e] = vj[i];
      acc += wr[e] * vr[e];
    }
  }
  const double ak = block_sum<LNT>(acc, sh);
  if (threadIdx.x == 0) a[(size_t)j * niter + k] = ak;
  if (k + 1 >= L) {
#pragma unroll
    for (int e = 0; e < EPT; ++e) {
      const int i = threadIdx.x + e * LNT;
      if (i < ncv) wj[i] = wr[e];
    }
    return;
  }
  acc = 0.0;
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int i = threadIdx.x + e * LNT;
    if (i < ncv) {
      wr[e] = wr[e] - ak * vr[e];
      acc += wr[e] * wr[e];
    }
  }
  const double bk1 = sqrt(block_sum<LNT>(acc, sh));
  const bool stop = clen && eps > 0.0 && bk1 < eps;
  if (threadIdx.x == 0) {
    b[(size_t)j * niter + k + 1] = bk1;
    if (stop) clen[j] = k + 1;
  }
  const bool pre = prescale_next && !stop;
  double *hj = hs ? hs + (size_t)j * ncv : nullptr;
#pragma unroll
  for (int e = 0; e < EPT; ++e) {
    const int i = threadIdx.x + e * LNT;
    if (i >= ncv) continue;
    if (pre) {
      const double wi = wr[e] / bk1;
      wj[i] = wi;
      vj[i] = -vr[e] * bk1;
      if (hj) hj[i] = tamm_d ? wi : s[i] * wi;
    } else {
      wj[i] = wr[e];
    }
  }
}

void launch_lanczos_step(double *w, double *v, const double *t, int ncv, int nb, int k, double *a,
                         double *b, int niter, const double *s, double *hs, int tamm_d,
                         int prescale_next, int *clen, double eps, cudaStream_t st) {
  if (nb <= 0) return;
  // The register form reads t, w, v once and writes w, v once; measured
  // (warm launch list, 720 chains): 15.8 us against 21.9 us for the three
  // passes at ncv = 2700, 81 against 98 us at ncv = 5776.  Below ncv = 1024
  // the three-pass form.  NGW_LSTEP=3 keeps the three-pass form at every
  // size, NGW_LSTEP=r takes the register form at every size it covers
  // (comparison runs; both forms give identical results).
  static const int mode = [] {
    const char *e = getenv("NGW_LSTEP");
    return (e && e[0] == '3') ? 3 : ((e && e[0] == 'r') ? 1 : 0);
  }();
  const bool three_pass = mode == 3 || (mode == 0 && ncv <= 4 * LNT);
#define NGW_LSR(E)                                                                                       \
  k_lanczos_step_reg<E><<<nb, LNT, 0, st>>>(w, v, t, ncv, k, a, b, niter, s, hs, tamm_d, prescale_next, \
                                            clen, eps)
  if (three_pass) {
    k_lanczos_step<<<nb, LNT, 0, st>>>(w, v, t, ncv, k, a, b, niter, s, hs, tamm_d, prescale_next, clen,
                                       eps);
  } else if (ncv <= 8 * LNT) {
    NGW_LSR(8);
  } else if (ncv <= 16 * LNT) {
    NGW_LSR(16);
  } else if (ncv <= 24 * LNT) {
    NGW_LSR(24);
  } else if (ncv <= 32 * LNT) {
    NGW_LSR(32);
  } else {
    k_lanczos_step<<<nb, LNT, 0, st>>>(w, v, t, ncv, k, a, b, niter, s, hs, tamm_d, prescale_next, clen,
                                       eps);
  }
#undef NGW_LSR
}

// ---------------------------------------------------------------------------
// Lanczos step with full reorthogonalisation (optional form of the Sigma_c
// chains; the reference recurrence has none).  Chain j keeps its Lanczos
// vectors v_0 .. v_k in basis[j * ldb + q * ncv] (FP64).  Step k:
//   w = w + t (k >= 1; at k = 0 w already holds p(H) v_0) ; a(k) = <w, v_k> ;
//   if k + 1 < L:  w = w - a(k) v_k ; h = V^T w, w = w - V h (classical
//   Gram-Schmidt against v_0 .. v_k), repeated once when the pass shrank
//   ||w|| below 1/sqrt(2) of its value (the "twice is enough" criterion of
//   Daniel, Gragg, Kaufman and Stewart, Math. Comp. 30 (1976)) ; b(k+1) = ||w|| ;
//   when prescale_next: w = w / b(k+1) (= v_{k+1}, also stored in the basis),
//   v = -v b(k+1), hs = (R^1/2 or 1) w.
// One CTA per chain; the dot products are summed eight at a time (warp
// shuffles, then the eight warps' sums in a fixed order) and the update sums
// run over q in ascending order, so the result is deterministic.
constexpr int RG_Q = 8;

__global__ void __launch_bounds__(LNT)
    k_lanczos_reorth_step(double *__restrict__ w, double *__restrict__ v, const double *__restrict__ t,
                          int ncv, int k, double *__restrict__ a, double *__restrict__ b, int niter,
                          const double *__restrict__ s, double *__restrict__ hs, int tamm_d,
                          int prescale_next, int *__restrict__ clen, double eps, double *__restrict__ basis,
                          long long ldb) {
  extern __shared__ double hq[];           // k + 1 Gram-Schmidt coefficients
  __shared__ double sh[33];
  __shared__ double red[LNT / 32][RG_Q];
  const int j = blockIdx.x;
  const int L = clen ? clen[j] : niter;
  if (k >= L) return;
  double *wj = w + (size_t)j * ncv;
  double *vj = v + (size_t)j * ncv;
  const double *tj = t ? t + (size_t)j * ncv : nullptr;
  double *Vj = basis + (size_t)j * (size_t)ldb;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double acc = 0.0;
  for (int i = threadIdx.x; i < ncv; i += LNT) {
    double wi = wj[i];
    if (tj) {
      wi += tj[i];
      wj[i] = wi;
    }
    acc += wi * vj[i];
  }
  const double ak = block_sum<LNT>(acc, sh);
  if (threadIdx.x == 0) a[(size_t)j * niter + k] = ak;
  if (k + 1 >= L) return;
  acc = 0.0;
  for (int i = threadIdx.x; i < ncv; i += LNT) {
    const double wi = wj[i] - ak * vj[i];
    wj[i] = wi;
    acc += wi * wi;
  }
  double nrm2 = block_sum<LNT>(acc, sh);   // ||w||^2 before the pass
  double out2 = 0.0;                        // ||w||^2 after the last pass
  for (int pass = 0; pass < 2; ++pass) {
    // h_q = <v_q, w>, q = 0 .. k
    for (int q0 = 0; q0 <= k; q0 += RG_Q) {
      double d[RG_Q];
#pragma unroll
      for (int u = 0; u < RG_Q; ++u) d[u] = 0.0;
      for (int i = threadIdx.x; i < ncv; i += LNT) {
        const double wi = wj[i];
#pragma unroll
        for (int u = 0; u < RG_Q; ++u)
          if (q0 + u <= k) d[u] += Vj[(size_t)(q0 + u) * ncv + i] * wi;
      }
#pragma unroll
      for (int u = 0; u < RG_Q; ++u) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) d[u] += __shfl_xor_sync(0xffffffffu, d[u], o);
      }
      if (lane == 0) {
#pragma unroll
        for (int u = 0; u < RG_Q; ++u) red[warp][u] = d[u];
      }
      __syncthreads();
      if (threadIdx.x < RG_Q && q0 + (int)threadIdx.x <= k) {
        double h = 0.0;
#pragma unroll
        for (int g = 0; g < LNT / 32; ++g) h += red[g][threadIdx.x];
        hq[q0 + threadIdx.x] = h;
      }
      __syncthreads();
    }
    // w = w - V h, and the new ||w||^2; the basis values of eight vectors
    // are loaded before they are summed (in q order) so their loads overlap
    acc = 0.0;
    for (int i = threadIdx.x; i < ncv; i += LNT) {
      double u = 0.0;
      int q = 0;
      for (; q + RG_Q <= k + 1; q += RG_Q) {
        double x[RG_Q];
#pragma unroll
        for (int r = 0; r < RG_Q; ++r) x[r] = Vj[(size_t)(q + r) * ncv + i];
#pragma unroll
        for (int r = 0; r < RG_Q; ++r) u += hq[q + r] * x[r];
      }
      for (; q <= k; ++q) u += hq[q] * Vj[(size_t)q * ncv + i];
      const double wi = wj[i] - u;
      wj[i] = wi;
      acc += wi * wi;
    }
    out2 = block_sum<LNT>(acc, sh);
    if (out2 >= 0.5 * nrm2) break;   // the pass kept most of w: once is enough
    nrm2 = out2;
  }
  const double bk1 = sqrt(out2);
  const bool stop = clen && eps > 0.0 && bk1 < eps;
  if (threadIdx.x == 0) {
    b[(size_t)j * niter + k + 1] = bk1;
    if (stop) clen[j] = k + 1;
  }
  if (!prescale_next || stop) return;
  double *vn = Vj + (size_t)(k + 1) * ncv;
  double *hj = hs ? hs + (size_t)j * ncv : nullptr;
  for (int i = threadIdx.x; i < ncv; i += LNT) {
    const double wi = wj[i] / bk1;
    wj[i] = wi;
    vn[i] = wi;
    vj[i] = -vj[i] * bk1;
    if (hj) hj[i] = tamm_d ? wi : s[i] * wi;
  }
}

void launch_lanczos_reorth_step(double *w, double *v, const double *t, int ncv, int nb, int k, double *a,
                                double *b, int niter, const double *s, double *hs, int tamm_d,
                                int prescale_next, int *clen, double eps, double *basis, long long ldb,
                                cudaStream_t st) {
  if (nb <= 0) return;
  k_lanczos_reorth_step<<<nb, LNT, (size_t)(k + 1) * sizeof(double), st>>>(
      w, v, t, ncv, k, a, b, niter, s, hs, tamm_d, prescale_next, clen, eps, basis, ldb);
}

// basis slot 0 of every chain = its normalised start vector
__global__ void k_basis_init(const double *__restrict__ vec, int ncv, double *__restrict__ basis, long long ldb) {
  const int j = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncv; i += gridDim.x * blockDim.x)
    basis[(size_t)j * (size_t)ldb + i] = vec[(size_t)j * ncv + i];
}

void launch_basis_init(const double *vec, int ncv, int nb, double *basis, long long ldb, cudaStream_t st) {
  if (nb <= 0) return;
  for (int j0 = 0; j0 < nb; j0 += 65535) {
    const int n = std::min(65535, nb - j0);
    k_basis_init<<<dim3(std::min(cdiv(ncv, 256), 16), n), 256, 0, st>>>(vec + (size_t)j0 * ncv, ncv,
                                                                        basis + (size_t)j0 * (size_t)ldb, ldb);
  }
}

// ---------------------------------------------------------------------------
// complex helpers (Smith's division)
struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx cdivd(cplx a, cplx b) {
  cplx r;
  if (fabs(b.re) >= fabs(b.im)) {
    double q = b.im / b.re, d = b.re + b.im * q;
    r.re = (a.re + a.im * q) / d;
    r.im = (a.im - a.re * q) / d;
  } else {
    double q = b.re / b.im, d = b.im + b.re * q;
    r.re = (a.re * q + a.im) / d;
    r.im = (a.im * q - a.re) / d;
  }
  return r;
}

// S = 0; for j = niter..1: S = (j == 1 ? 1 : b_j^2) / (z - a_j - S)
// (lanczos_spectra_lowcomsym.F90:175-188)
__device__ __forceinline__ cplx contfrac_eval(const double *a, const double *b, int niter, cplx z) {
  cplx sacc = {0.0, 0.0};
  for (int jj = niter - 1; jj >= 0; --jj) {
    cplx num = {jj == 0 ? 1.0 : b[jj] * b[jj], 0.0};
    cplx den = {z.re - a[jj] - sacc.re, z.im - sacc.im};
    sacc = cdivd(num, den);
  }
  return sacc;
}

__global__ void k_contfrac(const double *__restrict__ a, const double *__restrict__ b, int niter,
                           int nb, const double *__restrict__ zz, int nz,
                           double *__restrict__ spectra, const int *__restrict__ clen) {
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  if (iz >= nz) return;
  for (int j = blockIdx.y; j < nb; j += gridDim.y) {
    const size_t o = (size_t)j * nz + iz;
    cplx z = {zz[2 * o], zz[2 * o + 1]};
    cplx r = contfrac_eval(a + (size_t)j * niter, b + (size_t)j * niter, clen ? clen[j] : niter, z);
    spectra[2 * o] = r.re;
    spectra[2 * o + 1] = r.im;
  }
}

void launch_contfrac(const double *a, const double *b, int niter, int nb, const double *zz, int nz,
                     double *spectra, const int *clen, cudaStream_t st) {
  if (nb <= 0 || nz <= 0) return;
  k_contfrac<<<dim3(cdiv(nz, 128), ygrid(nb)), 128, 0, st>>>(a, b, niter, nb, zz, nz, spectra, clen);
}

// Per-chain spectra on the Sigma energy grid:
//   zz_i = zz0 + de * i ; ezz_i = (E_n - zz_i) * eta_n + i*ecuts ; ezz_nen = 0
// (calculate_sigma_lanczos_lowcomsym.F90:527-530,713-720).  S: (nen+1, nchain).
__global__ void k_sigma_spectra(const double *__restrict__ a, const double *__restrict__ b,
                                int niter, int nchain, const double *__restrict__ e1,
                                const int *__restrict__ chain_band,
                                const int *__restrict__ chain_qp, const double *__restrict__ zz0,
                                double de, int nen, double ecuts, int nval,
                                double *__restrict__ S, const int *__restrict__ clen) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > nen) return;
  for (int j = blockIdx.y; j < nchain; j += gridDim.y) {
    const int n = chain_band[j];
    const double eta = (n <= nval) ? 1.0 : -1.0;
    cplx z;
    if (i == nen) {
      z.re = 0.0;
      z.im = 0.0;
    } else {
      const double zz = de * (double)i + zz0[chain_qp[j]];
      z.re = (-zz + e1[n - 1]) * eta;
      z.im = ecuts;
    }
    cplx r = contfrac_eval(a + (size_t)j * niter, b + (size_t)j * niter, clen ? clen[j] : niter, z);
    const size_t o = (size_t)j * (nen + 1) + i;
    S[2 * o] = r.re;
    S[2 * o + 1] = r.im;
  }
}

void launch_sigma_spectra(const double *a, const double *b, int niter, int nchain,
                          const double *e1, const int *chain_band, const int *chain_qp,
                          const double *zz0, double de, int nen, double ecuts, int nval,
                          double *S, const int *clen, cudaStream_t st) {
  if (nchain <= 0) return;
  k_sigma_spectra<<<dim3(cdiv(nen + 1, 128), ygrid(nchain)), 128, 0, st>>>(
      a, b, niter, nchain, e1, chain_band, chain_qp, zz0, de, nen, ecuts, nval, S, clen);
}

// Sigma_c(i, iq) (+)= sum over the bands n of
//   non-TDA: (S_n(0) - S_n(ezz)) * eta_n * 2 * pnorm2_n / ezz
//   TDA:     -S_n(ezz) * eta_n * sqrt(2) * pnorm2_n   (sqrt(2) in single precision, as 2.0**0.5)
// (calculate_sigma_lanczos_lowcomsym.F90:736-745).  The chain of (QP iq,
// band nn) is slot[iq*nbsum + nn] of this block (iq*nbsum + nn without slot).
// Block (32 energies) x (8 band groups): lane x of warp y sums bands
// y, y + 8, ... for energy x (consecutive lanes read consecutive energies of
// a chain's spectrum); the 8 partial sums are added in a fixed order.
constexpr int SR_E = 32, SR_G = 8;
__global__ void __launch_bounds__(SR_E *SR_G)
    k_sigma_reduce(const double *__restrict__ S, const double *__restrict__ pnorm2,
                   const double *__restrict__ e1, const int *__restrict__ chain_band,
                   const double *__restrict__ zz0, double de, int nen, double ecuts, int nval, int nbsum,
                   int nqp, int tamm_d, double *__restrict__ sigma, int accumulate,
                   const int *__restrict__ slot) {
  __shared__ double part[SR_G][SR_E][2];
  const int iq = blockIdx.y;
  const int i = blockIdx.x * SR_E + threadIdx.x;
  const bool on = iq < nqp && i < nen;
  cplx acc = {0.0, 0.0};
  if (on) {
    const double zz = de * (double)i + zz0[iq];
    const double sqrt2f = (double)sqrtf(2.0f);
    for (int nn = threadIdx.y; nn < nbsum; nn += SR_G) {
      const int j = slot ? slot[iq * nbsum + nn] : iq * nbsum + nn;
      const int n = chain_band[j];
      const double eta = (n <= nval) ? 1.0 : -1.0;
      const size_t o = (size_t)j * (nen + 1);
      cplx s = {S[2 * (o + i)], S[2 * (o + i) + 1]};
      cplx t;
      if (tamm_d) {
        t.re = -s.re * eta * sqrt2f * pnorm2[j];
        t.im = -s.im * eta * sqrt2f * pnorm2[j];
      } else {
        cplx s0 = {S[2 * (o + nen)], S[2 * (o + nen) + 1]};
        cplx d = {(s0.re - s.re) * eta * 2.0 * pnorm2[j], (s0.im - s.im) * eta * 2.0 * pnorm2[j]};
        cplx ez = {(-zz + e1[n - 1]) * eta, ecuts};
        t = cdivd(d, ez);
      }
      acc.re += t.re;
      acc.im += t.im;
    }
  }
  part[threadIdx.y][threadIdx.x][0] = acc.re;
  part[threadIdx.y][threadIdx.x][1] = acc.im;
  __syncthreads();
  if (threadIdx.y == 0 && on) {
    cplx tot = {0.0, 0.0};
    if (accumulate) {
      tot.re = sigma[2 * ((size_t)iq * nen + i)];
      tot.im = sigma[2 * ((size_t)iq * nen + i) + 1];
    }
    for (int g = 0; g < SR_G; ++g) {
      tot.re += part[g][threadIdx.x][0];
      tot.im += part[g][threadIdx.x][1];
    }
    sigma[2 * ((size_t)iq * nen + i)] = tot.re;
    sigma[2 * ((size_t)iq * nen + i) + 1] = tot.im;
  }
}

void launch_sigma_reduce(const double *S, const double *pnorm2, const double *e1,
                         const int *chain_band, const double *zz0, double de, int nen,
                         double ecuts, int nval, int nbsum, int nqp, int tamm_d, double *sigma,
                         int accumulate, const int *slot, cudaStream_t st) {
  if (nqp <= 0) return;
  k_sigma_reduce<<<dim3(cdiv(nen, SR_E), nqp), dim3(SR_E, SR_G), 0, st>>>(
      S, pnorm2, e1, chain_band, zz0, de, nen, ecuts, nval, nbsum, nqp, tamm_d, sigma, accumulate, slot);
}

// P = P * sqrtR (non-TDA) ; pnorm2 = <P, P>   (calculate_sigma_lanczos_lowcomsym.F90:696-705)
__global__ void k_norms(const double *__restrict__ P, int ncv, const double *__restrict__ s,
                        int tamm_d, double *__restrict__ Pout, double *__restrict__ pnorm2) {
  __shared__ double sh[33];
  const int j = blockIdx.x;
  double acc = 0.0;
  for (int i = threadIdx.x; i < ncv; i += blockDim.x) {
    double p = P[(size_t)j * ncv + i];
    if (!tamm_d) p = p * s[i];
    Pout[(size_t)j * ncv + i] = p;
    acc += p * p;
  }
  double t = block_sum<LNT>(acc, sh);
  if (threadIdx.x == 0) pnorm2[j] = t;
}

void launch_norms(const double *P, int ncv, int nb, const double *s, int tamm_d, double *P_out,
                  double *pnorm2, cudaStream_t st) {
  if (nb <= 0) return;
  k_norms<<<nb, LNT, 0, st>>>(P, ncv, s, tamm_d, P_out, pnorm2);
}

// ---------------------------------------------------------------------------
// QP Newton solve: one thread per state.  spline / splint / spline_evaluate /
// newtonr restate SIGMA/spline.f90, splint.f90, spline_evaluate.f90:37-48,
// newtonr.f90:43-55; printsigma.F90:100-125 builds the table.
// Workspace per state: 4 * nen doubles.
__device__ void d_spline(const double *xx, const double *yy, int nn, double yp1, double ypn,
                         double *y2, double *uu) {
  const double HUGEV = 1.0e10;
  if (fabs(yp1) > HUGEV) {
    y2[0] = 0.0;
    uu[0] = 0.0;
  } else {
    y2[0] = -0.5;
    uu[0] = (3.0 / (xx[1] - xx[0])) * ((yy[1] - yy[0]) / (xx[1] - xx[0]) - yp1);
  }
  for (int i = 1; i < nn - 1; ++i) {
    double sig = (xx[i] - xx[i - 1]) / (xx[i + 1] - xx[i - 1]);
    double p = sig * y2[i - 1] + 2.0;
    y2[i] = (sig - 1.0) / p;
    uu[i] = (6.0 * ((yy[i + 1] - yy[i]) / (xx[i + 1] - xx[i]) - (yy[i] - yy[i - 1]) / (xx[i] - xx[i - 1])) /
                 (xx[i + 1] - xx[i - 1]) -
             sig * uu[i - 1]) /
            p;
  }
  double qn, un;
  if (ypn > HUGEV) {
    qn = 0.0;
    un = 0.0;
  } else {
    qn = 0.5;
    un = (3.0 / (xx[nn - 1] - xx[nn - 2])) * (ypn - (yy[nn - 1] - yy[nn - 2]) / (xx[nn - 1] - xx[nn - 2]));
  }
  y2[nn - 1] = (un - qn * uu[nn - 2]) / (qn * y2[nn - 2] + 1.0);
  for (int k = nn - 2; k >= 0; --k) y2[k] = y2[k] * y2[k + 1] + uu[k];
}

__device__ double d_splint(const double *xx, const double *yy, const double *y2a, int nn, double x0) {
  int klo = 0, khi = nn - 1;
  while (khi - klo > 1) {
    int k = (khi + klo + 2) / 2 - 1;
    if (xx[k] > x0) khi = k;
    else klo = k;
  }
  double hh = xx[khi] - xx[klo];
  double aa = (xx[khi] - x0) / hh, bb = (x0 - xx[klo]) / hh;
  return aa * yy[klo] + bb * yy[khi] + ((aa * aa * aa - aa) * y2a[klo] + (bb * bb * bb - bb) * y2a[khi]) * (hh * hh) / 6.0;
}

// real part only is needed for the root and the derivative
__device__ void d_spline_eval_re(const double *xt, const double *ft, int nt, double *y2, double *uu,
                                 double x, double *fx, double *df) {
  // spline through interior points 2..nt-1 with end slopes from the outer points
  const double yp1 = (ft[1] - ft[0]) / (xt[1] - xt[0]);
  const double ypn = (ft[nt - 1] - ft[nt - 2]) / (xt[nt - 1] - xt[nt - 2]);
  d_spline(xt + 1, ft + 1, nt - 2, yp1, ypn, y2, uu);
  *fx = d_splint(xt + 1, ft + 1, y2, nt - 2, x);
  const double ym = d_splint(xt + 1, ft + 1, y2, nt - 2, x - 1.0e-2);
  const double yp = d_splint(xt + 1, ft + 1, y2, nt - 2, x + 1.0e-2);
  *df = (yp - ym) / 1.0e-2 * 0.5;
}

__global__ void k_qp_newton(int nqp, int nen, const double *__restrict__ sig,
                            const double *__restrict__ e1, const double *__restrict__ e0,
                            double deltae, const double *__restrict__ sigx,
                            const double *__restrict__ vxc, double xacc, double *__restrict__ eqp,
                            double *__restrict__ zfac, int *__restrict__ ierr,
                            double *__restrict__ work) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nqp) return;
  double *xt = work + (size_t)q * 4 * nen;
  double *ft = xt + nen;
  double *y2 = ft + nen;
  double *uu = y2 + nen;
  for (int i = 0; i < nen; ++i) {
    xt[i] = e1[q] - deltae * 0.5 + deltae / (double)(nen - 1) * (double)i;
    ft[i] = sigx[q] + sig[2 * ((size_t)q * nen + i)] - vxc[q] + e0[q] - xt[i];
  }
  double x = e1[q], fx = 0.0, df = 1.0;
  int err = 21;   // Fortran loop counter after MAX_IT = 20 iterations
  for (int it = 1; it <= 20; ++it) {
    d_spline_eval_re(xt, ft, nen, y2, uu, x, &fx, &df);
    const double dx = fx / df;
    x = x - dx;
    if (fabs(dx) < xacc) {
      err = 0;
      break;
    }
  }
  d_spline_eval_re(xt, ft, nen, y2, uu, x, &fx, &df);
  eqp[q] = x;
  zfac[q] = -1.0 / df;
  ierr[q] = err;
}

void launch_qp_newton_ws(int nqp, int nen, const double *sig, const double *e1, const double *e0,
                         double deltae, const double *sigx, const double *vxc, double xacc,
                         double *eqp, double *zfac, int *ierr, double *work, cudaStream_t st) {
  if (nqp <= 0) return;
  k_qp_newton<<<cdiv(nqp, 32), 32, 0, st>>>(nqp, nen, sig, e1, e0, deltae, sigx, vxc, xacc, eqp,
                                            zfac, ierr, work);
}

__global__ void k_sqrt_vec(const double *__restrict__ x, double *__restrict__ y, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = sqrt(x[i]);
}

void launch_sqrt_vec(const double *x, double *y, int n, cudaStream_t st) {
  if (n <= 0) return;
  k_sqrt_vec<<<cdiv(n, 256), 256, 0, st>>>(x, y, n);
}

__global__ void k_k_combine(const double *__restrict__ M, const double *__restrict__ Mxc, size_t n,
                            int kflag, double *__restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    if (kflag < 2) v = M[i];
    if (kflag > 0) v = v + Mxc[i];
    out[i] = v;
  }
}

void launch_k_combine(const double *M, const double *Mxc, int n, int kflag, double *out,
                      cudaStream_t st) {
  size_t nn = (size_t)n * n;
  int blocks = cdiv((long long)nn, 256);
  if (blocks > 4096) blocks = 4096;
  k_k_combine<<<blocks, 256, 0, st>>>(M, Mxc, nn, kflag, out);
}

}  // namespace ngw

// Batched 3-D FFT convolution with the truncated Coulomb kernel, hand-written
// for the Poisson solves (shared/fft_module.F90z:122-177; FFTW there).
//
// Box edge n is any even number (the reference's box n = even(nint(4 rmax/h))
// is not restricted to FFT-friendly sizes), so the 1-D transforms use the
// mixed-radix Stockham formulation with a direct DFT of each radix: stage s
// with radix R and Ns = product of the earlier radices maps
//   y[(j/Ns) Ns R + j%Ns + q Ns] = sum_r x[j + r n/R] w_n^(r k n/(Ns R)),
//   k = j%Ns + q Ns,  j < n/R,  q < R,   w_n = exp(-2 pi i / n)
// (one thread per output, one table of n-th roots; radices 4, 2, 3, 5, 7, 11,
// 13 first, any remaining prime factor as one direct stage).  A transform of
// a batch of lines runs in shared memory, ping-ponging between two buffers.
//
// Data flow per batch of columns (layout of the cuFFT path it replaces):
//   box   [col][a][b][c] real, c fastest
//   spec  [col][a][b][k] complex, k = 0..n/2 (half spectrum along c)
//   1. rows along c: real -> complex FFT, keep k <= n/2
//   2. lines along b (stride n/2+1): forward
//   3. lines along a (stride n (n/2+1)): forward, times v(G), inverse (fused)
//   4. lines along b: inverse
//   5. rows along c: Hermitian half spectrum -> full line, inverse, real part
// The 1/n^3 scale is applied by the unpack kernel, as on the cuFFT path.
#include <cmath>
#include <vector>

#include "ngw_internal.h"

namespace ngw {

constexpr int FFT_MAX_STAGES = 24;

struct FftDesc {
  int n, nst;
  int R[FFT_MAX_STAGES];
};

// Radices of n: 4, 2, 3, 5, 7, 11, 13 while they divide, then the remaining
// prime factors in increasing order.
static int fft_factor(int n, FftDesc &D) {
  D.n = n;
  D.nst = 0;
  int m = n;
  for (int p : {4, 2, 3, 5, 7, 11, 13})
    while (m % p == 0 && D.nst < FFT_MAX_STAGES) {
      D.R[D.nst++] = p;
      m /= p;
    }
  for (int p = 17; m > 1 && D.nst < FFT_MAX_STAGES; p += 2)
    while (m % p == 0 && D.nst < FFT_MAX_STAGES) {
      D.R[D.nst++] = p;
      m /= p;
    }
  return m == 1 ? NGW_OK : NGW_ERR_ARG;
}

// All stages of the transform of nl lines of length n held in smem buffer a
// (line stride n); b is scratch of the same size.  Returns the buffer that
// holds the result.  INV: inverse transform (conjugate roots, unscaled).
template <bool INV>
__device__ double2 *fft_lines(double2 *a, double2 *b, int nl, const FftDesc &D, const double2 *__restrict__ root) {
  const int n = D.n;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthr = blockDim.x * blockDim.y;
  int Ns = 1;
  for (int s = 0; s < D.nst; ++s) {
    const int R = D.R[s], m = n / R, L = Ns * R, step = n / L;
    for (int idx = tid; idx < nl * n; idx += nthr) {
      const int line = idx / n, t = idx - line * n;
      const int j = t % m, q = t / m, jm = j % Ns, k = jm + q * Ns;
      const double2 *x = a + (size_t)line * n;
      const int de = (int)(((long long)k * step) % n);
      int e = 0;
      double re = 0.0, im = 0.0;
      for (int r = 0; r < R; ++r) {
        const double2 v = x[j + r * m];
        double2 w = __ldg(root + e);
        if (INV) w.y = -w.y;
        re = fma(v.x, w.x, fma(-v.y, w.y, re));
        im = fma(v.x, w.y, fma(v.y, w.x, im));
        e += de;
        if (e >= n) e -= n;
      }
      b[(size_t)line * n + (j / Ns) * L + jm + q * Ns] = make_double2(re, im);
    }
    __syncthreads();
    double2 *tmp = a;
    a = b;
    b = tmp;
    Ns = L;
  }
  return a;
}

// 1. rows along c, real -> half spectrum
__global__ void k_fft_rows_r2c(const double *__restrict__ box, size_t nrows, FftDesc D,
                               const double2 *__restrict__ root, double2 *__restrict__ spec) {
  extern __shared__ double2 sm[];
  const int n = D.n, h = n / 2 + 1;
  const int tl = blockDim.y;   // rows per block
  double2 *a = sm, *b = sm + (size_t)tl * n;
  for (size_t r0 = (size_t)blockIdx.x * tl; r0 < nrows; r0 += (size_t)gridDim.x * tl) {
    const int nl = (int)min((size_t)tl, nrows - r0);
    for (int i = threadIdx.y * blockDim.x + threadIdx.x; i < nl * n; i += blockDim.x * blockDim.y)
      a[i] = make_double2(box[r0 * n + i], 0.0);
    __syncthreads();
    double2 *res = fft_lines<false>(a, b, nl, D, root);
    for (int i = threadIdx.y * blockDim.x + threadIdx.x; i < nl * h; i += blockDim.x * blockDim.y) {
      const int line = i / h, k = i - line * h;
      spec[(r0 + line) * h + k] = res[(size_t)line * n + k];
    }
    __syncthreads();
  }
}

// 5. rows along c: half spectrum -> real (unscaled)
__global__ void k_fft_rows_c2r(const double2 *__restrict__ spec, size_t nrows, FftDesc D,
                               const double2 *__restrict__ root, double *__restrict__ box) {
  extern __shared__ double2 sm[];
  const int n = D.n, h = n / 2 + 1;
  const int tl = blockDim.y;
  double2 *a = sm, *b = sm + (size_t)tl * n;
  for (size_t r0 = (size_t)blockIdx.x * tl; r0 < nrows; r0 += (size_t)gridDim.x * tl) {
    const int nl = (int)min((size_t)tl, nrows - r0);
    for (int i = threadIdx.y * blockDim.x + threadIdx.x; i < nl * n; i += blockDim.x * blockDim.y) {
      const int line = i / n, k = i - line * n;
      double2 v;
      if (k < h) {
        v = spec[(r0 + line) * h + k];
      } else {
        v = spec[(r0 + line) * h + (n - k)];
        v.y = -v.y;
      }
      a[i] = v;
    }
    __syncthreads();
    double2 *res = fft_lines<true>(a, b, nl, D, root);
    for (int i = threadIdx.y * blockDim.x + threadIdx.x; i < nl * n; i += blockDim.x * blockDim.y)
      box[r0 * n + i] = res[i].x;
    __syncthreads();
  }
}

// 2-4. lines along a strided axis of spec.  Line (o, k): elements
// spec[o_base(o) + i*stride + k], i = 0..n-1, where o_base(o) = (o / inner) *
// outer_step + (o % inner) * inner_step.  A block takes TK consecutive k of
// one o (loads coalesced along k).  MODE 0: forward, 1: inverse, 2: forward,
// multiply by vtab, inverse (vtab indexed like spec of one column:
// ((a*n + b)*h + k) with a the line index i and b = o % n).
template <int MODE>
__global__ void k_fft_strided(double2 *__restrict__ spec, int nouter, int inner, size_t outer_step,
                              size_t inner_step, size_t stride, FftDesc D, const double2 *__restrict__ root,
                              const double *__restrict__ vtab) {
  extern __shared__ double2 sm[];
  const int n = D.n, h = n / 2 + 1;
  const int tk = blockDim.y;
  double2 *a = sm, *b = sm + (size_t)tk * n;
  const int k0 = blockIdx.x * tk;
  const int nk = min(tk, h - k0);
  for (int o = blockIdx.y; o < nouter; o += gridDim.y) {
    const size_t base = (size_t)(o / inner) * outer_step + (size_t)(o % inner) * inner_step + k0;
    // smem line kk holds elements i = 0..n-1 of line k0 + kk
    for (int i = threadIdx.y; i < n; i += blockDim.y)
      for (int kk = threadIdx.x; kk < nk; kk += blockDim.x) a[(size_t)kk * n + i] = spec[base + i * stride + kk];
    __syncthreads();
    double2 *res;
    if (MODE == 1) {
      res = fft_lines<true>(a, b, nk, D, root);
    } else {
      res = fft_lines<false>(a, b, nk, D, root);
      if (MODE == 2) {
        const int bidx = o % inner;
        double2 *oth = (res == a) ? b : a;
        for (int idx = threadIdx.y * blockDim.x + threadIdx.x; idx < nk * n; idx += blockDim.x * blockDim.y) {
          const int kk = idx / n, i = idx - kk * n;
          const double v = vtab[((size_t)i * n + bidx) * h + k0 + kk];
          res[idx].x *= v;
          res[idx].y *= v;
        }
        __syncthreads();
        res = fft_lines<true>(res, oth, nk, D, root);
      }
    }
    for (int i = threadIdx.y; i < n; i += blockDim.y)
      for (int kk = threadIdx.x; kk < nk; kk += blockDim.x) spec[base + i * stride + kk] = res[(size_t)kk * n + i];
    __syncthreads();
  }
}

// Forward FFT, multiply by the Coulomb table, inverse FFT of ncol boxes
// (box -> box, unscaled).  spec: ncol * n * n * (n/2+1) complex scratch.
int fft_coulomb_boxes(ngw_session *s, int n, int ncol, double *box, double2 *spec, const double *vtab) {
  FftDesc D;
  if (fft_factor(n, D) != NGW_OK) {
    set_error("FFT box edge %d has more than %d prime factors", n, FFT_MAX_STAGES);
    return NGW_ERR_ARG;
  }
  // n-th roots of unity, computed in long double
  std::vector<double2> hroot(n);
  for (int e = 0; e < n; ++e) {
    const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)e / (long double)n;
    hroot[e] = make_double2((double)cosl(ang), (double)sinl(ang));
  }
  static std::atomic<unsigned long long> attr[5] = {};
  const int mx = 200 * 1024;
  NGW_CUDA(smem_limit_once(k_fft_rows_r2c, mx, attr[0]));
  NGW_CUDA(smem_limit_once(k_fft_rows_c2r, mx, attr[1]));
  NGW_CUDA(smem_limit_once(k_fft_strided<0>, mx, attr[2]));
  NGW_CUDA(smem_limit_once(k_fft_strided<1>, mx, attr[3]));
  NGW_CUDA(smem_limit_once(k_fft_strided<2>, mx, attr[4]));
  double2 *root = nullptr;
  NGW_TRY(dalloc(s, (void **)&root, (size_t)n * sizeof(double2)));
  int rc = NGW_OK;
  do {
    if (cudaMemcpyAsync(root, hroot.data(), (size_t)n * sizeof(double2), cudaMemcpyHostToDevice, s->stream)) {
      set_error("copy of the FFT roots failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    const int h = n / 2 + 1;
    const size_t nrows = (size_t)ncol * n * n;
    const int tl = n > 128 ? 2 : 4;
    const size_t smem_rows = (size_t)2 * tl * n * sizeof(double2);
    const int row_blocks = (int)std::min<size_t>((nrows + tl - 1) / tl, 148 * 16);
    const int tk = 8;
    const size_t smem_str = (size_t)2 * tk * n * sizeof(double2);
    const dim3 rblk(64, tl), sblk(8, tk);
    const dim3 sgrid((h + tk - 1) / tk, ygrid((long long)ncol * n));
    const size_t colsz = (size_t)n * n * h;
    k_fft_rows_r2c<<<row_blocks, rblk, smem_rows, s->stream>>>(box, nrows, D, root, spec);
    // along b: lines (col, a), base = col*colsz + a*n*h, stride h
    k_fft_strided<0><<<sgrid, sblk, smem_str, s->stream>>>(spec, ncol * n, n, colsz, (size_t)n * h, h, D, root,
                                                          nullptr);
    // along a, with the Coulomb multiply: lines (col, b), base = col*colsz + b*h, stride n*h
    k_fft_strided<2><<<sgrid, sblk, smem_str, s->stream>>>(spec, ncol * n, n, colsz, (size_t)h, (size_t)n * h, D,
                                                          root, vtab);
    k_fft_strided<1><<<sgrid, sblk, smem_str, s->stream>>>(spec, ncol * n, n, colsz, (size_t)n * h, h, D, root,
                                                          nullptr);
    k_fft_rows_c2r<<<row_blocks, rblk, smem_rows, s->stream>>>(spec, nrows, D, root, box);
    if (cudaGetLastError() != cudaSuccess) {
      set_error("FFT kernels failed to launch");
      rc = NGW_ERR_CUDA;
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, root, (size_t)n * sizeof(double2));
  return rc;
}

}  // namespace ngw

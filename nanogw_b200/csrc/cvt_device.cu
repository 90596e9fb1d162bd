// CVT interpolation-point selection on the device, bit-identical to the host
// restatement (ngw_cvt, shared/cvt.F90:105-187).
//
// Per iteration the device does the O(N_grid x N_mu) work:
//   * nearest centre of every grid point (first minimum, cvt.F90:108-121),
//   * rho-weighted centroid sums, one thread per centre adding its points in
//     grid order (cvt.F90:126-142, the host's summation order),
//   * the new centre (IEEE division) or the previous one when the weight is
//     below 1e-10 (a single-precision literal in the reference),
//   * for every centre the nearest grid point over the whole grid (first
//     minimum of sqrt(distance^2), cvt.F90:143-174).
// The host then walks the centres in order: a centre keeps its nearest point
// unless an earlier centre of this sweep took it, in which case the host
// searches the untaken points itself (same arithmetic); it sums the moves
// and tests convergence.  Squared distances are formed as
// ((dx*dx) + dy*dy) + dz*dz with separately rounded products and sums
// (no fused multiply-add), as the host code compiled with -ffp-contract=off.
#include <cmath>
#include <cstring>
#include <vector>

#include "ngw_internal.h"

namespace ngw {

__device__ __forceinline__ double sqdist_rn(double ax, double ay, double az, double bx, double by, double bz) {
  const double dx = __dsub_rn(ax, bx), dy = __dsub_rn(ay, by), dz = __dsub_rn(az, bz);
  double r = __dmul_rn(dx, dx);
  r = __dadd_rn(r, __dmul_rn(dy, dy));
  r = __dadd_rn(r, __dmul_rn(dz, dz));
  return r;
}

constexpr int CVT_TILE = 1024;

// owner[g] = first p minimising |pts_p - grid_g|^2 below `far` (-1 if none)
__global__ void k_cvt_assign(const double *__restrict__ grid, int ngrid, const double *__restrict__ pts, int np,
                             double far, int *__restrict__ owner) {
  __shared__ double sp[3 * CVT_TILE];
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  double gx = 0, gy = 0, gz = 0;
  if (g < ngrid) {
    gx = grid[3 * (size_t)g];
    gy = grid[3 * (size_t)g + 1];
    gz = grid[3 * (size_t)g + 2];
  }
  double best = far;
  int who = -1;
  for (int p0 = 0; p0 < np; p0 += CVT_TILE) {
    const int nt = min(CVT_TILE, np - p0);
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * nt; i += blockDim.x) sp[i] = pts[3 * (size_t)p0 + i];
    __syncthreads();
    if (g < ngrid)
      for (int q = 0; q < nt; ++q) {
        const double d = sqdist_rn(sp[3 * q], sp[3 * q + 1], sp[3 * q + 2], gx, gy, gz);
        if (d < best) {
          best = d;
          who = p0 + q;
        }
      }
  }
  if (g < ngrid) owner[g] = who;
}

// acc[4p..4p+3] = sum over g with owner[g] == p, in grid order, of (x rho, y rho, z rho, rho)
__global__ void k_cvt_accumulate(const double *__restrict__ grid, const double *__restrict__ rho,
                                 const int *__restrict__ owner, int ngrid, int np, double *__restrict__ acc) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  for (int g = 0; g < ngrid; ++g) {
    if (owner[g] != p) continue;
    const double r = rho[g];
    a0 = __dadd_rn(a0, __dmul_rn(grid[3 * (size_t)g], r));
    a1 = __dadd_rn(a1, __dmul_rn(grid[3 * (size_t)g + 1], r));
    a2 = __dadd_rn(a2, __dmul_rn(grid[3 * (size_t)g + 2], r));
    a3 = __dadd_rn(a3, r);
  }
  acc[4 * (size_t)p] = a0;
  acc[4 * (size_t)p + 1] = a1;
  acc[4 * (size_t)p + 2] = a2;
  acc[4 * (size_t)p + 3] = a3;
}

// new centre: weighted centroid, or the previous centre when the weight is tiny
__global__ void k_cvt_newpos(const double *__restrict__ acc, const double *__restrict__ prev, int np,
                             double wtiny, double *__restrict__ pts) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const double *a = acc + 4 * (size_t)p;
  for (int d = 0; d < 3; ++d)
    pts[3 * (size_t)p + d] = (a[3] < wtiny) ? prev[3 * (size_t)p + d] : __ddiv_rn(a[d], a[3]);
}

// gsel[p] = first grid point minimising sqrt(|pts_p - grid_g|^2) below dmin0
__global__ void k_cvt_nearest_point(const double *__restrict__ grid, int ngrid, const double *__restrict__ pts,
                                    double dmin0, int *__restrict__ gsel) {
  __shared__ double sd[256];
  __shared__ int si[256];
  const int p = blockIdx.x;
  const double px = pts[3 * (size_t)p], py = pts[3 * (size_t)p + 1], pz = pts[3 * (size_t)p + 2];
  double best = dmin0;
  int who = -1;
  for (int g = threadIdx.x; g < ngrid; g += blockDim.x) {
    const double d = __dsqrt_rn(sqdist_rn(px, py, pz, grid[3 * (size_t)g], grid[3 * (size_t)g + 1],
                                          grid[3 * (size_t)g + 2]));
    if (d < best) {
      best = d;
      who = g;
    }
  }
  sd[threadIdx.x] = best;
  si[threadIdx.x] = who;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      const double d2 = sd[threadIdx.x + o];
      const int i2 = si[threadIdx.x + o];
      // lexicographic (distance, index) minimum = the first minimum in grid order
      if (i2 >= 0 && (d2 < sd[threadIdx.x] || (d2 == sd[threadIdx.x] && (si[threadIdx.x] < 0 || i2 < si[threadIdx.x])))) {
        sd[threadIdx.x] = d2;
        si[threadIdx.x] = i2;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) gsel[p] = si[0];
}

static inline double sqdist_host(const double *a, const double *b) {
  volatile double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  volatile double r = dx * dx;
  volatile double t = dy * dy;
  r = r + t;
  t = dz * dz;
  r = r + t;
  return r;
}

}  // namespace ngw

using namespace ngw;

extern "C" int ngw_cvt_device(ngw_session *s, int ngrid, const double *grid, const double *rho, int n_intp,
                              double *pts, int max_iter, int *intp, int *iters) {
  if (!s || ngrid <= 0 || n_intp <= 0 || n_intp > ngrid || !grid || !rho || !pts || !intp || max_iter <= 0) {
    set_error("ngw_cvt_device: bad arguments");
    return NGW_ERR_ARG;
  }
  NGW_CUDA(cudaSetDevice(s->device));
  const double tol_conv = (double)1e-3f;
  const double wtiny = (double)1.0e-10f;
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) lo[d] = hi[d] = grid[d];
  for (int g = 1; g < ngrid; ++g)
    for (int d = 0; d < 3; ++d) {
      const double v = grid[3 * g + d];
      lo[d] = v < lo[d] ? v : lo[d];
      hi[d] = v > hi[d] ? v : hi[d];
    }
  double bmax = hi[0], bmin = lo[0];
  for (int d = 1; d < 3; ++d) {
    bmax = hi[d] > bmax ? hi[d] : bmax;
    bmin = lo[d] < bmin ? lo[d] : bmin;
  }
  const double span = bmax - bmin;
  const double far = (double)100.0f * (span * span);
  const double dmin0 = (double)1.e9f;
  const size_t gb = (size_t)3 * ngrid * 8, pb = (size_t)3 * n_intp * 8;
  double *dgrid = nullptr, *drho = nullptr, *dpts = nullptr, *dprev = nullptr, *dacc = nullptr;
  int *downer = nullptr, *dsel = nullptr;
  int rc = NGW_OK;
  std::vector<double> prev(pts, pts + 3 * (size_t)n_intp);
  std::vector<int> gsel(n_intp);
  std::vector<unsigned char> used(ngrid);
  int it = 1;
  do {
    if (dalloc(s, (void **)&dgrid, gb) || dalloc(s, (void **)&drho, (size_t)ngrid * 8) || dalloc(s, (void **)&dpts, pb) ||
        dalloc(s, (void **)&dprev, pb) || dalloc(s, (void **)&dacc, (size_t)4 * n_intp * 8) ||
        dalloc(s, (void **)&downer, (size_t)ngrid * 4) || dalloc(s, (void **)&dsel, (size_t)n_intp * 4)) {
      rc = NGW_ERR_OOM;
      break;
    }
    if (cudaMemcpyAsync(dgrid, grid, gb, cudaMemcpyHostToDevice, s->stream) ||
        cudaMemcpyAsync(drho, rho, (size_t)ngrid * 8, cudaMemcpyHostToDevice, s->stream)) {
      set_error("copy to device failed");
      rc = NGW_ERR_CUDA;
      break;
    }
    for (; it <= max_iter; ++it) {
      if (cudaMemcpyAsync(dpts, pts, pb, cudaMemcpyHostToDevice, s->stream) ||
          cudaMemcpyAsync(dprev, prev.data(), pb, cudaMemcpyHostToDevice, s->stream)) {
        set_error("copy to device failed");
        rc = NGW_ERR_CUDA;
        break;
      }
      k_cvt_assign<<<(ngrid + 255) / 256, 256, 0, s->stream>>>(dgrid, ngrid, dpts, n_intp, far, downer);
      k_cvt_accumulate<<<(n_intp + 63) / 64, 64, 0, s->stream>>>(dgrid, drho, downer, ngrid, n_intp, dacc);
      k_cvt_newpos<<<(n_intp + 127) / 128, 128, 0, s->stream>>>(dacc, dprev, n_intp, wtiny, dpts);
      k_cvt_nearest_point<<<n_intp, 256, 0, s->stream>>>(dgrid, ngrid, dpts, dmin0, dsel);
      if (cudaGetLastError() != cudaSuccess ||
          cudaMemcpyAsync(pts, dpts, pb, cudaMemcpyDeviceToHost, s->stream) ||
          cudaMemcpyAsync(gsel.data(), dsel, (size_t)n_intp * 4, cudaMemcpyDeviceToHost, s->stream) ||
          cudaStreamSynchronize(s->stream)) {
        set_error("CVT iteration failed on the device");
        rc = NGW_ERR_CUDA;
        break;
      }
      // snap to the closest grid point not taken earlier in this sweep
      std::fill(used.begin(), used.end(), 0);
      double moved = 0.0;
      for (int p = 0; p < n_intp; ++p) {
        double *pp = pts + 3 * (size_t)p;
        int g = gsel[p];
        if (g >= 0 && used[g]) {   // taken: search the untaken points (host, same arithmetic)
          double dmin = dmin0;
          g = -1;
          for (int q = 0; q < ngrid; ++q) {
            if (used[q]) continue;
            const double d = std::sqrt(sqdist_host(pp, grid + 3 * (size_t)q));
            if (d < dmin) {
              dmin = d;
              g = q;
            }
          }
        }
        if (g >= 0) {
          pp[0] = grid[3 * (size_t)g];
          pp[1] = grid[3 * (size_t)g + 1];
          pp[2] = grid[3 * (size_t)g + 2];
          intp[p] = g + 1;
          used[g] = 1;
        }
        moved = moved + std::sqrt(sqdist_host(pp, &prev[3 * (size_t)p]));
      }
      if (moved < tol_conv) break;
      std::memcpy(prev.data(), pts, sizeof(double) * 3 * (size_t)n_intp);
    }
  } while (0);
  cudaStreamSynchronize(s->stream);
  dfree(s, dgrid, gb);
  dfree(s, drho, (size_t)ngrid * 8);
  dfree(s, dpts, pb);
  dfree(s, dprev, pb);
  dfree(s, dacc, (size_t)4 * n_intp * 8);
  dfree(s, downer, (size_t)ngrid * 4);
  dfree(s, dsel, (size_t)n_intp * 4);
  if (rc != NGW_OK) return rc;
  if (iters) *iters = it > max_iter ? max_iter : it;
  return NGW_OK;
}

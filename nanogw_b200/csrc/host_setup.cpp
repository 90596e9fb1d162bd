// Host-side setup of the ISDF path that must be bit-exact with the reference:
// the Shell sort (shared/quicksort.f90:19-70), CVT point selection
// (shared/cvt.F90:8-195, C1 symmetry) and the density de-duplication of the
// selected points (SIGMA/sigma.F90:377-461).  Integer results depend on FP64
// comparisons, so every expression is evaluated in the reference's order and
// this file is compiled with -ffp-contract=off.  The reference's
// single-precision literals (tol_conv = 1e-3, 1.0e-10, 100.0, 1.e9, 1.0e-14)
// are the same float values promoted to double.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/ngw_b200.h"

namespace ngw {
void set_error(const char *fmt, ...);
}

namespace {

// ascending Shell sort of a copy of x, permutation (0-based) in perm
void shell_sort_perm(int n, const double *x_in, int *perm) {
  for (int i = 0; i < n; ++i) perm[i] = i;
  if (n <= 1) return;
  std::vector<double> x(x_in, x_in + n);
  for (int gap = n / 2; gap > 0; gap /= 2) {
    for (int i = gap; i < n; ++i) {
      for (int j = i - gap; j >= 0; j -= gap) {
        if (!(x[j] > x[j + gap])) break;
        std::swap(x[j], x[j + gap]);
        std::swap(perm[j], perm[j + gap]);
      }
    }
  }
}

inline double sqdist(const double *a, const double *b) {
  const double dx = a[0] - b[0];
  const double dy = a[1] - b[1];
  const double dz = a[2] - b[2];
  double r = dx * dx;
  r = r + dy * dy;
  r = r + dz * dz;
  return r;
}

}  // namespace

extern "C" {

int ngw_shell_sort(int n, const double *arr, int *idx) {
  if (n < 0 || (n > 0 && (!arr || !idx))) {
    ngw::set_error("ngw_shell_sort: bad arguments");
    return NGW_ERR_ARG;
  }
  std::vector<int> p(n);
  shell_sort_perm(n, arr, p.data());
  for (int i = 0; i < n; ++i) idx[i] = p[i] + 1;
  return NGW_OK;
}

int ngw_cvt(int ngrid, const double *grid, const double *rho, int n_intp, double *pts,
            int max_iter, int *intp, int *iters) {
  if (ngrid <= 0 || n_intp <= 0 || n_intp > ngrid || !grid || !rho || !pts || !intp ||
      max_iter <= 0) {
    ngw::set_error("ngw_cvt: bad arguments");
    return NGW_ERR_ARG;
  }
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
  std::vector<double> prev(pts, pts + 3 * (size_t)n_intp);
  std::vector<int> owner(ngrid);
  std::vector<double> acc(4 * (size_t)n_intp);
  std::vector<unsigned char> used(ngrid);
  int it = 1;
  for (; it <= max_iter; ++it) {
    // nearest centre (first minimum)
    for (int g = 0; g < ngrid; ++g) {
      const double *gp = grid + 3 * (size_t)g;
      double best = far;
      int who = -1;
      for (int p = 0; p < n_intp; ++p) {
        const double d = sqdist(pts + 3 * (size_t)p, gp);
        if (d < best) {
          best = d;
          who = p;
        }
      }
      owner[g] = who;
    }
    // weighted centroids accumulated in grid order
    std::fill(acc.begin(), acc.end(), 0.0);
    for (int g = 0; g < ngrid; ++g) {
      const int p = owner[g];
      if (p < 0) continue;
      double *a = &acc[4 * (size_t)p];
      const double *gp = grid + 3 * (size_t)g;
      a[0] = a[0] + gp[0] * rho[g];
      a[1] = a[1] + gp[1] * rho[g];
      a[2] = a[2] + gp[2] * rho[g];
      a[3] = a[3] + rho[g];
    }
    std::fill(used.begin(), used.end(), 0);
    double moved = 0.0;
    for (int p = 0; p < n_intp; ++p) {
      double *pp = pts + 3 * (size_t)p;
      const double *a = &acc[4 * (size_t)p];
      if (a[3] < wtiny) {
        pp[0] = prev[3 * p];
        pp[1] = prev[3 * p + 1];
        pp[2] = prev[3 * p + 2];
      } else {
        pp[0] = a[0] / a[3];
        pp[1] = a[1] / a[3];
        pp[2] = a[2] / a[3];
      }
      // snap to the closest grid point not taken in this sweep
      double dmin = (double)1.e9f;
      int gsel = -1;
      for (int g = 0; g < ngrid; ++g) {
        if (used[g]) continue;
        const double d = std::sqrt(sqdist(pp, grid + 3 * (size_t)g));
        if (d < dmin) {
          dmin = d;
          gsel = g;
        }
      }
      if (gsel >= 0) {
        pp[0] = grid[3 * (size_t)gsel];
        pp[1] = grid[3 * (size_t)gsel + 1];
        pp[2] = grid[3 * (size_t)gsel + 2];
        intp[p] = gsel + 1;
        used[gsel] = 1;
      }
      moved = moved + std::sqrt(sqdist(pp, &prev[3 * (size_t)p]));
    }
    if (moved < tol_conv) break;
    std::memcpy(prev.data(), pts, sizeof(double) * 3 * (size_t)n_intp);
  }
  if (iters) *iters = it > max_iter ? max_iter : it;
  return NGW_OK;
}

int ngw_dedup_points(int n, const int *intp, const double *rho, int *out, int *nout) {
  if (n < 0 || (n > 0 && (!intp || !rho || !out)) || !nout) {
    ngw::set_error("ngw_dedup_points: bad arguments");
    return NGW_ERR_ARG;
  }
  *nout = 0;
  if (n == 0) return NGW_OK;
  std::vector<double> r(n);
  for (int i = 0; i < n; ++i) r[i] = rho[intp[i] - 1];
  std::vector<int> perm(n);
  shell_sort_perm(n, r.data(), perm.data());
  std::vector<unsigned char> keep(n, 1);
  const double tol = (double)1.0e-14f;
  int kept = 0;
  for (int i = 0; i + 1 < n; ++i) {
    if (std::fabs(r[perm[i]] - r[perm[i + 1]]) < tol) {
      keep[perm[i]] = 0;
    } else {
      keep[perm[i]] = 1;
      ++kept;
    }
  }
  keep[perm[n - 1]] = 1;
  ++kept;
  int w = 0;
  for (int i = 0; i < n && w < kept; ++i)
    if (keep[i]) out[w++] = intp[i];
  *nout = w;
  return NGW_OK;
}

}  // extern "C"

/* Oracle (test infrastructure only): CVT interpolation-point selection and the
 * Shell sort used by NanoGW, restated in plain C.
 *
 *  - ngw_oracle_shell_sort   : shared/quicksort.f90:19-70 (ascending Shell sort
 *                              returning a 1-based permutation; not stable, so
 *                              the exact gap sequence matters for ties).
 *  - ngw_oracle_cvt          : shared/cvt.F90:8-195 (C1 symmetry, ntrans = 1).
 *
 * Bit-exactness: compiled with -ffp-contract=off so every FP64 operation is
 * rounded exactly where the Fortran source rounds it.  Single-precision
 * literals of the reference (tol_conv = 1e-3, 1.0e-10, 100.0, 1.e9) are used
 * as the same float values promoted to double.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

void ngw_oracle_shell_sort(int nn, const double *arrin, int *indx) {
    for (int i = 0; i < nn; ++i) indx[i] = i + 1;
    if (nn <= 1) return;
    double *x = (double *)malloc(sizeof(double) * (size_t)nn);
    memcpy(x, arrin, sizeof(double) * (size_t)nn);
    int igap = nn / 2;
    while (igap > 0) {
        for (int i = igap; i < nn; ++i) {
            int j = i - igap;
            while (j >= 0) {
                if (x[j] > x[j + igap]) {
                    double t = x[j]; x[j] = x[j + igap]; x[j + igap] = t;
                    int it = indx[j]; indx[j] = indx[j + igap]; indx[j + igap] = it;
                } else {
                    break;
                }
                j -= igap;
            }
        }
        igap /= 2;
    }
    free(x);
}

/* grid: (ngrid, 3) row-major coordinates in grid order; rho: (ngrid);
 * pts: (n_intp, 3) initial centres (overwritten with the final ones);
 * intp: (n_intp) 1-based selected grid indices.  Returns iterations used. */
int ngw_oracle_cvt(int ngrid, const double *grid, const double *rho, int n_intp,
                   double *pts, int max_iter, int *intp) {
    const double tol_conv = (double)1e-3f;
    const double wtiny = (double)1.0e-10f;
    double bounds[2][3];
    for (int d = 0; d < 3; ++d) {
        double lo = grid[d], hi = grid[d];
        for (int g = 1; g < ngrid; ++g) {
            double v = grid[3 * g + d];
            if (v < lo) lo = v;
            if (v > hi) hi = v;
        }
        bounds[0][d] = lo; bounds[1][d] = hi;
    }
    double bmax = bounds[1][0], bmin = bounds[0][0];
    for (int d = 1; d < 3; ++d) {
        if (bounds[1][d] > bmax) bmax = bounds[1][d];
        if (bounds[0][d] < bmin) bmin = bounds[0][d];
    }
    double dinit = (double)100.0f * ((bmax - bmin) * (bmax - bmin));
    double *oldp = (double *)malloc(sizeof(double) * 3 * (size_t)n_intp);
    double *wsum = (double *)malloc(sizeof(double) * 3 * (size_t)n_intp);
    double *wt = (double *)malloc(sizeof(double) * (size_t)n_intp);
    int *icenter = (int *)malloc(sizeof(int) * (size_t)ngrid);
    unsigned char *taken = (unsigned char *)calloc((size_t)ngrid, 1);
    int *sel = (int *)malloc(sizeof(int) * (size_t)n_intp);
    memcpy(oldp, pts, sizeof(double) * 3 * (size_t)n_intp);
    int iter;
    for (iter = 1; iter <= max_iter; ++iter) {
        /* nearest centre, first minimum wins (cvt.F90:108-121) */
        for (int g = 0; g < ngrid; ++g) {
            double dist = dinit;
            int ic = -1;
            const double gx = grid[3 * g], gy = grid[3 * g + 1], gz = grid[3 * g + 2];
            for (int p = 0; p < n_intp; ++p) {
                double vx = pts[3 * p] - gx, vy = pts[3 * p + 1] - gy, vz = pts[3 * p + 2] - gz;
                double dt = vx * vx;
                dt = dt + vy * vy;
                dt = dt + vz * vz;
                if (dt < dist) { dist = dt; ic = p; }
            }
            icenter[g] = ic;
        }
        /* rho-weighted centroids, summed in grid order (cvt.F90:126-142) */
        for (int p = 0; p < n_intp; ++p) { wsum[3 * p] = wsum[3 * p + 1] = wsum[3 * p + 2] = 0.0; wt[p] = 0.0; }
        for (int g = 0; g < ngrid; ++g) {
            int p = icenter[g];
            if (p < 0) continue;
            wsum[3 * p] = wsum[3 * p] + grid[3 * g] * rho[g];
            wsum[3 * p + 1] = wsum[3 * p + 1] + grid[3 * g + 1] * rho[g];
            wsum[3 * p + 2] = wsum[3 * p + 2] + grid[3 * g + 2] * rho[g];
            wt[p] = wt[p] + rho[g];
        }
        double diff = 0.0;
        memset(taken, 0, (size_t)ngrid);
        for (int p = 0; p < n_intp; ++p) {
            if (wt[p] < wtiny) {
                pts[3 * p] = oldp[3 * p]; pts[3 * p + 1] = oldp[3 * p + 1]; pts[3 * p + 2] = oldp[3 * p + 2];
            } else {
                pts[3 * p] = wsum[3 * p] / wt[p];
                pts[3 * p + 1] = wsum[3 * p + 1] / wt[p];
                pts[3 * p + 2] = wsum[3 * p + 2] / wt[p];
            }
            /* snap to the nearest grid point not yet chosen in this sweep
             * (cvt.F90:143-174); strict '<' keeps the first minimum. */
            double mindist = (double)1.e9f;
            int ming = -1;
            for (int g = 0; g < ngrid; ++g) {
                if (taken[g]) continue;
                double vx = pts[3 * p] - grid[3 * g], vy = pts[3 * p + 1] - grid[3 * g + 1],
                       vz = pts[3 * p + 2] - grid[3 * g + 2];
                double dt = vx * vx;
                dt = dt + vy * vy;
                dt = dt + vz * vz;
                double d = sqrt(dt);
                if (d < mindist) { mindist = d; ming = g; }
            }
            if (ming >= 0) {
                pts[3 * p] = grid[3 * ming]; pts[3 * p + 1] = grid[3 * ming + 1]; pts[3 * p + 2] = grid[3 * ming + 2];
                intp[p] = ming + 1;
                taken[ming] = 1;
                sel[p] = ming;
            }
            double vx = pts[3 * p] - oldp[3 * p], vy = pts[3 * p + 1] - oldp[3 * p + 1],
                   vz = pts[3 * p + 2] - oldp[3 * p + 2];
            double dt = vx * vx;
            dt = dt + vy * vy;
            dt = dt + vz * vz;
            diff = diff + sqrt(dt);
        }
        if (diff < tol_conv) break;
        memcpy(oldp, pts, sizeof(double) * 3 * (size_t)n_intp);
    }
    free(oldp); free(wsum); free(wt); free(icenter); free(taken); free(sel);
    return iter > max_iter ? max_iter : iter;
}

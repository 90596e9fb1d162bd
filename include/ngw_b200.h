/*
 * ngw_b200 -- C ABI of the B200-native ISDF-Lanczos GW (Sigma_c) path.
 *
 * Every entry point takes plain pointers and sizes, returns an int status
 * (NGW_OK = 0; the Fortran shim calls die() on non-zero, as the reference's
 * shared/die.F90:10 does) and leaves the human-readable reason in
 * ngw_last_error().  Arrays are column-major with Fortran leading dimensions
 * and band / pair indices are 1-based, exactly as the reference passes them.
 * Energies are in Rydberg.  Host pointers are never kept after a call
 * returns; the session owns its device-resident copies.  A session is used by
 * one host thread at a time; calls are synchronous to the caller.
 *
 * Reference interfaces replaced (file:line in the NanoGW tree):
 *   ngw_set_isdf / ngw_set_pairs  -- the isdf_in%Psi_intp / Mmtrx / cvpair /
 *        sqrtR arguments of shared/apply_matvec.f90:25 and
 *        shared/apply_matvec_BLOCK.F90:25 (type ISDF, shared/typedefs.F90:24-72)
 *   ngw_matvec_isdf               -- matvec_isdf            shared/apply_matvec.f90:25
 *                                    matvec_isdf_BLOCK      shared/apply_matvec_BLOCK.F90:25
 *                                    matvec_isdf_lowcomsym  shared/apply_matvec_lowcomsym.F90:31
 *   ngw_polynomial_matvec_isdf    -- polynomial_matvec_isdf shared/apply_matvec.f90:142
 *                                    (_BLOCK :210, _lowcomsym :419)
 *   ngw_lanczos_spectra_isdf      -- lanczos_spectra_isdf   shared/lanczos_spectra.f90:7
 *                                    (_BLOCK shared/lanczos_spectra_BLOCK.F90:7,
 *                                     _lowcomsym shared/lanczos_spectra_lowcomsym.F90:7)
 *   ngw_k_integrate_isdf          -- Zk_integrate_isdf      shared/k_integrate_isdf.F90z:12
 *   ngw_sigma_lanczos             -- Zcalculate_sigma_lanczos(_lowcomsym)
 *                                    SIGMA/calculate_sigma_lanczos_lowcomsym.F90z:9
 *   ngw_qp_newton                 -- QP part of printsigma  SIGMA/printsigma.F90:97-125
 *                                    (newtonr SIGMA/newtonr.f90:18)
 *   ngw_cvt / ngw_dedup_points    -- cvt shared/cvt.F90:8 and SIGMA/sigma.F90:377-461
 *   ngw_cvt_device                -- cvt shared/cvt.F90:8, iterations on the device
 *   ngw_shell_sort                -- quicksort shared/quicksort.f90:19
 *   ngw_build_coulomb_kernel      -- Mmtrx build, shared/isdf_parallel_sym_UltraLowMem.F90:687-889
 *                                    (dpoisson shared/fft_module.F90z:122,
 *                                     dcreate_coul_0D shared/fft_module.F90z:628)
 *   ngw_build_fxc_kernel          -- f_xc block, shared/isdf_parallel_sym_UltraLowMem.F90:809-839
 *   ngw_build_isdf_kernel         -- ISDF fit + both kernel blocks on the device,
 *                                    shared/isdf_parallel_sym_UltraLowMem.F90:439-889
 *   ngw_parsec_read / _write      -- parsec_wfn              shared/parsec_wfn.F90:20 (file
 *                                    records :80-320,663-700)
 *   ngw_fock_exchange             -- Zfock_exchange          SIGMA/fock_exchange.F90z:2
 *   ngw_vxc_matrix                -- Zvxc / Zvxcmtxel        SIGMA/vxc.F90z:2,
 *                                    shared/vxcmtxel.F90z:2
 */
#ifndef NGW_B200_H
#define NGW_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define NGW_OK 0
#define NGW_ERR_ARG 1        /* bad shape / argument */
#define NGW_ERR_OOM 2        /* device allocation failed */
#define NGW_ERR_CUDA 3       /* CUDA runtime / library error */
#define NGW_ERR_TIMEOUT 4    /* a bounded device wait gave up */
#define NGW_ERR_NONFINITE 5  /* NaN / Inf in an input */
#define NGW_ERR_BUDGET 6     /* over the memory budget */
#define NGW_ERR_STATE 7      /* call order (e.g. no operator set) */
#define NGW_ERR_NOCONV 8     /* QP Newton did not converge */

/* precision modes of the matvec */
#define NGW_PREC_FP64 0      /* FP64 GEMMs + Horner: the reference's arithmetic */
#define NGW_PREC_MIXED 1     /* split-BF16 tcgen05 GEMMs (FP32 accumulate),
                                Chebyshev-Clenshaw form of the same polynomial,
                                FP64 Lanczos recurrence / continued fraction */

typedef struct ngw_session ngw_session;

int ngw_version(void);
const char *ngw_last_error(void);

int ngw_session_create(int device, ngw_session **out);
void ngw_session_destroy(ngw_session *s);
/* cudaStream_t of the session, as an opaque pointer (for event timing) */
void *ngw_session_stream(ngw_session *s);
int ngw_set_precision(ngw_session *s, int mode);
/* bytes of device memory the session holds now */
long long ngw_session_bytes(ngw_session *s);

/* ISDF operator: psi_intp (n_isdf x nmem), mmtrx (n_isdf x n_isdf) Coulomb
 * block, mxc optional (n_isdf x n_isdf) f_xc block or NULL. */
int ngw_set_isdf(ngw_session *s, int n_isdf, int nmem, const double *psi_intp,
                 const double *mmtrx, const double *mxc);
/* valence-conduction pairs: cvpair (2 x ncv) 1-based (v, c); sqrtR (ncv) */
int ngw_set_pairs(ngw_session *s, int ncv, const int *cvpair, const double *sqrtR);

/* Hvec = H vec for blksz columns (ld >= ncv).  tamm_d != 0: A = R + 2 C^T M C */
int ngw_matvec_isdf(ngw_session *s, const double *vec, double *hvec, int ld,
                    int blksz, int tamm_d);
/* Hvec = p(H) vec, polynomial (npoly+1) stored high -> low */
int ngw_polynomial_matvec_isdf(ngw_session *s, const double *polynomial, int npoly,
                               const double *vec, double *hvec, int ld, int blksz);
/* spectra(iz, j) = <v_j|(zz(iz,j) - p(H))^-1|v_j>, v_j = v0(:,j)/v0_norm(j).
 * zz / spectra: complex128 interleaved (nz x blksz).  alpha / beta (niter x
 * blksz) may be NULL.  tamm_d != 0 uses H = A and ignores the polynomial. */
int ngw_lanczos_spectra_isdf(ngw_session *s, const double *v0, const double *v0_norm,
                             int ld, const double *zz, int nz, int niter,
                             const double *polynomial, int npoly, int blksz, int tamm_d,
                             double *spectra, double *alpha, double *beta);
/* kmat(i, j) = (psi_r1 psi_r2)^T M (psi_c1 psi_c2) for row pairs rows(2, nrow)
 * and column pairs cols(2, ncol) (1-based bands);
 * M = [kflag < 2] M_C + [kflag > 0] M_xc.  kmat: nrow x ncol column-major. */
int ngw_k_integrate_isdf(ngw_session *s, int kflag, const int *rows, int nrow,
                         const int *cols, int ncol, double *kmat);

typedef struct {
  int nen;                 /* energy points per QP state */
  double deltae;           /* energy range (Ry) of the grid centred on e1(m) */
  double ecuts;            /* broadening eta (Ry) */
  int niter;               /* Lanczos steps */
  int npoly;               /* polynomial degree (ignored with tamm_d) */
  const double *polynomial;/* npoly+1 coefficients high -> low */
  int tamm_d;              /* Tamm-Dancoff */
  int nval;                /* occupied bands (eta_n = +1 for n <= nval) */
  int nqp;                 /* number of QP states */
  const int *qp_bands;     /* nqp 1-based band indices m */
  int nbands_sum;          /* bands n summed over: 1..nbands_sum (0 = nmem) */
  int block_chains;        /* chains per device block (0 = all that fit) */
  double cheb_lo, cheb_hi; /* mixed mode: Chebyshev interval (0,0 = auto) */
  const int *chain_niter;  /* optional per-chain Lanczos lengths 1..niter, nqp x nbands_sum
                              (chain = iq*nbands_sum + n-1); NULL = niter for every chain */
  double early_exit_eps;   /* > 0: a chain stops when |b_k| < eps (convergence mask, as
                              shared/lanczos_spectra.f90:24,58); 0 = never (lowcomsym) */
  int reorth;              /* 1: full reorthogonalisation of every chain (classical Gram-Schmidt
                              against all its earlier Lanczos vectors, applied twice, FP64); the
                              reference recurrence has none (shared/lanczos_spectra_lowcomsym.F90
                              :117-166), so 0 reproduces it.  The Krylov bases take
                              chains x (niter+1) x ncv x 8 bytes: the QP states are blocked so
                              they fit NGW_REORTH_MAX_GB (default 40 % of free device memory);
                              NGW_ERR_BUDGET when one QP state does not fit.  niter <= 6000. */
} ngw_sigma_params;

/* ngw_lanczos_spectra_isdf with per-chain lengths and a convergence mask:
 * chain_niter (blksz, 1..niter, NULL = niter) and early_exit_eps (> 0: a
 * chain stops when |b_k| < eps; its later alpha / beta are 0 and its
 * continued fraction ends there).  The single-vector reference routine
 * (lanczos_spectra_isdf, shared/lanczos_spectra.f90:7) is this call with
 * blksz = 1 and eps = 1e-8 (:24,58); the BLOCK / lowcomsym forms have no exit
 * (eps = 0, what ngw_lanczos_spectra_isdf does). */
int ngw_lanczos_spectra_isdf_masked(ngw_session *s, const double *v0, const double *v0_norm, int ld,
                                    const double *zz, int nz, int niter, const double *polynomial,
                                    int npoly, int blksz, int tamm_d, const int *chain_niter,
                                    double early_exit_eps, double *spectra, double *alpha,
                                    double *beta);

/* Sigma_c(omega) for every QP state: sigma_c complex128 interleaved,
 * (nen x nqp) column-major, in Ry.  e1: KS energies (nmem), Ry.
 * alpha/beta (niter x nchains, chain = iq*nbands_sum + n) optional; entries
 * past a chain's length (or its convergence stop) are 0.  With per-chain
 * lengths the chains of a block run longest first and each step's matvecs
 * cover only the chains still running. */
int ngw_sigma_lanczos(ngw_session *s, const ngw_sigma_params *p, const double *e1,
                      double *sigma_c, double *alpha, double *beta);

/* Batched Sigma_c of several molecules, one per session (sessions on one
 * device, each with its operator set): entry i solves params[i] with KS
 * energies e1[i] into sigma_c[i].  Mixed precision (all entries, no TDA, one
 * polynomial degree): the molecules' Lanczos recurrences run in lock step on
 * session 0's stream and each Clenshaw term of their p(C) v is one grouped
 * tcgen05 GEMM launch per operand product across all molecules (64-wide
 * tiles; bit-identical to single calls pinned to those tiles, QP energies
 * within 1 meV of single calls on their tuned tiles), one grouped
 * Lanczos-step launch per step.  Otherwise (FP64, TDA, or
 * NGW_BATCH_MODE=branches) entry i is a branch on session i's stream, forked
 * from and joined into session 0's stream, with the kernels and tiles of
 * ngw_sigma_lanczos (bit-identical results).  Either way the batch is one
 * CUDA graph, captured on the second call with the same shapes and replayed
 * by one launch afterwards.  Each entry's chains must fit one block
 * (block_chains 0 or >= nqp * nbands_sum).  The batched configuration of the
 * benchmarks (uneven molecules, per-chain lengths) runs through this call.
 * No reference counterpart: NanoGW blocks bands of one molecule only
 * (SIGMA/calculate_sigma_lanczos_lowcomsym.F90z:477-511). */
int ngw_sigma_lanczos_batch(ngw_session *const *sessions, int count, const ngw_sigma_params *params,
                            const double *const *e1, double *const *sigma_c);

/* QP Newton solve on the device (eV in, eV out), one state per column:
 * sigma_c (nen x nqp complex, eV), e1/e0/sigx/vxc (nqp) eV.
 * Grid: x_i = e1 - deltae/2 + deltae/(nen-1)*(i-1).  Tolerance xacc (eV). */
int ngw_qp_newton(ngw_session *s, int nqp, int nen, const double *sigma_c_ev,
                  const double *e1_ev, const double *e0_ev, double deltae_ev,
                  const double *sigx_ev, const double *vxc_ev, double xacc_ev,
                  double *eqp_ev, double *zfac, int *ierr);

/* QP Newton solve that allocates nothing; no counterpart in the reference.
 * For callers that cannot call cudaMalloc (a driver that hands out device
 * memory from its own pool, code running during stream capture, a process
 * whose allocator holds all free memory).  Every pointer is a DEVICE pointer
 * with the layout of ngw_qp_newton; the call is ordered on `stream`
 * (cudaStream_t, NULL = default stream) and returns without synchronising.
 * The spline workspace is a fixed device array of 2^18 doubles shared by all
 * calls on a device: nqp * 4 * nen must not exceed 262144 (NGW_ERR_BUDGET
 * otherwise), and calls whose kernels overlap on the GPU race on it.  The
 * first call on each device looks up the array's address; make it before any
 * stream capture. */
int ngw_qp_newton_noalloc(int nqp, int nen, const double *sigma_c_ev, const double *e1_ev,
                          const double *e0_ev, double deltae_ev, const double *sigx_ev,
                          const double *vxc_ev, double xacc_ev, double *eqp_ev, double *zfac,
                          int *ierr, void *stream);

/* ---- measurement ---- */
/* FP64 GEMM on the FP64 tensor cores, the kernel behind every FP64 contraction
 * of this library except the plain FP64 matvec (which stays on cuBLAS as the
 * comparison path): C = alpha op(A) op(B) + beta C with column-major DEVICE
 * pointers and cuBLAS's argument meaning (transa/transb 0 = N, 1 = T).  An
 * optional device workspace (ws, ws_bytes; 64 m n doubles cover every choice)
 * lets small tile grids split K, summed in a fixed order.  Ordered on
 * `stream` (cudaStream_t, NULL = default), no synchronisation.  No reference
 * counterpart (the reference calls BLAS dgemm): used by the tests and the
 * benchmark's FP64 GEMM line. */
int ngw_dgemm(int transa, int transb, int m, int n, int k, double alpha, const double *A, int lda,
              const double *B, int ldb, double beta, double *C, int ldc, double *ws, long long ws_bytes,
              void *stream);
/* Average device time (us) of one launch of each mixed-precision GEMM for nb
 * chains (GEMM1: T = C_isdf S, GEMM2: Z = (M C_isdf)^T T with its Clenshaw
 * epilogue), from CUDA events around `reps` back-to-back launches on the
 * session stream.  No reference counterpart: used by the benchmark. */
int ngw_profile_mixed_gemms(ngw_session *s, int nb, int reps, double *us_gemm1, double *us_gemm2);
/* shape[13] = {M1, N1, K1, BN1, splitK1, M2, N2, K2, BN2, variant1, variant2,
 * splitK2, 0} of the two GEMMs (valid sizes, N tile, split-K, kernel
 * variant; split-K > 1 of GEMM2 only with the cluster variants 5 / 6). */
int ngw_mixed_gemm_shapes(ngw_session *s, int nb, int *shape);
/* The mixed form's dense p(C) GEMM (built when the last mixed plan chose the
 * dense form, small N_cv): mean device time of one launch for nb chains to
 * *us and shape[5] = {M, N, K, N tile, 16 x variant + split-K}; NGW_ERR_STATE when the
 * session's plan used the factored form.  No reference counterpart: used by
 * the benchmark. */
int ngw_profile_dense_gemm(ngw_session *s, int nb, int reps, double *us, int *shape);

/* Top Ritz pairs of the Casida operator (tamm_d 0: C = R^2 + 4 R^1/2 K R^1/2,
 * 1: the TDA matrix A) from an FP64 Lanczos run of msteps steps with full
 * reorthogonalisation started from a fixed pseudo-random vector: the kmax
 * largest Ritz values (descending, Ry^2 or Ry) to vals and their residual
 * bounds |beta_m y_m| to res; *count = number written (<= min(kmax, msteps)).
 * These are the eigenpairs the mixed-precision path deflates.  No reference
 * counterpart (the reference's Lanczos has no deflation). */
int ngw_operator_eigenpairs(ngw_session *s, int tamm_d, int msteps, int kmax, double *vals,
                            double *res, int *count);

/* ---- setup path ---- */
/* Shell sort (ascending) returning a 1-based permutation. Host code. */
int ngw_shell_sort(int n, const double *arr, int *idx);
/* CVT interpolation points; grid (3 x ngrid), pts (3 x n_intp) in/out,
 * intp (n_intp) 1-based grid indices.  Bit-exact with the reference loops. */
int ngw_cvt(int ngrid, const double *grid, const double *rho, int n_intp, double *pts,
            int max_iter, int *intp, int *iters);
/* ngw_cvt with the O(N_grid x N_mu) work of every iteration on the device
 * (nearest centres, weighted centroids, nearest grid points) and the
 * order-dependent snap on the host; results bit-identical to ngw_cvt
 * (separately rounded products and sums, the same summation orders). */
int ngw_cvt_device(ngw_session *s, int ngrid, const double *grid, const double *rho, int n_intp,
                   double *pts, int max_iter, int *intp, int *iters);
/* de-duplicate CVT points by density (C1): returns the kept count in *nout */
int ngw_dedup_points(int n, const int *intp, const double *rho, int *out, int *nout);
/* Coulomb ISDF kernel: M = ntrans/hcub * zeta^T (v_c zeta) on the device.
 * zeta (ngrid x n_isdf) column-major, grid_idx (3 x ngrid) integer coords,
 * nfft box edge, h spacing, trunc = 2*rmax.  mmtrx out (n_isdf x n_isdf). */
int ngw_build_coulomb_kernel(ngw_session *s, int ngrid, int n_isdf, const double *zeta,
                             const int *grid_idx, int nfft, double h, double trunc,
                             double *mmtrx);

/* f_xc block: M_xc = ntrans/hcub * zeta^T (f_xc * zeta), f_xc the LDA kernel
 * of rho (shared/xc_module.F90:853-893, Ry bohr^3) -- replaces
 * shared/isdf_parallel_sym_UltraLowMem.F90:809-839.  rho (ngrid) > 0;
 * fxc_out (ngrid) optional. */
int ngw_build_fxc_kernel(ngw_session *s, int ngrid, int n_isdf, const double *zeta,
                         const double *rho, double h, double *mxc, double *fxc_out);

/* ISDF fit and kernel on the device (shared/isdf_parallel_sym_UltraLowMem.F90:439-889):
 * psi (ngrid x nmem) orbitals on the grid, intp (n_isdf) 1-based grid indices
 * of the interpolation points (after ngw_dedup_points), mv = highest band of
 * the "valence" product P (max(nval, QP bands)).  Fits zeta from
 *   P = psi_intp[:, :mv] psi[:, :mv]^T,  Q = psi_intp psi^T,
 *   A = P_intp * Q_intp,  B = P * Q,  A zeta^T = B  (LU, partial pivoting)
 * and builds M_C (and M_xc when rho != NULL) without copying zeta to the host.
 * Out: psi_intp (n_isdf x nmem), mmtrx (n_isdf x n_isdf), mxc (same; needed
 * when rho is given).  A singular A (repeated points) returns NGW_ERR_ARG. */
int ngw_build_isdf_kernel(ngw_session *s, int ngrid, int nmem, const double *psi,
                          const int *grid_idx, int n_isdf, const int *intp, int mv, int nfft,
                          double h, double trunc, const double *rho, double *psi_intp,
                          double *mmtrx, double *mxc);

/* PARSEC wavefunction file (parsec.dat), finite system, real orbitals, one
 * spin channel, in the record order shared/parsec_wfn.F90 reads.  Arrays
 * are in file order (the reader's density reordering is ngw_shell_sort's
 * job): gtable (3 x nwedge) integer grid coordinates, rho (nwedge), irep /
 * e0 (Ry) / occ (nstate), iord (nwfn, 1-based state of each stored
 * wavefunction), wfn (nwedge x nwfn), trans (3 x 3 x ntrans), chi
 * (ntrans x ntrans).  Read: ngw_parsec_read_header fills the sizes, the
 * caller allocates, ngw_parsec_read fills the arrays.  Periodic, complex or
 * spin-polarised files return NGW_ERR_ARG. */
typedef struct {
  char datelabel[27];
  int nspin, lcplx, per, ndim, nwedge, ntrans, nstate, nwfn;
  double step;
  double shift[3];
} ngw_parsec_header;
int ngw_parsec_read_header(const char *path, ngw_parsec_header *h);
int ngw_parsec_read(const char *path, ngw_parsec_header *h, int *gtable, double *rho, int *irep,
                    double *e0, double *occ, int *iord, double *wfn, double *trans, int *chi);
int ngw_parsec_write(const char *path, const ngw_parsec_header *h, const int *gtable,
                     const double *rho, const int *irep, const double *e0, const double *occ,
                     const int *iord, const double *wfn, const double *trans, const int *chi);

/* Bare exchange matrix Sigma_x (Ry) between the Sigma bands, finite system,
 * one spin, C1 (SIGMA/fock_exchange.F90z:16-228):
 *   K_x(m1, m2) = -(ntrans / h^3) sum_{n <= maxv} occ_n <psi_m1 | psi_n V_c[psi_n psi_m2]>
 * with V_c the FFT-Poisson solve of ngw_build_coulomb_kernel (box nfft, spacing
 * h, truncation radius trunc) and maxv the highest band with occ > 0.01.
 * psi (ngrid x nmem) orbitals on the grid (sum psi^2 ntrans = 1), grid_idx
 * (3 x ngrid), occ (nmem) occupations per spin, sig_bands (nsig, 1-based).
 * kx out: (nsig x nsig), symmetric. */
int ngw_fock_exchange(ngw_session *s, int ngrid, int nmem, const double *psi, const int *grid_idx,
                      int nfft, double h, double trunc, const double *occ, int nsig,
                      const int *sig_bands, int ntrans, double *kx);

/* V_xc matrix elements (Ry) of the LDA (Slater exchange + Perdew-Zunger
 * correlation, x2 to Rydberg as shared/xc_module.F90:523-829) between the
 * Sigma bands: V(m1, m2) = ntrans <psi_m1 | v(rho) | psi_m2>
 * (SIGMA/vxc.F90z:147-165, shared/vxcmtxel.F90z).  rho (ngrid) > 0.
 * vxc out (nsig x nsig); vx (optional) the exchange part alone. */
int ngw_vxc_matrix(ngw_session *s, int ngrid, int nmem, const double *psi, const double *rho, int nsig,
                   const int *sig_bands, int ntrans, double *vxc, double *vx);

#ifdef __cplusplus
}
#endif
#endif

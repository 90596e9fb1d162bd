"""CPU oracle for the ISDF-Lanczos GW (Sigma_c) path -- TEST INFRASTRUCTURE ONLY.

This package restates, in plain numpy (FP64) and a little C, the algorithm of
NanoGW's Lanczos GW self-energy path so that the CUDA implementation in
``nanogw_b200`` can be checked against it.  Nothing in the product imports it:
only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may call it, and only as the checker / timed CPU baseline.

Each function cites the reference file:line it follows (paths are relative to
the NanoGW source tree).

Parity status
-------------
* Lanczos recurrence + continued fraction: PINNED against the reference's only
  hot-path fixture (``shared/test_lanczos/H_aux_v0.txt``; see
  ``tests/golden/make_golden.py``).
* LDA f_xc: PINNED against libxc's own test-suite tables
  (``LIB/libxc/testsuite/lda_x.data``, ``lda_c_pz.data``).
* CVT point selection, pair maps, ISDF fit, FFT-Poisson, Sigma_c driver and the
  QP Newton solve: the reference ships no fixture for these (and it cannot be
  built here: no gfortran/MPI/FFTW/ScaLAPACK), so parity for them is against
  this restatement only -- "parity unpinned" for those rows.
"""

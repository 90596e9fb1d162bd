"""Host-side setup entry points of the library (bit-exact with the reference):
Shell sort, CVT point selection and density de-duplication."""
import numpy as np

from ._lib import check, lib


def _ptr(a):
    return a.ctypes.data


def shell_sort(arr):
    """1-based ascending permutation by NanoGW's Shell sort (``shared/quicksort.f90``)."""
    a = np.ascontiguousarray(arr, dtype=np.float64)
    idx = np.zeros(len(a), dtype=np.int32)
    check(lib().ngw_shell_sort(len(a), _ptr(a), _ptr(idx)))
    return idx


def cvt(grid, rho, init_pts, max_iter=100000, session=None):
    """CVT interpolation points (``shared/cvt.F90``): returns (intp 1-based, points, iterations).
    With a ``Session`` the iterations run on its device (``ngw_cvt_device``,
    bit-identical to the host form)."""
    g = np.ascontiguousarray(grid, dtype=np.float64)
    r = np.ascontiguousarray(rho, dtype=np.float64)
    p = np.array(init_pts, dtype=np.float64, order="C", copy=True)
    n = p.shape[0]
    intp = np.zeros(n, dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    if session is None:
        check(lib().ngw_cvt(g.shape[0], _ptr(g), _ptr(r), n, _ptr(p), int(max_iter), _ptr(intp), _ptr(it)))
    else:
        check(lib().ngw_cvt_device(session._h, g.shape[0], _ptr(g), _ptr(r), n, _ptr(p), int(max_iter),
                                   _ptr(intp), _ptr(it)))
    return intp, p, int(it[0])


def dedup_points(intp, rho):
    """Density de-duplication of the selected points (``SIGMA/sigma.F90:377-461``, C1)."""
    i = np.ascontiguousarray(intp, dtype=np.int32)
    r = np.ascontiguousarray(rho, dtype=np.float64)
    out = np.zeros(len(i), dtype=np.int32)
    nout = np.zeros(1, dtype=np.int32)
    check(lib().ngw_dedup_points(len(i), _ptr(i), _ptr(r), _ptr(out), _ptr(nout)))
    return out[: nout[0]].copy()

"""PARSEC wavefunction files (``parsec.dat``) through the library's C++
reader / writer (``ngw_parsec_read`` / ``ngw_parsec_write``): the record
order of ``shared/parsec_wfn.F90`` for a finite system with real orbitals and
one spin channel.  Arrays are in file order; ``load_molecule`` applies the
reader's density reordering (``shared/parsec_wfn.F90:468-483``) and returns
the inputs the setup pipeline takes."""
import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import ParsecHeader, check, lib


@dataclass
class ParsecData:
    datelabel: str
    step: float
    ndim: int
    shift: np.ndarray       # (3,)
    gtable: np.ndarray      # (nwedge, 3) int32 grid coordinates
    rho: np.ndarray         # (nwedge,) electron density
    irep: np.ndarray        # (nstate,)
    e0: np.ndarray          # (nstate,) Ry
    occ: np.ndarray         # (nstate,)
    iord: np.ndarray        # (nwfn,) 1-based state of each stored wavefunction
    wfn: np.ndarray         # (nwedge, nwfn)
    trans: np.ndarray       # (ntrans, 3, 3) symmetry operations (Fortran order per operation)
    chi: np.ndarray         # (ntrans, ntrans) int32


def _p(a):
    return a.ctypes.data


def write(path, d: ParsecData):
    h = ParsecHeader()
    h.datelabel = d.datelabel.encode()[:26]
    h.nspin, h.lcplx, h.per = 1, 0, 0
    h.ndim = int(d.ndim)
    h.nwedge = int(d.gtable.shape[0])
    h.ntrans = int(d.chi.shape[0])
    h.nstate = int(len(d.e0))
    h.nwfn = int(len(d.iord))
    h.step = float(d.step)
    for i in range(3):
        h.shift[i] = float(d.shift[i])
    gt = np.ascontiguousarray(d.gtable, dtype=np.int32)
    rho = np.ascontiguousarray(d.rho, dtype=np.float64)
    irep = np.ascontiguousarray(d.irep, dtype=np.int32)
    e0 = np.ascontiguousarray(d.e0, dtype=np.float64)
    occ = np.ascontiguousarray(d.occ, dtype=np.float64)
    iord = np.ascontiguousarray(d.iord, dtype=np.int32)
    wfn = np.asfortranarray(d.wfn, dtype=np.float64)
    trans = np.ascontiguousarray(d.trans, dtype=np.float64)
    chi = np.ascontiguousarray(d.chi, dtype=np.int32)
    check(lib().ngw_parsec_write(str(path).encode(), ctypes.byref(h), _p(gt), _p(rho), _p(irep), _p(e0),
                                 _p(occ), _p(iord), _p(wfn), _p(trans), _p(chi)))


def read(path):
    h = ParsecHeader()
    check(lib().ngw_parsec_read_header(str(path).encode(), ctypes.byref(h)))
    gt = np.zeros((h.nwedge, 3), dtype=np.int32)
    rho = np.zeros(h.nwedge)
    irep = np.zeros(h.nstate, dtype=np.int32)
    e0 = np.zeros(h.nstate)
    occ = np.zeros(h.nstate)
    iord = np.zeros(h.nwfn, dtype=np.int32)
    wfn = np.zeros((h.nwedge, h.nwfn), order="F")
    trans = np.zeros((h.ntrans, 3, 3))
    chi = np.zeros((h.ntrans, h.ntrans), dtype=np.int32)
    check(lib().ngw_parsec_read(str(path).encode(), ctypes.byref(h), _p(gt), _p(rho), _p(irep), _p(e0),
                                _p(occ), _p(iord), _p(wfn), _p(trans), _p(chi)))
    return ParsecData(datelabel=h.datelabel.decode().rstrip(), step=h.step, ndim=h.ndim,
                      shift=np.array(h.shift[:]), gtable=gt, rho=rho, irep=irep, e0=e0, occ=occ,
                      iord=iord, wfn=wfn, trans=trans, chi=chi)


def from_molecule(mol, label="ngw synthetic"):
    """ParsecData of a synthetic molecule (C1: one identity operation, every
    state in representation 1, all orbitals stored)."""
    n = mol.psi.shape[1]
    return ParsecData(datelabel=f"{label} {mol.seed}"[:26], step=float(mol.h), ndim=int(mol.psi.shape[0]),
                      shift=np.zeros(3), gtable=np.asarray(mol.grid_idx, dtype=np.int32), rho=mol.rho.copy(),
                      irep=np.ones(n, dtype=np.int32), e0=mol.e1.copy(), occ=mol.occ.copy(),
                      iord=np.arange(1, n + 1, dtype=np.int32), wfn=np.asfortranarray(mol.psi),
                      trans=np.eye(3)[None, :, :].copy(), chi=np.ones((1, 1), dtype=np.int32))


def load_molecule(path, order_fn=None):
    """A ``synth.Molecule`` from a parsec.dat file the way the reference reader
    prepares it: rmax = the largest |(g + shift) step| over the grid
    (``shared/parsec_wfn.F90:236-247``), grid points reordered by descending
    density with the reference's Shell sort (``:468-483``), orbitals placed by
    iord, nval = the states with occupation above tol_occ = 0.01."""
    from .synth import Molecule
    d = read(path)
    if d.trans.shape[0] != 1:
        raise ValueError("only C1 (one symmetry operation) is supported")
    r = (d.gtable + d.shift[None, :]) * d.step
    rmax = float(np.sqrt(np.max(np.einsum("ij,ij->i", r, r))))
    if order_fn is None:
        from .host import shell_sort as order_fn
    perm = np.asarray(order_fn(-d.rho)) - 1
    nstate = len(d.e0)
    psi = np.zeros((d.gtable.shape[0], nstate))
    psi[:, d.iord - 1] = d.wfn
    occ = d.occ.copy()
    return Molecule(grid_idx=d.gtable[perm].copy(), h=d.step, rmax=rmax,
                    psi=np.ascontiguousarray(psi[perm]), e1=d.e0.copy(), occ=occ,
                    nval=int(np.sum(occ > 0.01)), rho=d.rho[perm].copy(), atoms=np.zeros((0, 3)),
                    meta=dict(datelabel=d.datelabel))

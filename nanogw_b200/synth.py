"""Seeded synthetic molecules for the ISDF-Lanczos GW path.

A molecule is what NanoGW reads from ``parsec.dat`` (``shared/parsec_wfn.F90``):
a real-space grid inside a sphere (spacing ``h``), real orbitals normalised as
``sum_r psi^2 * ntrans = 1`` (``parsec_wfn.F90:724-734``), sorted KS energies
(Rydberg) and occupations, and the density ``rho = 2 sum_v psi_v^2 / hcub``.
Grid points are put in descending-density order with NanoGW's Shell sort, as
the reader does (``parsec_wfn.F90:464-475``), so that point selection sees the
same grid order.

Basis: every atom carries ``shells`` s+p Gaussian shells ``exp(-a r^2)`` with
``a ~ U[0.3, 1.2]``; the shell count is chosen so the basis has more
functions than requested orbitals (the published workload sizes would
otherwise be rank-deficient).  Orbitals are random combinations, Loewdin
orthonormalised on the grid.  Energies: occupied sorted U[-0.75,-0.25] Ha,
empty sorted U[-0.15, 0.5] Ha, stored in Ry.
"""
from dataclasses import dataclass, field

import numpy as np

HA_TO_RY = 2.0


@dataclass
class Molecule:
    grid_idx: np.ndarray        # (ngrid, 3) int32 integer coordinates (shift 0)
    h: float
    rmax: float
    psi: np.ndarray             # (ngrid, nmem) float64
    e1: np.ndarray              # (nmem,) Ry
    occ: np.ndarray             # (nmem,)
    nval: int
    rho: np.ndarray             # (ngrid,)
    atoms: np.ndarray           # (natom, 3)
    seed: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def hcub(self):
        return self.h ** 3

    @property
    def grid(self):
        return self.grid_idx.astype(np.float64) * self.h

    @property
    def nmem(self):
        return self.psi.shape[1]


def sphere_grid(radius, h):
    n = int(np.floor(radius / h))
    r = np.arange(-n, n + 1)
    X, Y, Z = np.meshgrid(r, r, r, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    d2 = (pts.astype(np.float64) * h) ** 2
    keep = d2.sum(axis=1) <= radius * radius
    return pts[keep].astype(np.int32)


def make_molecule(n_atoms, atom_radius, grid_radius, h, n_occ, n_empty, seed,
                  shells=None, order_fn=None):
    """Build a synthetic molecule.  ``order_fn(neg_rho) -> 1-based permutation``
    is the Shell sort used to order the grid (defaults to the library's)."""
    rng = np.random.default_rng(seed)
    nmem = n_occ + n_empty
    # atoms uniform in a sphere
    atoms = []
    while len(atoms) < n_atoms:
        p = rng.uniform(-atom_radius, atom_radius, 3)
        if p @ p <= atom_radius * atom_radius:
            atoms.append(p)
    atoms = np.array(atoms)
    if shells is None:
        shells = int(np.ceil(nmem / (4.0 * n_atoms))) + 1
    gidx = sphere_grid(grid_radius, h)
    r = gidx.astype(np.float64) * h
    nb = 4 * shells * n_atoms
    chi = np.empty((r.shape[0], nb))
    col = 0
    for a in atoms:
        d = r - a[None, :]
        d2 = (d * d).sum(axis=1)
        for _ in range(shells):
            alpha = rng.uniform(0.3, 1.2)
            g = np.exp(-alpha * d2)
            chi[:, col] = g
            chi[:, col + 1] = d[:, 0] * g
            chi[:, col + 2] = d[:, 1] * g
            chi[:, col + 3] = d[:, 2] * g
            col += 4
    coef = rng.standard_normal((nb, nmem))
    phi = chi @ coef
    S = phi.T @ phi
    w, U = np.linalg.eigh(S)
    psi = phi @ (U @ np.diag(w ** -0.5) @ U.T)
    e_occ = np.sort(rng.uniform(-0.75, -0.25, n_occ)) * HA_TO_RY
    e_emp = np.sort(rng.uniform(-0.15, 0.5, n_empty)) * HA_TO_RY
    e1 = np.concatenate([e_occ, e_emp])
    occ = np.concatenate([np.ones(n_occ), np.zeros(n_empty)])
    hcub = h ** 3
    rho = 2.0 * (psi[:, :n_occ] ** 2).sum(axis=1) / hcub
    if order_fn is None:
        from .host import shell_sort as order_fn
    perm = np.asarray(order_fn(-rho)) - 1       # descending density
    gidx = gidx[perm]
    psi = np.ascontiguousarray(psi[perm])
    rho = rho[perm]
    return Molecule(grid_idx=gidx, h=h, rmax=grid_radius, psi=psi, e1=e1, occ=occ,
                    nval=n_occ, rho=rho, atoms=atoms, seed=seed,
                    meta=dict(n_atoms=n_atoms, shells=shells))


def cvt_initial_points(grid, n_intp, seed):
    """Seeded initial CVT centres with NanoGW's formula
    ``bounds_lo + u * 0.9 * (bounds_hi - bounds_lo)`` (``shared/cvt.F90:89-99``,
    the 0.9 being a single-precision literal); the random stream is our own
    because gfortran's generator is not reproducible here."""
    rng = np.random.default_rng(seed + 7919)
    lo = grid.min(axis=0)
    hi = grid.max(axis=0)
    u = rng.uniform(0.0, 1.0, (n_intp, 3))
    return lo[None, :] + u * float(np.float32(0.9)) * (hi - lo)[None, :]


# Workload presets named by their sizes (energies in Ry, lengths in bohr).
CONFIG_SMALL_12ATOM = dict(n_atoms=12, atom_radius=4.0, grid_radius=9.0, h=0.35,
                           n_occ=30, n_empty=90, n_isdf=600, niter=150, n_qp=6,
                           nen=400, deltae=4.0, ecuts=0.02, npoly=12)

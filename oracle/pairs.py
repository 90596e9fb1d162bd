"""Oracle: valence-conduction pair indexing (test infrastructure only).

Three orderings exist in the reference:
* ``setup_g`` order -- conduction outer, valence inner, with occupancy and
  ``tdldacut`` filters (``shared/setup_g.F90z:147-173``);
* ``lowcomsym`` order -- representation, then valence, then conduction
  (``SIGMA/calculate_sigma_lanczos_lowcomsym.F90z:335-416,537-550``);
* the ``pairmap``/``invpairmap`` tables over every (iv <= mv, ic <= mc) combo
  used by ``k_integrate_isdf`` (``SIGMA/sigma.F90:556-569``).
All indices are 1-based as in the reference.
"""
import numpy as np

TOL_OCC = 0.01   # shared/myconstants.F90:51


def setup_g_pairs(vmap, cmap, occ, e0, tdldacut=0.0):
    """(v, c) list in ``setup_g`` order (``shared/setup_g.F90z:154-169``).
    vmap/cmap: 1-based band lists; occ/e0 indexed by band-1."""
    out = []
    for c in cmap:
        occ_c = occ[c - 1]
        if occ_c > 1.0 - TOL_OCC:
            continue
        for v in vmap:
            occ_v = occ[v - 1]
            if occ_v < TOL_OCC:
                continue
            if occ_c > TOL_OCC and occ_v < 1.0 - TOL_OCC:
                continue
            tmp = e0[c - 1] - e0[v - 1]
            if tdldacut > 0.0 and tdldacut < tmp:
                continue
            out.append((v, c))
    return np.array(out, dtype=np.int32).reshape(-1, 2)


def rep_pairs(irep, nval, prod, nmrep):
    """Pairs of representation ``nmrep`` in lowcomsym order.

    irep: (nmem,) 1-based irreducible-representation label of each band;
    prod: (ntrans, ntrans) 1-based product table.  Bands are split into
    valence (1..nval) and conduction (nval+1..nmem) lists per representation
    (``:335-388``); pairs loop jvrep -> v -> (the jcrep with
    prod(jcrep, jvrep) == nmrep) -> c (``:537-550``)."""
    nmem = len(irep)
    ntrans = prod.shape[0]
    lv = [[b for b in range(1, nval + 1) if irep[b - 1] == r] for r in range(1, ntrans + 1)]
    lc = [[b for b in range(nval + 1, nmem + 1) if irep[b - 1] == r] for r in range(1, ntrans + 1)]
    out = []
    for jvrep in range(1, ntrans + 1):
        jcrep = None
        for j in range(1, ntrans + 1):
            jcrep = j
            if prod[j - 1, jvrep - 1] == nmrep:
                break
        for v in lv[jvrep - 1]:
            for c in lc[jcrep - 1]:
                out.append((v, c))
    return np.array(out, dtype=np.int32).reshape(-1, 2)


def lowcomsym_pairs(nval, nmem):
    """C1 special case of :func:`rep_pairs`: v = 1..nval outer, c = nval+1..nmem inner."""
    v = np.repeat(np.arange(1, nval + 1), nmem - nval)
    c = np.tile(np.arange(nval + 1, nmem + 1), nval)
    return np.stack([v, c], axis=1).astype(np.int32)


def pair_maps(irep, mv, mc, prod):
    """``pairmap(iv, ic, irp)`` and ``invpairmap(2, icv, irp)`` over all
    iv <= mv, ic <= mc (``SIGMA/sigma.F90:556-569``).  Returns
    (pairmap (mv, mc) int32 holding the 1-based index within its rep, reps (mv, mc),
    invpairmap dict rep -> (n, 2))."""
    ntrans = prod.shape[0]
    icv = np.zeros(ntrans + 1, dtype=np.int64)
    pairmap = np.zeros((mv, mc), dtype=np.int32)
    reps = np.zeros((mv, mc), dtype=np.int32)
    inv = {r: [] for r in range(1, ntrans + 1)}
    for iv in range(1, mv + 1):
        for ic in range(1, mc + 1):
            vcirp = prod[irep[iv - 1] - 1, irep[ic - 1] - 1]
            icv[vcirp] += 1
            pairmap[iv - 1, ic - 1] = icv[vcirp]
            reps[iv - 1, ic - 1] = vcirp
            inv[vcirp].append((iv, ic))
    inv = {r: np.array(v, dtype=np.int32).reshape(-1, 2) for r, v in inv.items()}
    return pairmap, reps, inv

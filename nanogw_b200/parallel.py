"""Multi-GPU plumbing for the Sigma_c path (one process per GPU).

The path shards by QP state: every rank holds the same molecule's operator
(or its own molecule, for replicas) and solves a contiguous share of the QP
states; Sigma_c(omega) tables are gathered to every rank at the end.  There is
no collective inside the solve -- the reference's per-matvec allreduces
(shared/apply_matvec_lowcomsym.F90:264,295) and per-step scalar allreduces
(shared/lanczos_spectra_lowcomsym.F90:107,113) disappear because a chain
never leaves its GPU.
"""
import numpy as np


def shard_bounds(n, rank, world):
    """Contiguous block of n items for `rank`: the split of
    shared/apply_matvec.f90:56-64 (the first n % world ranks get one more)."""
    incr, res = divmod(n, world)
    if rank < res:
        start = rank * (incr + 1)
        end = start + incr + 1
    else:
        start = res * (incr + 1) + (rank - res) * incr
        end = start + incr
    return start, end


def shard_qp(qp_bands, rank, world):
    qp_bands = np.asarray(qp_bands)
    s, e = shard_bounds(len(qp_bands), rank, world)
    return qp_bands[s:e], s, e


def gather_sigma(sig_local, nqp_total, rank, world, group=None, device=None):
    """All-gather per-rank Sigma_c tables (nen, nqp_local) complex into the full
    (nen, nqp_total) table on every rank (torch.distributed, any backend)."""
    import torch
    import torch.distributed as dist
    nen = sig_local.shape[0]
    counts = [shard_bounds(nqp_total, r, world) for r in range(world)]
    maxq = max(e - s for s, e in counts)
    buf = np.zeros((maxq, nen, 2))
    loc = np.asarray(sig_local)
    buf[: loc.shape[1], :, 0] = loc.T.real
    buf[: loc.shape[1], :, 1] = loc.T.imag
    t = torch.from_numpy(buf)
    if device is not None:
        t = t.to(device)
    outs = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    full = np.zeros((nen, nqp_total), dtype=np.complex128)
    for r, (s, e) in enumerate(counts):
        o = outs[r].cpu().numpy()
        full[:, s:e] = (o[: e - s, :, 0] + 1j * o[: e - s, :, 1]).T
    return full

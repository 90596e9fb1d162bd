"""World-size-2 gloo test of the multi-GPU host logic (QP-state sharding and
the Sigma_c gather), with the oracle as each rank's solver on the CPU."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from nanogw_b200.parallel import shard_bounds


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, qp, out_path):
    import torch.distributed as dist

    from nanogw_b200.parallel import gather_sigma, shard_qp
    from oracle import sigma as OS
    from tests._system import make_small_system
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    S = make_small_system()
    mine, s, e = shard_qp(qp, rank, world)
    loc = np.stack([OS.sigma_c_state(S.psi_intp, S.M, S.e1, S.nval, int(m), 21, 2.0, 0.02, 6, S.poly)
                    for m in mine], axis=1) if len(mine) else np.zeros((21, 0), complex)
    full = gather_sigma(loc, len(qp), rank, world)
    if rank == 0:
        np.save(out_path, full)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_bounds_cover():
    for n in (0, 1, 5, 7, 16):
        for w in (1, 2, 3, 4):
            got = [shard_bounds(n, r, w) for r in range(w)]
            assert got[0][0] == 0 and got[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            assert max(e - s for s, e in got) - min(e - s for s, e in got) <= 1


def test_two_rank_gather_matches_single(tmp_path):
    from oracle import sigma as OS
    from tests._system import make_small_system
    S = make_small_system()
    qp = np.array([S.nval - 1, S.nval, S.nval + 1], dtype=np.int32)
    out = str(tmp_path / "full.npy")
    mp.start_processes(_worker, args=(2, _free_port(), qp, out), nprocs=2, join=True, start_method="spawn")
    full = np.load(out)
    ref = np.stack([OS.sigma_c_state(S.psi_intp, S.M, S.e1, S.nval, int(m), 21, 2.0, 0.02, 6, S.poly)
                    for m in qp], axis=1)
    assert np.array_equal(full, ref)


def test_two_rank_gather_with_an_empty_shard(tmp_path):
    # one QP state on two ranks: rank 1 holds none and still takes part in
    # the gather with an empty table
    from oracle import sigma as OS
    from tests._system import make_small_system
    S = make_small_system()
    qp = np.array([S.nval], dtype=np.int32)
    out = str(tmp_path / "full.npy")
    mp.start_processes(_worker, args=(2, _free_port(), qp, out), nprocs=2, join=True, start_method="spawn")
    full = np.load(out)
    ref = OS.sigma_c_state(S.psi_intp, S.M, S.e1, S.nval, int(qp[0]), 21, 2.0, 0.02, 6, S.poly)[:, None]
    assert full.shape == (21, 1) and np.array_equal(full, ref)

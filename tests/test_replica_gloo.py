"""The N > 1 plumbing of the band-parallel path on CPU: two gloo ranks on
127.0.0.1.  Each rank applies H*psi (the oracle, on the golden Si8 cell) to
its contiguous slice of bands with no collective; gathering the slices
reproduces the single-process block, the per-rank times reduce to
their maximum on every rank, and the whole-job throughput counts every
rank's units over the slowest rank's time."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from pspw import replica  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    for p in (os.path.join(here, "..", "oracle"), here,
              os.path.join(here, "..", "ffr-pspw-dft-c_b200")):
        sys.path.insert(0, p)
    import datetime

    import pspw_oracle as O
    from helpers import golden, oracle_cell
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        G = golden("si8_8ry")
        cell = oracle_cell(G)
        psi = G["psi"]
        nb = psi.shape[1]
        start, cnt = replica.band_slices(nb, world)[rank]
        mine = O.apply_ham_block(cell, psi[:, start:start + cnt], G["veff"])
        parts = [None] * world
        dist.all_gather_object(parts, (start, mine))
        t_max = replica.max_over_ranks(0.5 + rank)  # per-rank "times"
        replica.barrier()
        if rank == 0:
            full = np.zeros_like(psi)
            for s0, blk in parts:
                full[:, s0:s0 + blk.shape[1]] = blk
            ref = O.apply_ham_block(cell, psi, G["veff"])
            np.savez(os.path.join(out_dir, "result.npz"), full=full, ref=ref,
                     t_max=t_max, world=replica.world_size())
        else:
            np.savez(os.path.join(out_dir, f"rank{rank}.npz"), t_max=t_max)
    finally:
        dist.destroy_process_group()


def test_band_slices_cover_and_balance():
    for nb, world in ((144, 2), (144, 8), (7, 3), (5, 8)):
        sl = replica.band_slices(nb, world)
        assert len(sl) == world
        assert sum(c for _, c in sl) == nb
        assert all(sl[i][0] + sl[i][1] == sl[i + 1][0] for i in range(world - 1))
        assert max(c for _, c in sl) - min(c for _, c in sl) <= 1


def test_weak_throughput():
    assert replica.weak_throughput(10.0, 4, 2.0) == 20.0
    assert replica.max_over_ranks(3.5) == 3.5  # no process group: identity


def test_two_gloo_ranks_band_parallel_hpsi(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    z = np.load(tmp_path / "result.npz")
    assert int(z["world"]) == world
    # bands are independent: the gathered slices are the single-process
    # block (to the last bits that the oracle's batched FFT/BLAS blocking
    # moves)
    d = np.abs(z["full"] - z["ref"]).max() / np.abs(z["ref"]).max()
    assert d < 1e-14
    assert float(z["t_max"]) == 1.5
    assert float(np.load(tmp_path / "rank1.npz")["t_max"]) == 1.5

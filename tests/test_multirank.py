"""Multi-rank path on CPU (gloo, world size 2): each rank renders the same
flux map with its own streams (the oracle stands in for the GPU renderer,
which this CPU test cannot run) and the accumulators are summed on rank 0
with the same reduction bench.py uses over NCCL.  Rank 0 checks the sum
against the two maps recomputed locally, and that the combined estimate is
the same integral as a single-rank render (3 sigma)."""
import math
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _scene():
    from htrdr_kmin_b200 import scene as S
    sc, rq = S.config_c2(scale=8 / 128, spp=64, cloud_def=(8, 8, 4))
    return sc, rq


def _worker(rank, world, port, out_path):
    import torch
    import torch.distributed as dist
    from htrdr_kmin_b200 import multigpu as M
    from htrdr_kmin_b200 import scene as S
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc, rq = _scene()
        rq = S.Request(**{**rq.__dict__, "seed": M.rank_seed(rq.seed, rank)})
        buf, _ = O.OracleScene(sc, 0b100).draw_map(rq, nthreads=1)
        t = torch.from_numpy(np.frombuffer(buf.tobytes(), dtype=np.uint8).copy())
        M.reduce_flux_map(t, dist, dst=0)
        if rank == 0:
            np.save(out_path, t.numpy())
    finally:
        dist.destroy_process_group()


def test_two_rank_flux_reduction(tmp_path):
    import torch.multiprocessing as mp
    from htrdr_kmin_b200 import multigpu as M
    from htrdr_kmin_b200 import scene as S
    from oracle import oracle as O
    O.build()
    out = str(tmp_path / "reduced.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    sc, rq = _scene()
    os_ = O.OracleScene(sc, 0b100)
    maps = []
    for rank in range(2):
        b, _ = os_.draw_map(S.Request(**{**rq.__dict__, "seed": M.rank_seed(rq.seed, rank)}), nthreads=1)
        maps.append(b)
    expect = M.combine_flux_maps(maps)
    got = np.frombuffer(np.load(out).tobytes(), dtype=O.PIXEL_FLUX).reshape(expect.shape)
    np.testing.assert_array_equal(got["n"], expect["n"])
    np.testing.assert_allclose(got["sum"], expect["sum"], rtol=1e-12)
    np.testing.assert_allclose(got["sum2"], expect["sum2"], rtol=1e-12)
    assert np.all(got["n"] == 2 * rq.spp)
    # the combination estimates the same flux as one rank with twice the spp
    single, _ = os_.draw_map(S.Request(**{**rq.__dict__, "spp": 2 * rq.spp, "seed": 999}), nthreads=1)
    E1, S1 = M.flux_estimate(got)
    E2, S2 = M.flux_estimate(single)
    z = (E1 - E2) / np.sqrt(S1 ** 2 + S2 ** 2 + 1e-300)
    assert np.mean(np.abs(z) > 3) <= 0.05
    assert abs(z.mean()) < 5 / math.sqrt(z.size) + 0.1


def test_rank_seeds_are_distinct():
    from htrdr_kmin_b200 import multigpu as M
    seeds = {M.rank_seed(2, r) for r in range(4096)}
    assert len(seeds) == 4096 and M.rank_seed(2, 0) == 2
    assert all(0 <= s < (1 << 32) for s in seeds)

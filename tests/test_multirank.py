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


def _image_cases():
    from htrdr_kmin_b200 import scene as S
    sc, rq = S.config_c2(scale=6 / 128, spp=128, cloud_def=(8, 8, 4))
    rq.mode = S.MODE_XWAVE_LW
    rq.cam_pos, rq.cam_tgt, rq.cam_up = (400, 400, 10), (450, 450, 1500), (0, 1, 0)
    out = [("xwave_lw", sc, rq, 0b100, 1)]
    sc, rq = S.config_c3(scale=6 / 512, spp=8, cloud_def=(16, 16, 4), nbands=4, nquad=2)
    out.append(("image_cie", sc, rq, 0b111, 3))
    return out


def _accum_worker(rank, world, port, out_path, case):
    import torch
    import torch.distributed as dist
    from htrdr_kmin_b200 import multigpu as M
    from htrdr_kmin_b200 import scene as S
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        name, sc, rq, props, nch = [c for c in _image_cases() if c[0] == case][0]
        rq = S.Request(**{**rq.__dict__, "seed": M.rank_seed(rq.seed, rank)})
        w = O.OracleScene(sc, props).realisation_weights(rq, 0, rq.width * rq.height, nthreads=1)
        acc = M.accumulators_from_weights(w, rq.spp, nch)
        t = torch.from_numpy(np.frombuffer(acc.tobytes(), dtype=np.uint8).copy())
        M.reduce_accumulators(t, dist, dst=0)
        if rank == 0:
            np.save(out_path, t.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["xwave_lw", "image_cie"])
def test_two_rank_image_accumulators(tmp_path, case):
    """Images (radiance and CIE XYZ) combine like flux maps: each rank's FP64
    accumulators, summed on rank 0, hold both ranks' realisations and estimate
    the same pixels as one rank with twice the realisations."""
    import torch.multiprocessing as mp
    from htrdr_kmin_b200 import multigpu as M
    from htrdr_kmin_b200 import scene as S
    from oracle import oracle as O
    O.build()
    out = str(tmp_path / "acc.npy")
    mp.start_processes(_accum_worker, args=(2, _free_port(), out, case), nprocs=2, start_method="spawn")
    name, sc, rq, props, nch = [c for c in _image_cases() if c[0] == case][0]
    os_ = O.OracleScene(sc, props)
    npix = rq.width * rq.height
    per_rank = [M.accumulators_from_weights(
        os_.realisation_weights(S.Request(**{**rq.__dict__, "seed": M.rank_seed(rq.seed, r)}), 0, npix,
                                nthreads=1), rq.spp, nch) for r in range(2)]
    expect = M.combine_accumulators(per_rank)
    got = np.frombuffer(np.load(out).tobytes(), dtype=M.ACCUM_DTYPE)
    np.testing.assert_array_equal(got["n"], expect["n"])
    np.testing.assert_allclose(got["s"], expect["s"], rtol=1e-12)
    np.testing.assert_allclose(got["s2"], expect["s2"], rtol=1e-12)
    assert np.all(got["n"][:npix * nch] == 2 * rq.spp)
    # one rank, twice the realisations, other streams: the same estimates within 3 sigma
    single, _ = os_.draw_map(S.Request(**{**rq.__dict__, "spp": 2 * rq.spp, "seed": 999}), nthreads=1)
    E1, S1 = M.estimate(got[:npix * nch])
    if nch == 1:
        E2, S2 = single["L"].ravel(), single["L_se"].ravel()
    else:
        E2 = np.stack([single[c].ravel() for c in ("X", "Y", "Z")], axis=1).ravel()
        S2 = np.stack([single[c + "_se"].ravel() for c in ("X", "Y", "Z")], axis=1).ravel()
    m = (S1 > 0) | (S2 > 0)
    z = (E1[m] - E2[m]) / np.sqrt(S1[m] ** 2 + S2[m] ** 2)
    n = z.size
    assert n > 0
    # heavy-tailed weights at small samples: 3x the Gaussian 0.27 % plus binomial noise
    assert np.mean(np.abs(z) > 3) <= 3 * 0.0027 + 3 * math.sqrt(0.0027 / n) + 1.0 / n
    assert abs(z.mean()) < 5 / math.sqrt(n) + 0.1

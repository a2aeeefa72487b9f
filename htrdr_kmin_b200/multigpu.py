"""Multi-GPU plumbing: one process per GPU, weak scaling.

Realisations are independent, so every rank renders the whole workload with
its own random streams (the request seed is moved by the rank) and the only
exchange is a sum, on one rank, of the maps' FP64 accumulators -- the
combination htrdr does over MPI when its ranks render different tiles
(src/core/htrdr_draw_map.c:186-268), here over NCCL (or gloo on CPU) -- after
which that rank finalizes every map once (estimates, standard errors,
brightness temperatures).

An accumulator record (htrdr_accum, src/core/htrdr_accum.h:31-36) is 32 bytes:
{sum f64, sum of squares f64, count u64, failures u64}.  A map's accumulators
(htrdr_gpu_draw_map_accum_device) are one record per pixel and channel, then
one per pixel for the time per realisation; a flux pixel
(atmosphere_pixel_flux, src/atmosphere/htrdr_atmosphere_c.h:59-62) is two
records.  Floating and integer words are reduced separately, in their own
types.
"""
from __future__ import annotations

import numpy as np

ACCUM_DTYPE = np.dtype([("s", "<f8"), ("s2", "<f8"), ("n", "<u8"), ("nfail", "<u8")])

# Odd 32-bit multiplier (the golden-ratio Weyl increment): rank -> rank * K
# is a bijection modulo 2^32, so the ranks of one job never share a seed.
_RANK_STRIDE = 0x9E3779B9


def rank_seed(seed: int, rank: int) -> int:
    """Seed of a rank's random streams.  Rank 0 keeps the request's seed
    (the single-GPU streams); rank r adds r times an odd constant modulo 2^32,
    so two ranks of one job never draw the same streams for a request."""
    if not 0 <= rank < (1 << 32):
        raise ValueError(f"rank {rank} out of range")
    return (seed + rank * _RANK_STRIDE) & 0xFFFFFFFF


def reduce_accumulators(buf, dist, dst: int = 0) -> None:
    """Sum the accumulator records held in `buf' (a uint8 torch tensor whose
    size is a multiple of 32 bytes) over all ranks into rank `dst'.  Works
    with NCCL (CUDA tensors) and gloo (CPU tensors).  Every rank must call it
    with a buffer of the same size."""
    import torch
    if buf.numel() % 32:
        raise ValueError("accumulator buffers hold 32-byte records")
    n = buf.numel() // 32
    f = buf.view(torch.float64).view(n, 4)[:, :2].contiguous()
    u = buf.view(torch.int64).view(n, 4)[:, 2:].contiguous()
    dist.reduce(f, dst=dst, op=dist.ReduceOp.SUM)
    dist.reduce(u, dst=dst, op=dist.ReduceOp.SUM)
    if dist.get_rank() == dst:
        buf.view(torch.float64).view(n, 4)[:, :2] = f
        buf.view(torch.int64).view(n, 4)[:, 2:] = u


def reduce_flux_map(buf, dist, dst: int = 0) -> None:
    """Sum flux maps (height x width atmosphere_pixel_flux structs, two
    accumulator records each) over all ranks into rank `dst'."""
    reduce_accumulators(buf, dist, dst)


def combine_accumulators(maps) -> np.ndarray:
    """Host-side reference of the reduction: record-wise sum of accumulator
    arrays (ACCUM_DTYPE, or any structured array of the same 32-byte
    records)."""
    out = np.array(maps[0], copy=True).view(ACCUM_DTYPE)
    for m in maps[1:]:
        v = np.asarray(m).view(ACCUM_DTYPE)
        for k in ("s", "s2", "n", "nfail"):
            out[k] = out[k] + v[k]
    return out.view(np.asarray(maps[0]).dtype)


def combine_flux_maps(maps) -> np.ndarray:
    return combine_accumulators(maps)


def accumulators_from_weights(weights: np.ndarray, spp: int, nch: int) -> np.ndarray:
    """The accumulator records of a map from its realisation weights
    ([npix, nch * spp], channel-major inside a pixel, NaN: rejected sample),
    channels of all pixels first, then a zeroed time record per pixel."""
    npix = weights.shape[0]
    acc = np.zeros(npix * (nch + 1), dtype=ACCUM_DTYPE)
    for ch in range(nch):
        w = weights[:, ch * spp:(ch + 1) * spp]
        ok = ~np.isnan(w)
        wz = np.where(ok, w, 0.0)
        # record (pixel, channel) at index pixel * nch + channel
        acc["s"][ch::nch][:npix] = wz.sum(axis=1)
        acc["s2"][ch::nch][:npix] = (wz * wz).sum(axis=1)
        acc["n"][ch::nch][:npix] = ok.sum(axis=1)
    return acc


def estimate(acc: np.ndarray):
    """htrdr_accum_get_estimation (src/core/htrdr_accum.h:48-68) per record:
    (E, SE)."""
    a = np.asarray(acc).view(ACCUM_DTYPE)
    n = a["n"].astype(np.float64)
    N = np.maximum(n, 1)
    E = np.where(n > 0, a["s"] / N, 0.0)
    V = np.maximum(a["s2"] / N - E * E, 0)
    return E, np.where(n > 0, np.sqrt(V / N), 0.0)


def flux_estimate(buf: np.ndarray):
    """Per-probe estimate and standard error of a flux map."""
    n = np.maximum(buf["n"].astype(np.float64), 1)
    E = buf["sum"] / n
    V = np.maximum(buf["sum2"] / n - E * E, 0)
    return E, np.sqrt(V / n)

"""Multi-GPU plumbing: one process per GPU, weak scaling.

Realisations are independent, so every rank renders the whole map with its
own random streams (the request seed is offset by the rank) and the only
exchange is a sum of the flux maps' per-probe accumulators on rank 0, the
combination htrdr does over MPI when ranks render different tiles
(src/core/htrdr_draw_map.c:186-268), here over NCCL (or gloo on CPU).

A flux pixel (atmosphere_pixel_flux, src/atmosphere/htrdr_atmosphere_c.h:59-62)
is 8 words: {sum, sum2} f64, {n, nfail} u64 for the flux, then the same for the
per-realisation time.  Floating and integer words are reduced separately, in
their own types.
"""
from __future__ import annotations

import numpy as np

F64_WORDS = [0, 1, 4, 5]
U64_WORDS = [2, 3, 6, 7]


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


def reduce_flux_map(buf, dist, dst: int = 0) -> None:
    """Sum the flux accumulators of `buf` (a uint8 torch tensor holding
    height x width atmosphere_pixel_flux structs) over all ranks into rank
    `dst`.  Works with NCCL (CUDA tensors) and gloo (CPU tensors)."""
    import torch
    npix = buf.numel() // 64
    f = buf.view(torch.float64).view(npix, 8)[:, F64_WORDS].contiguous()
    u = buf.view(torch.int64).view(npix, 8)[:, U64_WORDS].contiguous()
    dist.reduce(f, dst=dst, op=dist.ReduceOp.SUM)
    dist.reduce(u, dst=dst, op=dist.ReduceOp.SUM)
    if dist.get_rank() == dst:
        buf.view(torch.float64).view(npix, 8)[:, F64_WORDS] = f
        buf.view(torch.int64).view(npix, 8)[:, U64_WORDS] = u


def combine_flux_maps(maps) -> np.ndarray:
    """Host-side reference of the reduction: sum of structured flux buffers."""
    out = maps[0].copy()
    for m in maps[1:]:
        for k in ("sum", "sum2", "n", "nfail", "t_sum", "t_sum2", "t_n", "t_nfail"):
            out[k] = out[k] + m[k]
    return out


def flux_estimate(buf: np.ndarray):
    """Per-probe estimate and standard error (htrdr_accum_get_estimation)."""
    n = np.maximum(buf["n"].astype(np.float64), 1)
    E = buf["sum"] / n
    V = np.maximum(buf["sum2"] / n - E * E, 0)
    return E, np.sqrt(V / n)

"""Particle sharding across ranks (one process per GPU).

The path shards without a data-path collective: particles are independent and the
medium is read-only.  Every rank runs a contiguous block of global particle ids and
passes the block's first id as `particle_offset`, so each particle draws the same
counter-based noise whatever the sharding.  Observables are reduced once at the end
as FP64 sums (one small all-reduce).
"""
from __future__ import annotations

import numpy as np

OBS = 12


def shard(n_total: int, rank: int, world: int) -> tuple[int, int]:
    """(first global id, count) of rank's block: sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(int(n_total), int(world))
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


def observable_sums(p, x, m, cut=5.0, width=0.1) -> np.ndarray:
    """FP64 sums of the engine's observables (LIM_OBS_* order) for (rows, N) arrays."""
    p = np.asarray(p, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros(OBS)
    if p.shape[1] == 0:
        return out
    px = p[0]
    py = p[1] if p.shape[0] >= 2 else np.zeros_like(px)
    pt2 = px * px + py * py
    pt = np.sqrt(pt2)
    p2 = np.sum(p * p, axis=0)
    E = np.sqrt(m * m + p2)
    w = m / E
    with np.errstate(invalid="ignore", divide="ignore"):
        c2 = np.where(pt2 > 0, (px * px - py * py) / pt2, 0.0)
    out[0] = p.shape[1]
    out[1] = pt.sum()
    out[2] = c2.sum()
    out[3] = np.count_nonzero(pt > cut)
    out[4] = np.sum(1.0 / (1.0 + np.exp(-(pt - cut) / width)))
    out[5] = p2.sum()
    out[6] = E.sum()
    out[7] = np.sum(w * p2)
    out[8] = px.sum()
    out[9] = np.sum(w * px)
    out[10] = np.sum(p[2] ** 2) if p.shape[0] == 3 else 0.0
    out[11] = np.sum(np.sum(x * x, axis=0))
    return out

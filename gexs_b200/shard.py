"""Splitting one cross-section, or a set of jobs, over ranks (one GPU each).

The path shards with no data-path collective: a bin's value depends only on
the lines within the cutoff of it, so disjoint bin ranges are computed
independently (each rank reads the line sub-list its range needs) and the
full grid is the concatenation of the slices.  Jobs ((T, P) pairs) shard
round-robin.  The multi-GPU manager of the reference instead gives whole
line chunks to GPUs and sums full-size grids on the host
(Managers/Accel/GPU/MultiGPUManager.cpp:104-126).
"""
import numpy as np


def equal_slices(grid_points, world):
    """[start_idx, n_points) per rank, equal bin counts."""
    cuts = [grid_points * r // world for r in range(world + 1)]
    return [(cuts[r], cuts[r + 1] - cuts[r]) for r in range(world)]


def balanced_slices(nu_sorted, nu_start, dnu, grid_points, cutoff, world, sample=256):
    """[start_idx, n_points) per rank with equal numbers of (line, bin)
    evaluations: the work of bin j is the number of lines within the cutoff
    of it, estimated on every `sample`-th bin from the sorted centres."""
    nu = np.asarray(nu_sorted)
    js = np.arange(0, grid_points, sample, dtype=np.int64)
    f = nu_start + js * dnu
    w = (np.searchsorted(nu, f + cutoff, side="right") -
         np.searchsorted(nu, f - cutoff, side="left")).astype(np.float64) + 1e-9
    cum = np.concatenate([[0.0], np.cumsum(w)])
    tot = cum[-1]
    bounds = [0]
    for r in range(1, world):
        k = int(np.searchsorted(cum, tot * r / world))
        bounds.append(min(grid_points, max(bounds[-1], k * sample)))
    bounds.append(grid_points)
    return [(bounds[r], bounds[r + 1] - bounds[r]) for r in range(world)]


def line_range(nu_sorted, nu_start, dnu, start_idx, n_points, cutoff):
    """Indices [lo, hi) of the lines a bin range can reach (for ranks that
    hold only their own part of the list)."""
    nu = np.asarray(nu_sorted)
    f0 = nu_start + start_idx * dnu
    f1 = nu_start + (start_idx + max(n_points, 1) - 1) * dnu
    margin = 2.0 * dnu + 1e-9 * (abs(f1) + cutoff)
    lo = int(np.searchsorted(nu, f0 - cutoff - margin, side="left"))
    hi = int(np.searchsorted(nu, f1 + cutoff + margin, side="right"))
    return lo, hi


def plan(nu_sorted, nu_start, dnu, start_idx, n_points, reach, nshards, align=4096):
    """gexs_shard_plan (host code of the library): bin cuts (nshards + 1)
    with about equal evaluations on multiples of `align` from start_idx,
    and each shard's line index range [lo, hi) within `reach`."""
    import ctypes as C
    from . import _capi as capi
    nu = np.ascontiguousarray(nu_sorted, dtype=np.float64)
    b = np.zeros(nshards + 1, dtype=np.int64)
    lo = np.zeros(nshards, dtype=np.int64)
    hi = np.zeros(nshards, dtype=np.int64)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    capi.check(capi.lib().gexs_shard_plan(p(nu), len(nu), nu_start, dnu, start_idx, n_points,
                                          reach, align, nshards, p(b), p(lo), p(hi)),
               "gexs_shard_plan")
    return b, lo, hi


def round_robin(jobs, rank, world):
    """The jobs of one rank when (T, P) pairs are spread over ranks."""
    return [j for i, j in enumerate(jobs) if i % world == rank]


def max_over_ranks(dist, value, device=None):
    """All-reduce MAX of a per-rank time (the job ends with its slowest
    rank)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, value, device=None):
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())

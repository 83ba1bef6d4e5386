"""Multi-rank logic on CPU with the gloo backend (world size 2): grid
slices cover the grid exactly once, the slices computed independently (here
with the FP64 oracle, one rank each, each holding only the lines that
gexs_shard_plan gives its bins) concatenate to the single-process result
bit for bit, and the timing reduction takes the slowest rank.  The plan
itself (the library's host code behind B200MultiManager) is checked for
coverage, alignment, line ranges and balance."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gexs_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_slices_partition_the_grid():
    nu = np.sort(np.random.default_rng(1).exponential(4000.0, 200000) + 100.0)
    for world in (1, 2, 3, 8):
        for sl in (shard.equal_slices(999_999, world),
                   shard.balanced_slices(nu, 100.0, 0.01, 999_999, 25.0, world)):
            assert sl[0][0] == 0
            assert sum(n for _, n in sl) == 999_999
            for (a, n), (b, _) in zip(sl[:-1], sl[1:]):
                assert a + n == b


def test_balanced_slices_even_out_work():
    nu = np.sort(np.random.default_rng(2).exponential(4000.0, 400000) + 100.0)
    G, dnu, cut = 2_990_001, 0.01, 25.0
    sl = shard.balanced_slices(nu, 100.0, dnu, G, cut, 4)
    work = []
    for a, n in sl:
        f = 100.0 + np.arange(a, a + n, 97) * dnu
        work.append(np.sum(np.searchsorted(nu, f + cut) - np.searchsorted(nu, f - cut)))
    work = np.array(work, dtype=float)
    assert work.max() / work.min() < 1.2
    eq = shard.equal_slices(G, 4)
    assert eq[0][1] > 3 * sl[0][1]          # the dense low-nu end gets fewer bins


def test_plan_cuts_align_cover_and_balance():
    nu = np.sort(np.random.default_rng(3).exponential(4000.0, 400000) + 100.0)
    G, dnu, cut = 2_990_001, 0.01, 25.0
    for world, start, n in ((1, 0, G), (2, 0, G), (4, 12345, G - 20000), (8, 0, G), (3, 7, 5000)):
        b, lo, hi = shard.plan(nu, 100.0, dnu, start, n, cut, world)
        assert b[0] == start and b[-1] == start + n and np.all(np.diff(b) >= 0)
        assert np.all((b[1:-1] - start) % 4096 == 0)
        for r in range(world):
            if b[r + 1] == b[r]:
                continue
            fa, fb = 100.0 + b[r] * dnu, 100.0 + (b[r + 1] - 1) * dnu
            need = np.nonzero((nu >= fa - cut) & (nu <= fb + cut))[0]
            if need.size:
                assert lo[r] <= need[0] and hi[r] > need[-1]
    b, _, _ = shard.plan(nu, 100.0, dnu, 0, G, cut, 4)
    work = []
    for r in range(4):
        f = 100.0 + np.arange(b[r], b[r + 1], 97) * dnu
        work.append(np.sum(np.searchsorted(nu, f + cut) - np.searchsorted(nu, f - cut)))
    work = np.array(work, dtype=float)
    assert work.max() / work.min() < 1.25
    b, lo, hi = shard.plan(nu[:0], 100.0, dnu, 0, 1000, cut, 2)
    assert b[0] == 0 and b[-1] == 1000 and np.all(lo == 0) and np.all(hi == 0)


def _worker(rank, world, port, lines, q):
    import torch.distributed as dist
    from gexs_b200 import _capi as capi
    from gexs_b200.engine import job_init
    from tests.helpers import host_job
    from oracle import pyoracle as po
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    G, nu0, dnu = 60000, 100.0, 0.05
    b, los, his = shard.plan(lines["nu"], nu0, dnu, 0, G, 25.0 + 1.0, world)
    a, n = int(b[rank]), int(b[rank + 1] - b[rank])
    lo, hi = int(los[rank]), int(his[rank])
    part = {k: np.ascontiguousarray(v[lo:hi]) for k, v in lines.items()}
    j = job_init(capi.CONV_PHYSICAL, capi.VOIGT, 1500.0, 1.0, 3000.0, 18.0, nu0, dnu, G,
                 cutoff=25.0)
    j.start_idx, j.n_points = a, n
    out = po.cross_section(host_job(j, part), nthreads=1)
    slices = [None] * world
    dist.all_gather_object(slices, (a, n, out[a:a + n].copy()))
    tmax = shard.max_over_ranks(dist, 10.0 + rank)
    tot = shard.sum_over_ranks(dist, 1.0)
    if rank == 0:
        q.put((slices, tmax, tot))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_grid_sharding_matches_single_process(small_lines):
    from gexs_b200 import _capi as capi
    from gexs_b200.engine import job_init
    from tests.helpers import host_job
    from oracle import pyoracle as po
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, small_lines, q)) for r in range(2)]
    for p in procs:
        p.start()
    slices, tmax, tot = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    G, nu0, dnu = 60000, 100.0, 0.05
    j = job_init(capi.CONV_PHYSICAL, capi.VOIGT, 1500.0, 1.0, 3000.0, 18.0, nu0, dnu, G,
                 cutoff=25.0)
    full = po.cross_section(host_job(j, small_lines), nthreads=1)
    got = np.concatenate([s[2] for s in sorted(slices, key=lambda s: s[0])])
    np.testing.assert_array_equal(got, full)
    assert tmax == 11.0 and tot == 2.0

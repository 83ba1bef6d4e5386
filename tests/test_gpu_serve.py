"""Request loop: admission by HBM budget, continuous batching, results
identical alone and in a mix, failures reported per request."""
import threading
import time

import numpy as np
import pytest

from gexs_b200 import _capi as capi
from gexs_b200.engine import Server, job_init
from tests import helpers as H

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served(small_states, small_lines):
    srv = Server(0, hbm_budget=1 << 30, streams=4)
    lid = srv.add_list(small_lines, small_states.energy, small_states.g, 18.0)
    dop = {k: v for k, v in small_lines.items() if k not in ("gamma", "n")}
    lid_dop = srv.add_list(dop, small_states.energy, small_states.g, 28.0)
    yield srv, lid, lid_dop
    srv.close()


def _requests(lid, lid_dop, n=10, seed=5):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n):
        T = float(10 ** rng.uniform(2.0, np.log10(3000.0)))
        P = float(10 ** rng.uniform(-6.0, 2.0))
        d = float(10 ** rng.uniform(-2.5, -1.0))
        nu0 = float(rng.uniform(100.0, 3000.0))
        G = int(rng.integers(2000, 60000))
        voigt = i % 2 == 0
        out.append(Server.request(lid if voigt else lid_dop,
                                  capi.VOIGT if voigt else capi.DOPPLER, T, P, nu0, d, G,
                                  precision=capi.FP32 if i % 3 else capi.FP64, cutoff=25.0))
    return out


def test_alone_equals_mixed(served):
    srv, lid, lid_dop = served
    reqs = _requests(lid, lid_dop)
    alone = []
    for r in reqs:
        t = srv.submit(r)
        alone.append(srv.wait(t, r.grid_points)[0])
    tickets = [srv.submit(r) for r in reqs]
    mixed, sizes = [], []
    for r, t in zip(reqs, tickets):
        out, info = srv.wait(t, r.grid_points)
        mixed.append(out)
        sizes.append(info.batch_size)
    for a, b in zip(alone, mixed):
        np.testing.assert_array_equal(a, b)
    assert max(sizes) > 1, "requests submitted together were never batched"


def test_concurrent_waiters_of_one_batch(served):
    """Many threads fetch the requests of the same batches at once, in an
    order unrelated to submission: each gets its own result (equal to the
    request run alone) and the batch's completion event outlives every
    waiter that still uses it."""
    srv, lid, lid_dop = served
    reqs = _requests(lid, lid_dop, n=48, seed=11)
    alone = [srv.wait(srv.submit(r), r.grid_points)[0] for r in reqs]
    for _ in range(3):
        tickets = [srv.submit(r) for r in reqs]
        got = [None] * len(reqs)
        errors = []

        def fetch(idx):
            try:
                for i in idx:
                    got[i] = srv.wait(tickets[i], reqs[i].grid_points)[0]
            except Exception as e:  # pragma: no cover
                errors.append(e)
        order = np.random.Generator(np.random.PCG64(7)).permutation(len(reqs))
        threads = [threading.Thread(target=fetch, args=(order[k::12],)) for k in range(12)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        assert not errors, errors[0]
        for a, b in zip(alone, got):
            np.testing.assert_array_equal(a, b)


def test_served_results_match_oracle(served, small_states, small_lines):
    from oracle import pyoracle as po
    srv, lid, lid_dop = served
    for prof, prec, L, l_id, mass in ((capi.VOIGT, capi.FP64, small_lines, lid, 18.0),
                                      (capi.DOPPLER, capi.FP64, small_lines, lid_dop, 28.0),
                                      (capi.VOIGT, capi.FP32, small_lines, lid, 18.0)):
        T, P, nu0, d, G = 900.0, 0.3, 500.0, 0.02, 50000
        r = Server.request(l_id, prof, T, P, nu0, d, G, precision=prec, cutoff=25.0)
        out, info = srv.wait(srv.submit(r), G)
        q = po.partition(small_states.energy, small_states.g, T)
        j = job_init(capi.CONV_PHYSICAL, prof, T, P, q, mass, nu0, d, G, cutoff=25.0)
        Lh = L if prof == capi.VOIGT else {k: v for k, v in L.items() if k not in ("gamma", "n")}
        ref = H.oracle_of(j, Lh)
        if prec == capi.FP64:
            # Q(T) comes from the device's tree reduction: 1e-12 relative
            floor = 1e-290 if prof == capi.DOPPLER else 0.0
            d_ = np.abs(out - ref)
            assert np.all(d_ <= 1e-10 * np.abs(ref) + floor)
        else:
            rel, band = H.fp32_errors(out, ref)
            assert rel <= H.FP32_REL and band <= H.FP32_BAND


def test_compact_resident_list(small_states, small_lines):
    """A list kept resident in the 24-byte compact layout: served results
    equal gexs_run on the same compact list bit for bit, and the oracle on
    the widened values within the stated tolerances."""
    from oracle import pyoracle as po
    from gexs_b200.engine import Context, Job, LineList
    import torch
    srv = Server(0, hbm_budget=1 << 30, streams=2)
    try:
        lid = srv.add_list(small_lines, small_states.energy, small_states.g, 18.0, compact=True)
        ll = LineList(small_lines["nu"], small_lines["elow"], small_lines["aif"],
                      small_lines["gns"], small_lines["gamma"], small_lines["n"], compact=True)
        wide = ll.widened()
        ctx = Context(0)
        T, P, nu0, d, G = 900.0, 0.3, 500.0, 0.02, 50000
        for prec in (capi.FP32, capi.FP64):
            r = Server.request(lid, capi.VOIGT, T, P, nu0, d, G, precision=prec, cutoff=25.0)
            out, _ = srv.wait(srv.submit(r), G)
            q, _ = srv.partition(lid, T)
            direct = torch.zeros(G, dtype=torch.float64, device="cuda")
            j = Job(ll, direct, convention=capi.CONV_PHYSICAL, profile=capi.VOIGT, temperature=T,
                    pressure=P, partition=q, mass=18.0, nu_start=nu0, dnu=d, grid_points=G,
                    precision=prec, cutoff=25.0)
            ctx.run([j])
            ctx.check()
            np.testing.assert_array_equal(out, direct.cpu().numpy())
            jo = job_init(capi.CONV_PHYSICAL, capi.VOIGT, T, P,
                          po.partition(small_states.energy, small_states.g, T), 18.0, nu0, d, G,
                          cutoff=25.0)
            ref = H.oracle_of(jo, wide)
            if prec == capi.FP64:
                assert np.all(np.abs(out - ref) <= 1e-10 * np.abs(ref))
            else:
                rel, band = H.fp32_errors(out, ref)
                assert rel <= H.FP32_REL and band <= H.FP32_BAND
    finally:
        srv.close()


def test_out_of_memory_requeue_and_failure(small_states):
    """Host-side fault injection (gexs_debug_fail_allocs refuses the next
    allocation without calling CUDA): with nothing else running, the request
    fails with GEXS_ERR_OOM and the server keeps serving; while another
    batch runs, the group goes back to the queue and completes after that
    batch with the same result as alone."""
    from gexs_b200 import synth
    from gexs_b200._capi import lib
    L = synth.make_lines(small_states, 400000, 100.0, 4000.0, 2101, broadening_seed=3101)
    srv = Server(0, hbm_budget=8 << 30, streams=2)
    try:
        lid = srv.add_list(L, small_states.energy, small_states.g, 18.0)
        small = Server.request(lid, capi.VOIGT, 700.0, 0.5, 1000.0, 0.02, 20000,
                               precision=capi.FP32, cutoff=25.0)
        alone = srv.wait(srv.submit(small), 20000)[0]
        assert lib().gexs_debug_fail_allocs(1) == 0
        assert srv.wait_status(srv.submit(small), -1) == capi.GEXS_ERR_OOM
        np.testing.assert_array_equal(srv.wait(srv.submit(small), 20000)[0], alone)
        # a slow FP64 Gauss-Hermite batch holds the device meanwhile
        big = Server.request(lid, capi.VOIGT_QUAD, 700.0, 0.5, 100.0, 0.01, 390001,
                             precision=capi.FP64, cutoff=25.0, quad_nodes=32)
        b0 = srv.stats()["batches"]
        tb = srv.submit(big)
        deadline = time.time() + 60
        while srv.stats()["batches"] == b0 and time.time() < deadline:
            time.sleep(0.0005)
        assert lib().gexs_debug_fail_allocs(1) == 0
        ts = srv.submit(small)
        out, _ = srv.wait(ts, 20000)
        assert srv.poll(tb) in (capi.GEXS_OK, capi.GEXS_ERR_NOT_READY)
        srv.wait(tb, 390001)
        np.testing.assert_array_equal(out, alone)
    finally:
        lib().gexs_debug_fail_allocs(0)
        srv.close()


def test_admission_by_budget(small_states, small_lines):
    line_bytes = sum(v.nbytes for v in small_lines.values()) + small_states.energy.nbytes * 2
    G = 200000
    # room for about three outputs; a request is also charged the scratch of
    # its launch (prep arrays, tables, slice rows), so two run at a time
    budget = line_bytes + 3 * G * 8 + 4096
    srv = Server(0, hbm_budget=budget, streams=2)
    try:
        lid = srv.add_list(small_lines, small_states.energy, small_states.g, 18.0)
        too_big = Server.request(lid, capi.VOIGT, 1000.0, 1.0, 100.0, 0.01, 10 * G)
        st, _ = srv.try_submit(too_big)
        assert st == capi.GEXS_ERR_ADMISSION
        reqs = [Server.request(lid, capi.VOIGT, 300.0 + 100 * i, 1.0, 100.0 + 50 * i, 0.02, G)
                for i in range(8)]
        tickets = [srv.submit(r) for r in reqs]
        peak = [0]
        done = threading.Event()

        def watch():
            while not done.is_set():
                peak[0] = max(peak[0], srv.stats()["inflight_bytes"])
        th = threading.Thread(target=watch)
        th.start()
        outs = [srv.wait(t, G)[0] for t in tickets]
        done.set()
        th.join()
        assert peak[0] <= 3 * G * 8
        assert all(np.max(o) > 0 for o in outs)
        st = srv.stats()
        assert st["submitted"] == st["completed"] == 8
    finally:
        srv.close()


def test_wait_timeout_and_bad_requests(served):
    srv, lid, lid_dop = served
    r = Server.request(lid, capi.VOIGT, 1500.0, 1.0, 100.0, 0.001, 3000000)
    t = srv.submit(r)
    st = srv.wait_status(t, 0)
    assert st in (capi.GEXS_ERR_TIMEOUT, 0)
    if st == capi.GEXS_ERR_TIMEOUT:
        srv.wait(t, r.grid_points)
    bad = Server.request(99, capi.VOIGT, 1500.0, 1.0, 100.0, 0.01, 1000)
    assert srv.try_submit(bad)[0] == capi.GEXS_ERR_INVALID
    no_broadening = Server.request(lid_dop, capi.VOIGT, 1500.0, 1.0, 100.0, 0.01, 1000)
    assert srv.try_submit(no_broadening)[0] == capi.GEXS_ERR_INVALID


def test_resident_partition_table(served, small_states):
    """Q(T) from the list's resident table (4096 temperatures over 10-10000 K,
    4-point Lagrange in ln Q / ln T) within 1e-12 of the oracle's exact sum;
    temperatures outside the table take the exact device sum."""
    from oracle import pyoracle as po
    srv, lid, _ = served
    rng = np.random.Generator(np.random.PCG64(17))
    for T in list(10 ** rng.uniform(1.2, 3.95, 40)) + [10.0, 10000.0, 296.0]:
        q, tab = srv.partition(lid, float(T))
        want = po.partition(small_states.energy, small_states.g, float(T))
        assert tab
        assert abs(q - want) <= 1e-12 * want, (T, q, want)
    for T in (5.0, 20000.0):
        q, tab = srv.partition(lid, T)
        want = po.partition(small_states.energy, small_states.g, T)
        assert not tab and abs(q - want) <= 1e-13 * want

"""B200ExomolReader, the StateReader drop-in (gexs_b200/host), through its C
view (include/gexs_reader.h): the records it streams equal those of the
reference's own ExomolStateReader compiled from its sources
(oracle/_ref/gexsref_reader), in file order; Q(T) from its device states
matches the oracle; its device lines feed the compute path directly."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from gexs_b200 import Job, LineList, synth, _capi as capi
from gexs_b200._capi import check, lib
from oracle import pyoracle as po
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _files(tmp_path, seed=91, broad=True):
    st = synth.make_states(2500, 40, seed)
    u, l, a = synth.make_exomol_transitions(st, 8000, 30.0, 7000.0, seed + 1)
    names = {"states": synth.exomol_states_text(st), "trans": synth.exomol_trans_text(u, l, a)}
    if broad:
        names["broad"] = synth.exomol_broad_text(40, seed + 2, a1_pairs=10)
    paths = {}
    for k, data in names.items():
        p = os.path.join(str(tmp_path), "r." + k)
        with open(p, "wb") as f:
            f.write(data)
        paths[k] = p
    return st, paths


def _stream(r):
    vals = [C.c_double() for _ in range(6)]
    more = C.c_int()
    rows = []
    while True:
        check(lib().gexs_reader_next(r, *[C.byref(v) for v in vals], C.byref(more)),
              "gexs_reader_next")
        if not more.value:
            break
        rows.append([v.value for v in vals])
    return np.array(rows).reshape(-1, 6)


def test_reader_streams_what_the_reference_reads(tmp_path):
    st, p = _files(tmp_path)
    r = C.c_void_p()
    check(lib().gexs_reader_create(p["states"].encode(), p["broad"].encode(), 0.07, 0.5, 0,
                                   capi.BROAD_DEFAULTS, 0, C.byref(r)), "gexs_reader_create")
    try:
        n = C.c_int64()
        check(lib().gexs_reader_open(r, p["trans"].encode(), C.byref(n)), "gexs_reader_open")
        got = _stream(r)
        assert got.shape[0] == n.value > 0
        if po.ref_reader_available():
            ref = po.ref_exomol_read(p["states"], p["trans"], p["broad"], 0.07, 0.5)
            for col, k in enumerate(("nu", "gns", "elow", "aif", "gamma", "n")):
                assert np.array_equal(got[:, col].view(np.int64), ref[k].view(np.int64)), k
        q = C.c_double()
        e, g, _ = po.exomol_states(open(p["states"], "rb").read())   # energies as in the file
        for T in (300.0, 1500.0, 3000.0):
            check(lib().gexs_reader_partition(r, T, C.byref(q)), "gexs_reader_partition")
            want = po.partition(e, g, T)
            assert abs(q.value - want) <= 1e-13 * want
    finally:
        lib().gexs_reader_destroy(r)


def test_reader_device_lines_to_cross_section(tmp_path):
    st, p = _files(tmp_path, seed=97)
    r = C.c_void_p()
    check(lib().gexs_reader_create(p["states"].encode(), p["broad"].encode(), 0.07, 0.5, 0,
                                   capi.BROAD_BY_J, 1, C.byref(r)), "gexs_reader_create")
    try:
        check(lib().gexs_reader_open(r, p["trans"].encode(), None), "gexs_reader_open")
        dl = capi.GexsLines()
        check(lib().gexs_reader_device_lines(r, C.byref(dl)), "gexs_reader_device_lines")
        q = C.c_double()
        check(lib().gexs_reader_partition(r, 900.0, C.byref(q)), "gexs_reader_partition")
        G = 15000
        out = torch.zeros(G, dtype=torch.float64, device="cuda")
        j = capi.GexsJob()
        check(lib().gexs_job_init(C.byref(j), capi.CONV_PHYSICAL, capi.VOIGT, 900.0, 0.3,
                                  q.value, 18.0, 296.0, 1.0, 0.0, 25.0, 50.0, 0.5, G),
              "gexs_job_init")
        j.lines = dl
        j.out = out.data_ptr()
        j.precision = capi.FP64
        j.start_idx, j.n_points = 0, G
        ctx = C.c_void_p()
        check(lib().gexs_ctx_create(0, C.byref(ctx)), "gexs_ctx_create")
        try:
            check(lib().gexs_run(ctx, C.byref(j), 1, None, None), "gexs_run")
            check(lib().gexs_ctx_check(ctx, None), "gexs_ctx_check")
        finally:
            lib().gexs_ctx_destroy(ctx)
        e, g, jj = po.exomol_states(open(p["states"], "rb").read())
        host = po.exomol_trans(open(p["trans"], "rb").read(), e, g, jj,
                               open(p["broad"], "rb").read(), capi.BROAD_BY_J, 0.07, 0.5,
                               sort_by_nu=True)
        want = po.cross_section(H.host_job(j, host))
        worst, nbad = H.fp64_mismatch(out.cpu().numpy(), want)
        assert nbad == 0, worst
    finally:
        lib().gexs_reader_destroy(r)


def test_reader_reports_missing_files(tmp_path):
    r = C.c_void_p()
    st = lib().gexs_reader_create(os.path.join(str(tmp_path), "none.states").encode(), None, 0.1,
                                  0.1, 0, capi.BROAD_DEFAULTS, 0, C.byref(r))
    assert st == capi.GEXS_ERR_INVALID

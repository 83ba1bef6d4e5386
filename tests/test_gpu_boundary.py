"""The drop-ins driven through the reference's own base-class pointers on
the GPU (oracle/boundary_driver.cpp, compiled on the reference's
Readers/StateReader.h and Managers/BaseManager.h alone; see
tests/test_boundary_abi.py for the layout and link checks).

Both builds - the product library's classes (drive_so) and the drop-in
sources compiled against the reference's headers (drive_src) - stream, through
StateReader*, the records the FP64 oracle parses from the same files (bit
for bit, sorted by nu), give Q(T) within 1e-13 of the oracle, and through
BaseManager* produce two (T, P) cross-sections that match the FP64 oracle
within 1e-10 relative per bin (reference-GPU convention, FP64 form).
"""
import json
import os
import subprocess

import numpy as np
import pytest

from gexs_b200 import synth, _capi as capi
from gexs_b200.engine import job_init
from oracle import pyoracle as po
from tests import helpers as H

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BND = os.path.join(ROOT, "oracle", "_ref", "boundary")


@pytest.mark.parametrize("variant", ["drive_so", "drive_src"])
def test_drop_ins_through_reference_pointers(tmp_path, variant):
    exe = os.path.join(BND, variant)
    if not os.path.exists(exe):
        pytest.fail("%s was not built (oracle/Makefile target boundary)" % exe)
    st = synth.make_states(2000, 30, 71)
    u, l, a = synth.make_exomol_transitions(st, 5000, 40.0, 4000.0, 72)
    sp, tp = os.path.join(str(tmp_path), "b.states"), os.path.join(str(tmp_path), "b.trans")
    open(sp, "wb").write(synth.exomol_states_text(st))
    open(tp, "wb").write(synth.exomol_trans_text(u, l, a))
    T1, P1, T2, P2, mass, nu0, dnu, G = 1500.0, 1.0, 700.0, 0.2, 18.0, 30.0, 0.05, 80000
    p = subprocess.run([exe, sp, tp, str(tmp_path), repr(T1), repr(P1), repr(T2), repr(P2),
                        repr(mass), repr(nu0), repr(dnu), str(G), "0"],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-1000:]
    r = json.loads(p.stdout.strip().splitlines()[-1])
    assert r["opened"] == 1 and r["closed"] == 1 and r["reopened"] == 1 and r["closed2"] == 1
    assert r["got4"] == 1 and r["match4"] == 1 and r["ready"] == 1
    assert r["deprecated_left_buffer"] == 1
    assert r["ntrans_capacity"] >= r["records"] > 0 and r["ntrans_capacity2"] > 0

    e, g, jj = po.exomol_states(open(sp, "rb").read())
    host = po.exomol_trans(open(tp, "rb").read(), e, g, jj, b"", capi.BROAD_DEFAULTS, 0.07, 0.5,
                           sort_by_nu=True)
    rec = np.fromfile(os.path.join(str(tmp_path), "records.bin"), dtype=np.float64).reshape(-1, 6)
    assert rec.shape[0] == r["records"] == len(host["nu"])
    for col, k in enumerate(("nu", "gns", "elow", "aif", "gamma", "n")):
        want = host[k].astype(np.float64)
        assert np.array_equal(rec[:, col].view(np.int64), want.view(np.int64)), k
    for T, key in ((T1, "q1"), (T2, "q2")):
        want = po.partition(e, g, T)
        assert abs(r[key] - want) <= 1e-13 * want

    lines = {"nu": rec[:, 0].copy(), "gns": rec[:, 1].astype(np.int32), "elow": rec[:, 2].copy(),
             "aif": rec[:, 3].copy(), "gamma": rec[:, 4].copy(), "n": rec[:, 5].copy()}
    for T, P, key, name in ((T1, P1, "q1", "sigma0.bin"), (T2, P2, "q2", "sigma1.bin")):
        j = job_init(capi.CONV_REF_GPU, capi.VOIGT, T, P, r[key], mass, nu0, dnu, G,
                     ref_temp=296.0, ref_press=1.0)
        want = po.cross_section(H.host_job(j, lines))
        got = np.fromfile(os.path.join(str(tmp_path), name), dtype=np.float64)
        assert np.max(want) > 0
        worst, nbad = H.fp64_mismatch(got, want)
        assert nbad == 0, "%s: worst %.3g of tolerance" % (name, worst)

"""The multi-GPU manager (gexs_manager_create_multi, B200MultiManager)
through the BaseManager C view, as BaseProfile drives it
(Profiles/BaseProfile.cpp:65-71,100-116,279-281): two line chunks, two
(T, P) pairs per chunk, results added into a pre-zeroed host grid.

Every run here has one GPU, so the shards are several entries of device 0
(each its own manager, context and streams; nothing waits on another
shard).  Cuts fall on multiples of 4096 bins, so each shard computes the
tiles of a single launch: for one chunk and the zero initial grid
BaseProfile passes, the sharded results equal the one-device manager's bit
for bit, in the FP64 and FP32 forms.  Each chunk is cut for its own lines,
so a bin that two chunks reach may belong to different devices in the two;
the host then adds the devices' sums, where one device adds the second
chunk onto the first: the association differs, one rounding per chunk
(1e-15 relative).  A non-zero initial grid is likewise added once on the
host, after the devices' sums.  The FP64 form matches the
FP64 oracle within 1e-10 per bin.  A shard may be empty (more shards than
the band needs) without changing the result.
"""
import numpy as np
import pytest

from gexs_b200 import synth, _capi as capi
from gexs_b200.engine import Manager, job_init
from tests import helpers as H

pytestmark = pytest.mark.gpu

G, NU0, DNU = 120000, 100.0, 0.05
PAIRS = [(1500.0, 1.0), (600.0, 0.05)]


def _range(C):
    lo = max(0, int(np.floor((C["nu"][0] - 25.0 - NU0) / DNU)) - 1)
    hi = min(G, int(np.ceil((C["nu"][-1] + 25.0 - NU0) / DNU)) + 2)
    return lo, hi


def _drive(m, L, chunks, initial):
    freq = NU0 + np.arange(G, dtype=np.float64) * DNU
    m.initialize_vectors(G, len(PAIRS))
    m.transfer_freq(freq, initial.copy())
    m.initialize_constants(0.0, PAIRS[0][0], 1000.0, DNU, 18.0, PAIRS[0][1], 296.0, 1.0)
    for a, b in chunks:
        C = {k: np.ascontiguousarray(v[a:b]) for k, v in L.items()}
        m.transfer_vectors(C["elow"], C["nu"], C["aif"], C["gns"], C["gamma"], C["n"])
        lo, hi = _range(C)
        for T, P in PAIRS:
            m.execute(hi - lo, b - a, lo, T, P, 1000.0 + T)
    outs = []
    for i in range(len(PAIRS)):
        o = np.zeros(G)
        m.transfer_results(freq, o, i)
        outs.append(o)
    m.close()
    return outs


@pytest.mark.parametrize("prec", [capi.FP64, capi.FP32])
def test_multi_equals_single_device_and_oracle(prec):
    st = synth.make_states(3000, 40, 1007)
    L = synth.make_lines(st, 60000, 150.0, 5900.0, 2007, broadening_seed=3007)
    chunks = [(0, 25000), (25000, 60000)]
    zero = np.zeros(G)
    one = [(0, 60000)]
    single1 = _drive(Manager(capi.VOIGT, 0, capi.CONV_PHYSICAL, prec, 1 << 28), L, one, zero)
    single = _drive(Manager(capi.VOIGT, 0, capi.CONV_PHYSICAL, prec, 1 << 28), L, chunks, zero)
    for devices in ([0, 0], [0, 0, 0], [0] * 6):
        kw = dict(convention=capi.CONV_PHYSICAL, precision=prec, memory_bytes=1 << 27,
                  devices=devices)
        multi1 = _drive(Manager(capi.VOIGT, **kw), L, one, zero)
        for k, (s, m) in enumerate(zip(single1, multi1)):
            bad = np.flatnonzero(m != s)
            assert bad.size == 0, "devices %d pair %d: %d bins differ, first %s: %r vs %r" % (
                len(devices), k, bad.size, bad[:4].tolist(), m[bad[:4]].tolist(),
                s[bad[:4]].tolist())
        multi = _drive(Manager(capi.VOIGT, **kw), L, chunks, zero)
        for s, m in zip(single, multi):
            assert np.all(np.abs(m - s) <= 1e-15 * np.abs(s))
    initial = np.linspace(0.0, 1e-22, G)
    single = _drive(Manager(capi.VOIGT, 0, capi.CONV_PHYSICAL, prec, 1 << 28), L, chunks,
                    initial)
    multi = _drive(Manager(capi.VOIGT, convention=capi.CONV_PHYSICAL, precision=prec,
                           memory_bytes=1 << 27, devices=[0, 0, 0]), L, chunks, initial)
    for s, m in zip(single, multi):
        assert np.all(np.abs(m - s) <= 1e-15 * np.abs(s))
    if prec == capi.FP64:
        for (T, P), got in zip(PAIRS, single):
            want = initial.copy()
            for a, b in chunks:
                C = {k: np.ascontiguousarray(v[a:b]) for k, v in L.items()}
                j = job_init(capi.CONV_PHYSICAL, capi.VOIGT, T, P, 1000.0 + T, 18.0, NU0, DNU, G)
                j.start_idx, j.n_points = _range(C)
                j.n_points -= j.start_idx
                j.accumulate = 1
                want = H.oracle_of(j, C, out=want)
            worst, nbad = H.fp64_mismatch(got, want)
            assert nbad == 0, worst

"""The drop-in manager (B200Manager) driven exactly as BaseProfile drives a
manager (Profiles/BaseProfile.cpp:42-116,269-301): lines streamed in
nu-ordered chunks, each chunk's grid sub-range [ib, ie), one
ExecuteCrossSection per (T, P) pair filling result slot i, results read
per slot.  Compared with the FP64 oracle on the whole list."""
import numpy as np
import pytest

from gexs_b200 import _capi as capi
from gexs_b200.engine import Manager, job_init
from tests import helpers as H

pytestmark = pytest.mark.gpu

PAIRS = [(296.0, 1.0), (1500.0, 0.5), (2500.0, 3.0)]


def _drive(m, lines, freq, dfreq, mass, qs, hw, chunk, ref_temp, ref_press):
    npts = len(freq)
    m.initialize_vectors(npts, len(PAIRS))
    m.transfer_freq(freq, np.zeros(npts))
    m.initialize_constants(hw, PAIRS[0][0], qs[0], dfreq, mass, PAIRS[0][1], ref_temp, ref_press)
    assert m.ntrans() >= chunk
    n = len(lines["nu"])
    start_nu = freq[0]
    for c0 in range(0, n, chunk):
        sl = slice(c0, min(n, c0 + chunk))
        part = {k: np.ascontiguousarray(v[sl]) for k, v in lines.items()}
        m.transfer_vectors(part["elow"], part["nu"], part["aif"], part["gns"], part.get("gamma"),
                           part.get("n"))
        ib = int(max(round((part["nu"].min() - hw - start_nu) / dfreq), 0.0))
        ie = int(min(round((part["nu"].max() + hw - start_nu) / dfreq), float(npts)))
        for (T, P), q in zip(PAIRS, qs):
            m.execute(ie - ib, len(part["nu"]), ib, T, P, q)
    outs = []
    for i in range(len(PAIRS)):
        f = np.zeros(npts)
        o = np.zeros(npts)
        m.transfer_results(f, o, i)
        np.testing.assert_array_equal(f, freq)
        outs.append(o)
    return outs


@pytest.mark.parametrize("conv,profile", [(capi.CONV_REF_CPU, capi.VOIGT),
                                          (capi.CONV_REF_GPU, capi.VOIGT),
                                          (capi.CONV_REF_GPU, capi.DOPPLER),
                                          (capi.CONV_PHYSICAL, capi.VOIGT)])
def test_manager_protocol_matches_oracle(small_states, small_lines, conv, profile):
    from oracle import pyoracle as po
    nu0, dfreq, npts = 100.0, 0.05, 80000
    freq = nu0 + np.arange(npts, dtype=np.float64) * dfreq
    mass, ref_temp, ref_press = 18.0, 256.0, 1.0 / 0.986923267   # ExoMol, BaseProfile.cpp:53-54
    qs = [po.partition(small_states.energy, small_states.g, T) for T, _ in PAIRS]
    lines = small_lines if profile == capi.VOIGT else \
        {k: v for k, v in small_lines.items() if k not in ("gamma", "n")}
    m = Manager(profile, 0, conv, capi.FP64, memory_bytes=256 << 20)
    outs = _drive(m, lines, freq, dfreq, mass, qs, 101.0, 1500, ref_temp, ref_press)
    m.close()
    for (T, P), q, got in zip(PAIRS, qs, outs):
        j = job_init(conv, profile, T, P, q, mass, nu0, dfreq, npts, ref_temp=ref_temp,
                     ref_press=ref_press)
        ref = H.oracle_of(j, lines)
        floor = 1e-14 * np.max(ref) if (profile == capi.DOPPLER) else 0.0
        d = np.abs(got - ref)
        assert np.all(d <= 1e-10 * np.abs(ref) + floor), float(np.max(d / (np.abs(ref) + 1e-300)))


def test_manager_fp32_form(small_states, small_lines):
    from oracle import pyoracle as po
    nu0, dfreq, npts = 100.0, 0.05, 80000
    freq = nu0 + np.arange(npts, dtype=np.float64) * dfreq
    qs = [po.partition(small_states.energy, small_states.g, T) for T, _ in PAIRS]
    m = Manager(capi.VOIGT, 0, capi.CONV_PHYSICAL, capi.FP32, memory_bytes=256 << 20)
    outs = _drive(m, small_lines, freq, dfreq, 18.0, qs, 26.0, 1000, 296.0, 1.0)
    m.close()
    for (T, P), q, got in zip(PAIRS, qs, outs):
        j = job_init(capi.CONV_PHYSICAL, capi.VOIGT, T, P, q, 18.0, nu0, dfreq, npts)
        rel, band = H.fp32_errors(got, H.oracle_of(j, small_lines))
        assert rel <= H.FP32_REL and band <= H.FP32_BAND

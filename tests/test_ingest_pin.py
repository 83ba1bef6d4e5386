"""Pin the CPU restatement of the ExoMol reader (oracle/ingest_oracle.cpp)
to the reference's own reader, compiled from its sources
(Readers/Exomol/ExomolStateReader.cpp, exomol_functions.cpp, common/Util.cpp
-> oracle/_ref/gexsref_reader), on seeded synthetic files.  Runs on
the CPU; the GPU ingest is checked against the oracle in test_gpu_ingest.py.
"""
import os

import numpy as np
import pytest

from gexs_b200 import synth
from oracle import pyoracle as po

pytestmark = pytest.mark.skipif(not po.ref_reader_available(),
                                reason="reference reader not built (oracle/_ref)")


def _write(tmp_path, name, data):
    p = os.path.join(str(tmp_path), name)
    with open(p, "wb") as f:
        f.write(data)
    return p


def _files(tmp_path, nst=3000, ntr=5000, seed=41, nu_col=False):
    st = synth.make_states(nst, 40, seed)
    u, l, a = synth.make_exomol_transitions(st, ntr, 50.0, 6000.0, seed + 1)
    stext = synth.exomol_states_text(st)
    ttext = synth.exomol_trans_text(u, l, a, nu=(st.energy[u] - st.energy[l]) if nu_col else None)
    return st, stext, ttext


def _oracle(stext, ttext, broad=b"", mode=0, dg=0.07, dn=0.5):
    e, g, j = po.exomol_states(stext)
    return po.exomol_trans(ttext, e, g, j, broad, mode, dg, dn)


def _same(ref, orc, keys=("nu", "elow", "aif")):
    for k in keys:
        assert ref[k].shape == orc[k].shape, k
        assert np.array_equal(ref[k].view(np.int64), orc[k].view(np.int64)), k
    assert np.array_equal(ref["gns"], orc["gns"].astype(np.float64))


def test_oracle_matches_reference_reader(tmp_path):
    st, stext, ttext = _files(tmp_path)
    sp, tp = _write(tmp_path, "m.states", stext), _write(tmp_path, "m.trans", ttext)
    ref = po.ref_exomol_read(sp, tp, None, 0.07, 0.5)
    orc = _oracle(stext, ttext)
    assert len(orc["nu"]) == 5000 or len(orc["nu"]) > 4000
    _same(ref, orc)
    # no broadener file: the reference leaves gamma and n untouched (NaN in)
    assert np.isnan(ref["gamma"]).all() and np.isnan(ref["n"]).all()


def test_broadener_file_gives_defaults_in_the_reference(tmp_path):
    """ExomolStateReader.cpp:21: the lookup key keeps the failed 'a1' text
    after key.clear(), so every line gets the defaults."""
    st, stext, ttext = _files(tmp_path, seed=43)
    broad = synth.exomol_broad_text(40, 7, a1_pairs=5)
    sp, tp = _write(tmp_path, "m.states", stext), _write(tmp_path, "m.trans", ttext)
    bp = _write(tmp_path, "m.broad", broad)
    ref = po.ref_exomol_read(sp, tp, bp, 0.07, 0.5)
    orc = _oracle(stext, ttext, broad, mode=0, dg=0.07, dn=0.5)
    _same(ref, orc)
    assert (ref["gamma"] == 0.07).all() and (ref["n"] == 0.5).all()
    assert np.array_equal(orc["gamma"], ref["gamma"]) and np.array_equal(orc["n"], ref["n"])
    # the intended J'' rule differs from the defaults
    by_j = _oracle(stext, ttext, broad, mode=1, dg=0.07, dn=0.5)
    assert not np.array_equal(by_j["gamma"], orc["gamma"])


def test_edge_cases_match_reference(tmp_path):
    """No final newline, CRLF endings, blank lines between transitions, and
    states fields with leading zeros (strtol base 0 reads them as octal)."""
    st, stext, ttext = _files(tmp_path, nst=500, ntr=800, seed=47)
    lines = stext.split(b"\n")
    # give some g fields a leading zero: "    010" -> octal 8
    fixed = []
    for i, ln in enumerate(lines):
        if ln and i % 7 == 3:
            parts = ln.split()
            parts[2] = b"0" + parts[2]
            ln = b" ".join(parts)
        fixed.append(ln)
    stext2 = b"\r\n".join(fixed).rstrip(b"\r\n")              # CRLF, no final newline
    tl = ttext.split(b"\n")
    ttext2 = b"\n\n".join(tl[:300]) + b"\n" + b"\r\n".join(tl[300:]).rstrip(b"\r\n")
    sp, tp = _write(tmp_path, "e.states", stext2), _write(tmp_path, "e.trans", ttext2)
    ref = po.ref_exomol_read(sp, tp, None)
    orc = _oracle(stext2, ttext2)
    _same(ref, orc)
    e, g, j = po.exomol_states(stext2)
    assert (g[3::7] != st.g[3::7]).any()                    # octal took effect


def test_states_energies_are_strtod(tmp_path):
    st, stext, _ = _files(tmp_path, nst=2000, ntr=10, seed=53)
    e, g, j = po.exomol_states(stext)
    expect = np.array([float(ln.split()[1]) for ln in stext.splitlines()])
    assert np.array_equal(e.view(np.int64), expect.view(np.int64))
    assert np.array_equal(g, st.g) and np.array_equal(j, st.j)


def test_hitran_oracle_matches_reference_reader(tmp_path):
    """HITRANStateReader compiled from its sources (TIPS replaced by a
    constant Q(296), the Fortran being unbuildable here): nu, E'', g', n and
    gamma bit-exact; A bit-exact where the file has it, and within 4 ulp
    where the reader rebuilds it from S (glibc exp on both sides, the same
    operation order)."""
    text = synth.make_hitran_par(4000, 83)
    p = _write(tmp_path, "h.par", text)
    ref = po.ref_hitran_read(p, pressure=0.8, mixture=0.7, ref_q=174.58)
    orc = po.hitran(text, pressure=0.8, mixture=0.7, ref_q=174.58)
    assert len(orc["nu"]) == 4000 and len(ref["nu"]) == 4000
    for k in ("nu", "elow", "gamma", "n"):
        assert np.array_equal(ref[k].view(np.int64), orc[k].view(np.int64)), k
    assert np.array_equal(ref["gns"], orc["gns"].astype(np.float64))
    assert np.array_equal(ref["aif"].view(np.int64), orc["aif"].view(np.int64))
    rebuilt = np.arange(4000) % 7 == 0
    assert (orc["gns"][rebuilt] == 1).all() and (orc["aif"][rebuilt] > 0).all()

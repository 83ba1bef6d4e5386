"""TIPS-2011 partition sums (gexs_tips_2011, host code) without a GPU.

The expected values are computed here independently: the 3- and 4-point
Lagrange rule of the reference's AtoB (Readers/HITRAN/BD_TIPS_2011_v1p0.for
:5830-5920) evaluated in numpy on table values transcribed from the DATA
statement of QT_H2O (isotopologue 161, :379-398) as single-precision
literals, as the Fortran DATA statement stores them.  When the reference
tree is present, the committed tips2011_data.h is also checked to be
exactly what gen_tips2011.py extracts from the Fortran source.
"""
import ctypes as C
import filecmp
import os
import subprocess
import sys

import numpy as np
import pytest

from gexs_b200 import _capi as capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# H2O 161, Q at 60, 85, ..., 360 K (first thirteen entries of its DATA row)
H2O_161 = np.array([0.16824e+02, 0.27771e+02, 0.40408e+02, 0.54549e+02, 0.70054e+02,
                    0.86817e+02, 0.10475e+03, 0.12380e+03, 0.14391e+03, 0.16503e+03,
                    0.18714e+03, 0.21021e+03, 0.23425e+03], dtype=np.float32).astype(np.float64)
TDAT = 60.0 + 25.0 * np.arange(119)


def tips(mol, iso, T):
    gi, q = C.c_double(), C.c_double()
    st = capi.lib().gexs_tips_2011(mol, iso, T, C.byref(gi), C.byref(q))
    return st, gi.value, q.value


def lagrange(T, xs, ys):
    tot = 0.0
    for i in range(len(xs)):
        w = 1.0
        for j in range(len(xs)):
            if j != i:
                w *= (T - xs[j]) / (xs[i] - xs[j])
        tot += w * ys[i]
    return tot


@pytest.mark.parametrize("k", [1, 4, 9, 10, 12])
def test_tabulated_temperatures_return_the_table(k):
    st, gi, q = tips(1, 1, float(TDAT[k]))
    assert st == 0 and gi == 1.0
    assert abs(q - H2O_161[k]) <= 1e-15 * H2O_161[k]


@pytest.mark.parametrize("T", [70.0, 96.5, 200.0, 296.0, 300.0, 333.3])
def test_interpolated_temperatures(T):
    i = int(np.argmax(TDAT >= T))          # first grid point >= T (0-based)
    I = max(i, 1) + 1                      # AtoB's 1-based I, searched from 2
    if I < 3:
        idx = [0, 1, 2]                    # 3 points ending at index 3
    else:
        idx = [I - 3, I - 2, I - 1, I]     # 4 points I-2 .. I+1
    want = lagrange(T, TDAT[idx], H2O_161[idx])
    st, _, q = tips(1, 1, T)
    assert st == 0
    assert abs(q - want) <= 1e-13 * want, (T, q, want)


def test_h2o_q296_and_the_range_ends():
    st, gi, q = tips(1, 1, 296.0)
    assert st == 0 and abs(q - 174.58) / 174.58 < 2e-3     # the published Q(296) of H2O 161
    assert tips(1, 1, 3000.0)[0] == 0 and tips(1, 1, 70.0)[0] == 0
    st, _, q = tips(1, 1, 69.9)
    assert st == capi.GEXS_ERR_INVALID and q == -1.0
    st, _, q = tips(1, 1, 3000.5)
    assert st == capi.GEXS_ERR_INVALID and q == -1.0


def test_molecules_without_tables_and_bad_arguments():
    assert tips(34, 1, 500.0) == (0, 0.0, 0.0)      # atomic oxygen: gi = 0, Q = 0
    assert tips(39, 1, 500.0) == (0, 0.0, 0.0)
    assert tips(52, 1, 500.0)[0] == capi.GEXS_ERR_INVALID
    assert tips(0, 1, 500.0)[0] == capi.GEXS_ERR_INVALID
    assert tips(1, 7, 500.0)[0] == capi.GEXS_ERR_INVALID  # H2O has 6 isotopologues
    st, gi, q = tips(2, 11, 1000.0)                        # last CO2 isotopologue
    assert st == 0 and q > 0 and gi > 0


def test_committed_tables_are_what_the_generator_extracts(tmp_path):
    src = None
    r = subprocess.run(["make", "-s", "--no-print-directory", "-C", os.path.join(ROOT, "oracle"),
                        "print-tips-src"], capture_output=True, text=True)
    if r.returncode == 0:
        src = r.stdout.strip()
    if not src or not os.path.exists(src):
        pytest.skip("reference tree not present")
    out = os.path.join(str(tmp_path), "tips.h")
    subprocess.run([sys.executable, os.path.join(ROOT, "gexs_b200", "host", "gen_tips2011.py"),
                    src, out], check=True, capture_output=True)
    assert filecmp.cmp(out, os.path.join(ROOT, "gexs_b200", "host", "tips2011_data.h"),
                       shallow=False)

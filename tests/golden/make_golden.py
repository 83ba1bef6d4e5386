"""Generate tests/golden/reference_cpu.npz from the reference's own CPU code.

The reference has no tests, fixtures or golden vectors of its own, so the
vectors here come from running its CPU path compiled unmodified from its
sources (oracle/Makefile -> oracle/_ref/libgexsref.so, built with
-ffp-contract=off):
  - humlic(x, y)                 compute/CPU/profiles.cpp:11-44
  - compute_partition            Readers/Exomol/exomol_functions.cpp:50-73
  - OpenMPManager::ComputeVoigtTP  Managers/CPU/OpenMPManager.cpp:376-426
  - OpenMPManager::ComputeDoppler  Managers/CPU/OpenMPManager.cpp:280-323
The inputs (seeded synthetic line lists) are stored beside the outputs so
the fixture does not depend on the generator's random streams.

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gexs_b200 import synth  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

VOIGT_CASES = [  # (T [K], P) ; the CPU path's cutoff is min(25 P, 100)
    (296.0, 1.0),
    (1500.0, 0.4),
    (3000.0, 4.0),
]
DOPPLER_T = [296.0, 1500.0]
Q_TEMPS = [100.0, 296.0, 1000.0, 1500.0, 3000.0]
MASS = 18.0
REF_TEMP = 256.0      # Profiles/BaseProfile.cpp:53, ExoMol
NU0, DNU, NPTS = 100.0, 0.05, 10000


def main():
    out = {}
    st = synth.make_states(3000, 40, 1001)
    out["states_energy"] = st.energy
    out["states_g"] = st.g
    out["q_temps"] = np.array(Q_TEMPS)
    out["q_ref"] = np.array([po.ref_partition(st.energy, st.g, t) for t in Q_TEMPS])

    xs = np.concatenate([np.linspace(0.0, 20.0, 81), [1e-3, 0.5, 3.9, 4.1, 5.49, 5.51, 14.99, 15.01, 50.0, 1e3]])
    ys = np.concatenate([10.0 ** np.linspace(-6, 1.3, 25), [0.0, 0.75, 5.5, 15.0]])
    X, Y = np.meshgrid(xs, ys)
    out["hum_x"] = X.ravel()
    out["hum_y"] = Y.ravel()
    out["hum_ref"] = np.array([po.ref_humlic(x, y) for x, y in zip(X.ravel(), Y.ravel())])

    freq = NU0 + np.arange(NPTS, dtype=np.float64) * DNU
    out["grid"] = np.array([NU0, DNU, NPTS], dtype=np.float64)
    for tag, gscale in (("wide", 1.0), ("narrow", 0.01)):
        L = synth.make_lines(st, 3000, 100.0, 600.0, 2001 if tag == "wide" else 2002,
                             broadening_seed=3001)
        L["gamma"] = L["gamma"] * gscale
        for k, v in L.items():
            out["lines_%s_%s" % (tag, k)] = v
        for i, (T, P) in enumerate(VOIGT_CASES):
            q = po.ref_partition(st.energy, st.g, T)
            out["voigt_%s_%d" % (tag, i)] = po.ref_voigt_tp(freq, L, T, P, q, MASS, REF_TEMP, DNU,
                                                            nthreads=4)
            out["voigt_%s_%d_q" % (tag, i)] = np.array([q])
    Lw = {k[len("lines_wide_"):]: v for k, v in out.items() if k.startswith("lines_wide_")}
    for i, T in enumerate(DOPPLER_T):
        q = po.ref_partition(st.energy, st.g, T)
        out["doppler_%d" % i] = po.ref_doppler(freq, Lw, T, q, MASS, DNU, nthreads=4)
        out["doppler_%d_q" % i] = np.array([q])
    out["voigt_cases"] = np.array(VOIGT_CASES)
    out["doppler_t"] = np.array(DOPPLER_T)
    np.savez_compressed(os.path.join(HERE, "reference_cpu.npz"), **out)


if __name__ == "__main__":
    main()

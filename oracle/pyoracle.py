"""ctypes access to the CPU checkers (test infrastructure only).

liboracle.so  FP64 restatement of the reference algorithm (oracle.cpp)
_ref/libgexsref*.so  the reference's own CPU code built from its sources
Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use these.
"""
import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libgexsref.so")
REF_FAST_LIB = os.path.join(HERE, "_ref", "libgexsref_fast.so")
REF_READER_BIN = os.path.join(HERE, "_ref", "gexsref_reader")
REF_GPU_BIN = os.path.join(HERE, "_ref", "gexsref_gpu")

_orc = None
_refs = {}


def build(with_reference=None):
    """Build the oracle (and oracle/_ref when the reference tree exists).
    The tree is the Makefile's REF, or the GEXS_REFERENCE environment
    variable when it is set."""
    import subprocess
    ref = os.environ.get("GEXS_REFERENCE")
    var = ["REF=" + ref] if ref else []
    targets = ["oracle"]
    if with_reference is None:
        with_reference = subprocess.run(["make", "-s", "-C", HERE] + var + ["has-ref"],
                                        capture_output=True).returncode == 0
    if with_reference:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE] + var + targets, check=True)


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            build(with_reference=False)
        from gexs_b200._capi import GexsJob
        h = C.CDLL(ORACLE_LIB)
        h.orc_humlicek.restype = C.c_double
        h.orc_humlicek.argtypes = [C.c_double, C.c_double]
        h.orc_humlicek_region.restype = C.c_int
        h.orc_humlicek_region.argtypes = [C.c_double, C.c_double]
        h.orc_voigt_gh.restype = C.c_double
        h.orc_voigt_gh.argtypes = [C.c_double, C.c_double, C.c_int]
        h.orc_partition.restype = C.c_double
        h.orc_partition.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_double]
        h.orc_cross_section.restype = C.c_int
        h.orc_cross_section.argtypes = [C.POINTER(GexsJob), C.c_void_p, C.c_int]
        h.orc_count_evals.restype = C.c_int64
        h.orc_count_evals.argtypes = [C.POINTER(GexsJob)]
        h.orc_region_hist.restype = C.c_int
        h.orc_region_hist.argtypes = [C.POINTER(GexsJob), C.POINTER(C.c_int64)]
        h.orc_line_params.restype = C.c_int
        h.orc_line_params.argtypes = [C.POINTER(GexsJob), C.c_void_p, C.c_void_p, C.c_void_p]
        h.orc_exomol_states.restype = C.c_int64
        h.orc_exomol_states.argtypes = [C.c_char_p, C.c_int64] + [C.c_void_p] * 3 + [C.c_int64]
        h.orc_exomol_trans.restype = C.c_int64
        h.orc_exomol_trans.argtypes = ([C.c_char_p, C.c_int64] + [C.c_void_p] * 3 +
                                       [C.c_int64, C.c_char_p, C.c_int64, C.c_int, C.c_double,
                                        C.c_double] + [C.c_void_p] * 6 + [C.c_int64])
        h.orc_sort_by_nu.restype = None
        h.orc_sort_by_nu.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        h.orc_hitran.restype = C.c_int64
        h.orc_hitran.argtypes = [C.c_char_p, C.c_int64, C.c_double, C.c_double, C.c_double] + \
            [C.c_void_p] * 6 + [C.c_int64]
        h.orc_strtod.restype = C.c_double
        h.orc_strtod.argtypes = [C.c_char_p]
        _orc = h
    return _orc


def cross_section(host_job, out=None, nthreads=0):
    """Run the oracle on a job whose line pointers are host arrays."""
    if out is None:
        out = np.zeros(host_job.grid_points, dtype=np.float64)
    st = orc().orc_cross_section(C.byref(host_job), out.ctypes.data_as(C.c_void_p), nthreads)
    if st != 0:
        raise RuntimeError("oracle rejected the job (%d)" % st)
    return out


def count_evals(host_job):
    return int(orc().orc_count_evals(C.byref(host_job)))


def region_hist(host_job):
    h = (C.c_int64 * 4)()
    orc().orc_region_hist(C.byref(host_job), h)
    return [int(v) for v in h]


def partition(energy, g, temp):
    energy = np.ascontiguousarray(energy, np.float64)
    g = np.ascontiguousarray(g, np.int32)
    return orc().orc_partition(energy.ctypes.data_as(C.c_void_p), g.ctypes.data_as(C.c_void_p),
                               len(energy), temp)


def humlicek(x, y):
    return orc().orc_humlicek(x, y)


def voigt_gh(x, y, nodes):
    return orc().orc_voigt_gh(x, y, nodes)


def ref_available(fast=False):
    return os.path.exists(REF_FAST_LIB if fast else REF_LIB)


def ref(fast=False):
    path = REF_FAST_LIB if fast else REF_LIB
    if path not in _refs:
        if not os.path.exists(path):
            raise RuntimeError("reference build missing: %s (make -C oracle ref)" % path)
        h = C.CDLL(path)
        h.ref_voigt_tp.restype = C.c_int
        h.ref_voigt_tp.argtypes = [C.c_int, C.c_void_p, C.c_int] + [C.c_void_p] * 6 + \
            [C.c_double] * 6 + [C.c_int, C.c_void_p]
        h.ref_doppler.restype = C.c_int
        h.ref_doppler.argtypes = [C.c_int, C.c_void_p, C.c_int] + [C.c_void_p] * 4 + \
            [C.c_double] * 4 + [C.c_int, C.c_void_p]
        h.ref_partition.restype = C.c_double
        h.ref_partition.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_double]
        h.ref_humlic.restype = C.c_double
        h.ref_humlic.argtypes = [C.c_double, C.c_double]
        _refs[path] = h
    return _refs[path]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def ref_voigt_tp(freq, lines, temperature, pressure, partition_q, mass, ref_temp, dfreq,
                 nthreads=1, fast=False):
    """Managers/CPU/OpenMPManager.cpp:376-426 on the whole grid."""
    out = np.zeros(len(freq), np.float64)
    st = ref(fast).ref_voigt_tp(len(freq), _p(freq), len(lines["nu"]), _p(lines["nu"]),
                                _p(lines["elow"]), _p(lines["aif"]), _p(lines["gns"]),
                                _p(lines["gamma"]), _p(lines["n"]), temperature, pressure,
                                partition_q, mass, ref_temp, dfreq, nthreads, _p(out))
    if st != 0:
        raise RuntimeError("reference harness failed")
    return out


def ref_doppler(freq, lines, temperature, partition_q, mass, dfreq, nthreads=1, fast=False):
    """Managers/CPU/OpenMPManager.cpp:280-323 on the whole grid."""
    out = np.zeros(len(freq), np.float64)
    st = ref(fast).ref_doppler(len(freq), _p(freq), len(lines["nu"]), _p(lines["nu"]),
                               _p(lines["elow"]), _p(lines["aif"]), _p(lines["gns"]),
                               temperature, partition_q, mass, dfreq, nthreads, _p(out))
    if st != 0:
        raise RuntimeError("reference harness failed")
    return out


def ref_partition(energy, g, temp, fast=False):
    energy = np.ascontiguousarray(energy, np.float64)
    g = np.ascontiguousarray(g, np.int32)
    return ref(fast).ref_partition(len(energy), _p(energy), _p(g), temp)


def ref_humlic(x, y):
    return ref().ref_humlic(x, y)


# ------------------------------------------------------------------ ExoMol ingest
def exomol_states(text):
    """Restated exomol_functions.cpp:8-48: (energy, g, J) per fgets line."""
    h = orc()
    n = h.orc_exomol_states(text, len(text), None, None, None, 0)
    e = np.zeros(n, np.float64); g = np.zeros(n, np.int32); j = np.zeros(n, np.int32)
    h.orc_exomol_states(text, len(text), _p(e), _p(g), _p(j), n)
    return e, g, j


def exomol_trans(text, energy, g, j, broad=b"", mode=0, default_gamma=0.1, default_n=0.1,
                 sort_by_nu=False):
    """Restated ExomolStateReader.cpp:132-172 (token stream), file order or
    stably sorted by nu."""
    h = orc()
    energy = np.ascontiguousarray(energy, np.float64)
    g = np.ascontiguousarray(g, np.int32); j = np.ascontiguousarray(j, np.int32)
    args = (text, len(text), _p(energy), _p(g), _p(j), len(energy), broad, len(broad), mode,
            default_gamma, default_n)
    n = h.orc_exomol_trans(*args, None, None, None, None, None, None, 0)
    if n < 0:
        raise ValueError("state id out of range")
    d = {k: np.zeros(n, np.float64) for k in ("nu", "elow", "aif", "gamma", "n")}
    d["gns"] = np.zeros(n, np.int32)
    h.orc_exomol_trans(*args, _p(d["nu"]), _p(d["elow"]), _p(d["aif"]), _p(d["gns"]),
                       _p(d["gamma"]), _p(d["n"]), n)
    if sort_by_nu and n:
        perm = np.zeros(n, np.int64)
        h.orc_sort_by_nu(_p(d["nu"]), n, _p(perm))
        d = {k: v[perm] for k, v in d.items()}
    return d


def strtod(s):
    return orc().orc_strtod(s)


def ref_reader_available():
    return os.path.exists(REF_READER_BIN)


def ref_exomol_read(states_path, trans_path, broad_path=None, default_gamma=0.1, default_n=0.1):
    """The reference's ExomolStateReader (compiled from its sources, run as
    oracle/_ref/gexsref_reader): every transition in file order as
    (nu, gns, e_i, aif, gamma, n)."""
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "ref.bin")
        subprocess.run([REF_READER_BIN, states_path, trans_path, broad_path or "-",
                        repr(float(default_gamma)), repr(float(default_n)), out], check=True,
                       stdout=subprocess.DEVNULL)
        raw = np.fromfile(out, dtype=np.uint8)
    n = int(raw[:8].view(np.int64)[0])
    arr = raw[8:].view(np.float64).reshape(6, n) if n else np.zeros((6, 0))
    keys = ("nu", "gns", "elow", "aif", "gamma", "n")
    return {k: arr[i].copy() for i, k in enumerate(keys)}


def hitran(text, pressure=1.0, mixture=1.0, ref_q=1.0, sort_by_nu=False):
    """Restated HITRANStateReader.cpp:137-250 (Q(296) = ref_q)."""
    h = orc()
    args = (text, len(text), pressure, mixture, ref_q)
    n = h.orc_hitran(*args, None, None, None, None, None, None, 0)
    d = {k: np.zeros(n, np.float64) for k in ("nu", "elow", "aif", "gamma", "n")}
    d["gns"] = np.zeros(n, np.int32)
    h.orc_hitran(*args, _p(d["nu"]), _p(d["elow"]), _p(d["aif"]), _p(d["gns"]), _p(d["gamma"]),
                 _p(d["n"]), n)
    if sort_by_nu and n:
        perm = np.zeros(n, np.int64)
        h.orc_sort_by_nu(_p(d["nu"]), n, _p(perm))
        d = {k: v[perm] for k, v in d.items()}
    return d


def ref_hitran_read(path, pressure=1.0, mixture=1.0, ref_q=1.0):
    """The reference's HITRANStateReader (compiled from its sources, TIPS
    replaced by the constant ref_q): every record in file order as
    (nu, gns, e_i, aif, gamma, n)."""
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "ref.bin")
        subprocess.run([REF_READER_BIN, "hitran", path, repr(float(pressure)), repr(float(mixture)),
                        repr(float(ref_q)), out], check=True, stdout=subprocess.DEVNULL)
        raw = np.fromfile(out, dtype=np.uint8)
    n = int(raw[:8].view(np.int64)[0])
    arr = raw[8:].view(np.float64).reshape(6, n) if n else np.zeros((6, 0))
    keys = ("nu", "gns", "elow", "aif", "gamma", "n")
    return {k: arr[i].copy() for i, k in enumerate(keys)}


def ref_gpu_available():
    return os.path.exists(REF_GPU_BIN)


def ref_gpu_voigt(lines, nu_start, dnu, npts, temperature, pressure, partition, mass,
                  ref_temp=296.0, ref_press=1.0, half_width=0.0, reps=1,
                  budget_bytes=1 << 30, timeout=600):
    """The reference's GPU manager and v2 Voigt kernel (GpuManager,
    compute/CUDA/cross_kernal_v2.cu:403-457, built for sm_100a as
    oracle/_ref/gexsref_gpu) on one (T, P) pair over the grid nu_start +
    j*dnu, j < npts: returns (sigma, [ms per repetition]).  Needs a GPU; the
    reference window is its LORENTZ_CUTOFF (100 cm^-1, inclusive)."""
    import json
    import subprocess
    import tempfile
    n = int(len(lines["nu"]))
    hdr = np.array([n, int(npts), int(reps), int(budget_bytes)], dtype=np.int64)
    par = np.array([nu_start, dnu, temperature, pressure, partition, mass, ref_temp, ref_press,
                    half_width], dtype=np.float64)
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(inp, "wb") as f:
            f.write(hdr.tobytes()); f.write(par.tobytes())
            for k in ("elow", "nu", "aif"):
                f.write(np.ascontiguousarray(lines[k], dtype=np.float64).tobytes())
            f.write(np.ascontiguousarray(lines["gns"], dtype=np.int32).tobytes())
            for k in ("gamma", "n"):
                f.write(np.ascontiguousarray(lines[k], dtype=np.float64).tobytes())
        p = subprocess.run([REF_GPU_BIN, inp, out], check=True, capture_output=True, text=True,
                           timeout=timeout)
        sigma = np.fromfile(out, dtype=np.float64)
    ms = json.loads(p.stdout.strip().splitlines()[-1])["ms"]
    return sigma, ms

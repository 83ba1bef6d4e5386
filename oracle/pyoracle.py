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

_orc = None
_refs = {}


def build(with_reference=None):
    """Build the oracle (and oracle/_ref when the reference tree exists)."""
    import subprocess
    ref = os.environ.get("GEXS_REFERENCE", "/root/reference")
    targets = ["oracle"]
    if with_reference is None:
        with_reference = os.path.isdir(ref)
    if with_reference:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, "REF=" + ref] + targets, check=True)


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

"""gexs_b200 — B200 (sm_100a) cross-section engine for GEXS line lists.

The compute path is libgexs_b200.so (CUDA kernels + C ABI, see
include/gexs_b200.h); B200Manager (gexs_b200/host) is the drop-in for the
reference's BaseManager plug-in interface.  This package adds the Python
view used by tests and the benchmark.
"""
from ._capi import (GAUSSIAN, DOPPLER, VOIGT, VOIGT_QUAD, FP64, FP32,  # noqa: F401
                    WINDOW_INCLUSIVE, WINDOW_ROUNDED, ERF_STABLE, ERF_LITERAL,
                    CONV_PHYSICAL, CONV_REF_CPU, CONV_REF_GPU, GexsError, LIB_PATH)
from .engine import (Context, Job, LineList, Manager, Batch, Server, job_init,  # noqa: F401
                     parse_exomol, load_exomol)

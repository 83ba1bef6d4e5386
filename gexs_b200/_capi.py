"""ctypes binding of include/gexs_b200.h (libgexs_b200.so, built in-tree).

Loading fails loudly when the library is missing: there is no fallback
path.  Structures mirror the C layouts field by field.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgexs_b200.so")

GEXS_OK = 0
GEXS_ERR_INVALID = -1
GEXS_ERR_OOM = -2
GEXS_ERR_TIMEOUT = -4
GEXS_ERR_NOT_READY = -5
GEXS_ERR_ADMISSION = -6
GEXS_ERR_KERNEL = -8
KERR_PIPELINE = 1
NOALLOC_MAX_JOBS = 64

GAUSSIAN, DOPPLER, VOIGT, VOIGT_QUAD = 0, 1, 2, 4
FP64, FP32 = 0, 1
WINDOW_INCLUSIVE, WINDOW_ROUNDED = 0, 1
ERF_STABLE, ERF_LITERAL = 0, 1
CONV_PHYSICAL, CONV_REF_CPU, CONV_REF_GPU = 0, 1, 2


LINES_FP64, LINES_COMPACT = 0, 1


class GexsLines(C.Structure):
    _fields_ = [("nu", C.c_void_p), ("elow", C.c_void_p), ("aif", C.c_void_p),
                ("gns", C.c_void_p), ("gamma", C.c_void_p), ("n", C.c_void_p),
                ("count", C.c_int64), ("format", C.c_int32), ("reserved", C.c_int32)]


class GexsJob(C.Structure):
    _fields_ = [("lines", GexsLines), ("out", C.c_void_p),
                ("nu_start", C.c_double), ("dnu", C.c_double),
                ("grid_points", C.c_int64), ("start_idx", C.c_int64), ("n_points", C.c_int64),
                ("profile", C.c_int32), ("precision", C.c_int32),
                ("window_rule", C.c_int32), ("accumulate", C.c_int32),
                ("quad_nodes", C.c_int32), ("erf_form", C.c_int32),
                ("cutoff", C.c_double), ("partition", C.c_double), ("beta", C.c_double),
                ("s_scale", C.c_double), ("s_scale2", C.c_double), ("dop_coef", C.c_double),
                ("inv_width", C.c_double), ("t_ratio", C.c_double),
                ("gamma_scale", C.c_double), ("out_scale", C.c_double)]


class GexsLaunchCfg(C.Structure):
    _fields_ = [("bins_per_lane", C.c_int32), ("warps", C.c_int32),
                ("ctas_per_sm", C.c_int32), ("flags", C.c_int32), ("wait_spins", C.c_int32)]

LAUNCH_DERIVE_ON_LOAD = 1
LAUNCH_LONG_STAGES = 2
LAUNCH_JOB_MAJOR = 4


class GexsRequest(C.Structure):
    _fields_ = [("list_id", C.c_int32), ("profile", C.c_int32), ("precision", C.c_int32),
                ("convention", C.c_int32), ("quad_nodes", C.c_int32), ("reserved", C.c_int32),
                ("temperature", C.c_double), ("pressure", C.c_double),
                ("nu_start", C.c_double), ("dnu", C.c_double), ("grid_points", C.c_int64),
                ("cutoff", C.c_double), ("half_width", C.c_double), ("ref_temp", C.c_double),
                ("ref_press", C.c_double)]


class GexsRequestInfo(C.Structure):
    _fields_ = [("submit_ms", C.c_double), ("admit_ms", C.c_double), ("done_ms", C.c_double),
                ("fetched_ms", C.c_double), ("evals", C.c_int64), ("batch_size", C.c_int32),
                ("status", C.c_int32)]


BROAD_DEFAULTS, BROAD_BY_J = 0, 1
OUT_BINARY, OUT_TEXT = 0, 1


class GexsStateTable(C.Structure):
    _fields_ = [("energy", C.c_void_p), ("g", C.c_void_p), ("J", C.c_void_p),
                ("count", C.c_int64)]


class GexsLineTable(C.Structure):
    _fields_ = [("nu", C.c_void_p), ("elow", C.c_void_p), ("aif", C.c_void_p),
                ("gns", C.c_void_p), ("gamma", C.c_void_p), ("n", C.c_void_p),
                ("count", C.c_int64)]


# (name, restype, argtypes) for every symbol of include/gexs_b200.h,
# include/gexs_serve.h and include/gexs_reader.h
SIGNATURES = [
    ("gexs_version", C.c_int, []),
    ("gexs_status_string", C.c_char_p, [C.c_int]),
    ("gexs_last_error", C.c_char_p, []),
    ("gexs_job_init", C.c_int, [C.POINTER(GexsJob), C.c_int, C.c_int, C.c_double, C.c_double,
                                C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                C.c_double, C.c_double, C.c_double, C.c_int64]),
    ("gexs_ctx_create", C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    ("gexs_ctx_destroy", C.c_int, [C.c_void_p]),
    ("gexs_ctx_check", C.c_int, [C.c_void_p, C.c_void_p]),
    ("gexs_run_noalloc", C.c_int, [C.POINTER(GexsJob), C.c_int, C.POINTER(GexsLaunchCfg),
                                   C.c_void_p]),
    ("gexs_noalloc_status", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("gexs_run", C.c_int, [C.c_void_p, C.POINTER(GexsJob), C.c_int,
                           C.POINTER(GexsLaunchCfg), C.c_void_p]),
    ("gexs_count_evals", C.c_int, [C.c_void_p, C.POINTER(GexsJob), C.c_int,
                                   C.POINTER(C.c_int64)]),
    ("gexs_batch_create", C.c_int, [C.c_void_p, C.POINTER(GexsJob), C.c_int,
                                    C.POINTER(GexsLaunchCfg), C.POINTER(C.c_void_p)]),
    ("gexs_batch_launch", C.c_int, [C.c_void_p, C.c_void_p]),
    ("gexs_batch_capture", C.c_int, [C.c_void_p, C.c_void_p]),
    ("gexs_batch_replay", C.c_int, [C.c_void_p, C.c_void_p]),
    ("gexs_batch_destroy", C.c_int, [C.c_void_p]),
    ("gexs_autotune", C.c_int, [C.c_void_p, C.POINTER(GexsJob), C.c_int,
                                C.POINTER(GexsLaunchCfg), C.POINTER(C.c_float)]),
    ("gexs_partition", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                 C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double)]),
    ("gexs_probe_fp32_tflops", C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    ("gexs_probe_fp64_tflops", C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    ("gexs_probe_rcp_gops", C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    ("gexs_exomol_parse_states", C.c_int, [C.c_void_p, C.c_char_p, C.c_int64,
                                           C.POINTER(GexsStateTable)]),
    ("gexs_exomol_parse_trans", C.c_int, [C.c_void_p, C.POINTER(GexsStateTable), C.c_char_p,
                                          C.c_int64, C.c_char_p, C.c_int64, C.c_int, C.c_double,
                                          C.c_double, C.c_int, C.POINTER(GexsLineTable)]),
    ("gexs_exomol_load", C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int,
                                   C.c_double, C.c_double, C.c_int, C.POINTER(GexsStateTable),
                                   C.POINTER(GexsLineTable)]),
    ("gexs_hitran_parse", C.c_int, [C.c_void_p, C.c_char_p, C.c_int64, C.c_double, C.c_double,
                                    C.c_double, C.c_int, C.POINTER(GexsLineTable)]),
    ("gexs_tips_2011", C.c_int, [C.c_int, C.c_int, C.c_double, C.POINTER(C.c_double),
                                 C.POINTER(C.c_double)]),
    ("gexs_state_table_export", C.c_int, [C.POINTER(GexsStateTable)] + [C.c_void_p] * 3),
    ("gexs_line_table_export", C.c_int, [C.POINTER(GexsLineTable)] + [C.c_void_p] * 6),
    ("gexs_state_table_free", C.c_int, [C.POINTER(GexsStateTable)]),
    ("gexs_write_sigma", C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double,
                                   C.c_double, C.c_double, C.c_double, C.c_int64, C.c_void_p,
                                   C.c_int]),
    ("gexs_reader_create", C.c_int, [C.c_char_p, C.c_char_p, C.c_double, C.c_double, C.c_int,
                                     C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("gexs_reader_open", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int64)]),
    ("gexs_reader_next", C.c_int, [C.c_void_p] + [C.POINTER(C.c_double)] * 6 +
     [C.POINTER(C.c_int)]),
    ("gexs_reader_partition", C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_double)]),
    ("gexs_reader_device_lines", C.c_int, [C.c_void_p, C.POINTER(GexsLines)]),
    ("gexs_reader_close", C.c_int, [C.c_void_p]),
    ("gexs_reader_destroy", C.c_int, [C.c_void_p]),
    ("gexs_line_table_free", C.c_int, [C.POINTER(GexsLineTable)]),
    ("gexs_manager_create", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_size_t,
                                      C.POINTER(C.c_void_p)]),
    ("gexs_manager_destroy", C.c_int, [C.c_void_p]),
    ("gexs_manager_create_multi", C.c_int, [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                            C.c_size_t, C.POINTER(C.c_void_p)]),
    ("gexs_shard_plan", C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_int64,
                                  C.c_int64, C.c_double, C.c_int, C.c_int, C.c_void_p,
                                  C.c_void_p, C.c_void_p]),
    ("gexs_manager_initialize_vectors", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("gexs_manager_initialize_constants", C.c_int, [C.c_void_p] + [C.c_double] * 8),
    ("gexs_manager_transfer_freq", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    ("gexs_manager_transfer_vectors", C.c_int, [C.c_void_p, C.c_size_t] + [C.c_void_p] * 6),
    ("gexs_manager_execute", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                       C.c_double, C.c_double, C.c_double]),
    ("gexs_manager_transfer_results", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_int, C.c_int]),
    ("gexs_manager_ntrans", C.c_int, [C.c_void_p, C.POINTER(C.c_size_t)]),
    ("gexs_manager_ready", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("gexs_server_create", C.c_int, [C.c_int, C.c_size_t, C.c_int, C.c_int,
                                     C.POINTER(C.c_void_p)]),
    ("gexs_server_destroy", C.c_int, [C.c_void_p]),
    ("gexs_server_add_list", C.c_int, [C.c_void_p] + [C.c_void_p] * 6 +
     [C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_double, C.POINTER(C.c_int)]),
    ("gexs_debug_fail_allocs", C.c_int, [C.c_int]),
    ("gexs_debug_tile_order", C.c_int, [C.POINTER(C.c_int32), C.c_int, C.POINTER(C.c_int32)]),
    ("gexs_server_add_lines", C.c_int, [C.c_void_p, C.POINTER(GexsLines), C.c_void_p, C.c_void_p,
                                        C.c_int64, C.c_double, C.POINTER(C.c_int)]),
    ("gexs_server_submit", C.c_int, [C.c_void_p, C.POINTER(GexsRequest), C.POINTER(C.c_uint64)]),
    ("gexs_server_wait", C.c_int, [C.c_void_p, C.c_uint64, C.c_int, C.c_void_p,
                                   C.POINTER(GexsRequestInfo)]),
    ("gexs_server_poll", C.c_int, [C.c_void_p, C.c_uint64]),
    ("gexs_server_stats", C.c_int, [C.c_void_p] + [C.POINTER(C.c_int64)] * 4),
    ("gexs_server_partition", C.c_int, [C.c_void_p, C.c_int, C.c_double,
                                        C.POINTER(C.c_double), C.POINTER(C.c_int)]),
]

_lib = None


def lib():
    """Load libgexs_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libgexs_b200.so is missing: run `python -m gexs_b200.build` "
                               "(the CUDA library is required; there is no CPU fallback)")
        h = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


class GexsError(RuntimeError):
    def __init__(self, status, where):
        L = lib()
        msg = L.gexs_last_error().decode(errors="replace")
        super().__init__("%s failed: %s (%d): %s" % (
            where, L.gexs_status_string(status).decode(), status, msg))
        self.status = status


def check(status, where):
    if status != GEXS_OK:
        raise GexsError(status, where)
    return status

"""Python view of the engine's C ABI (device memory via torch tensors).

The product path is the C ABI in libgexs_b200.so; this module only packs
descriptors and keeps the tensors they point at alive.
"""
import ctypes as C
import numpy as np

from . import _capi as capi
from ._capi import check, lib


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream_handle(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


class LineList:
    """Device-resident line list (structure of arrays, sorted by nu).

    compact=True stores nu in FP64 and E'', g'A, gamma, n as float
    (GEXS_LINES_COMPACT, 24 bytes per line): gns is folded into aif."""

    def __init__(self, nu, elow, aif, gns, gamma=None, n=None, device="cuda", compact=False):
        import torch
        def to(a, dt):
            if a is None:
                return None
            return torch.as_tensor(a, dtype=dt).to(device).contiguous()
        self.compact = compact
        self.nu = to(nu, torch.float64)
        if compact:
            ga = torch.as_tensor(aif, dtype=torch.float64).to(device) * \
                torch.as_tensor(gns).to(device).to(torch.float64)
            self.elow = to(elow, torch.float32)
            self.aif = ga.to(torch.float32).contiguous()
            self.gns = None
            self.gamma = to(gamma, torch.float32)
            self.n = to(n, torch.float32)
        else:
            self.elow = to(elow, torch.float64)
            self.aif = to(aif, torch.float64)
            self.gns = to(gns, torch.int32)
            self.gamma = to(gamma, torch.float64)
            self.n = to(n, torch.float64)
        self.count = int(self.nu.shape[0])

    def widened(self):
        """The values the kernels compute with, as FP64 host arrays (g' = 1
        for a compact list): what the oracle is given to check it."""
        d = {"nu": self.nu.cpu().numpy(), "elow": self.elow.double().cpu().numpy(),
             "aif": self.aif.double().cpu().numpy()}
        d["gns"] = (np.ones(self.count, dtype=np.int32) if self.compact
                    else self.gns.cpu().numpy())
        if self.gamma is not None:
            d["gamma"] = self.gamma.double().cpu().numpy()
            d["n"] = self.n.double().cpu().numpy()
        return d

    @classmethod
    def from_dict(cls, d, device="cuda"):
        return cls(d["nu"], d["elow"], d["aif"], d["gns"], d.get("gamma"), d.get("n"), device)

    def c_lines(self):
        return capi.GexsLines(_ptr(self.nu), _ptr(self.elow), _ptr(self.aif), _ptr(self.gns),
                              _ptr(self.gamma), _ptr(self.n), self.count,
                              capi.LINES_COMPACT if self.compact else capi.LINES_FP64)

    def nbytes(self):
        return sum(t.numel() * t.element_size() for t in
                   (self.nu, self.elow, self.aif, self.gns, self.gamma, self.n) if t is not None)


def job_init(convention, profile, temperature, pressure, partition, mass, nu_start, dnu,
             grid_points, ref_temp=296.0, ref_press=1.0, half_width=0.0, cutoff=-1.0):
    """gexs_job_init: physics constants of a convention (no pointers set)."""
    j = capi.GexsJob()
    check(lib().gexs_job_init(C.byref(j), convention, profile, temperature, pressure, partition,
                              mass, ref_temp, ref_press, half_width, cutoff, nu_start, dnu,
                              int(grid_points)), "gexs_job_init")
    return j


class Job:
    """One cross-section job: a GexsJob plus the tensors it references."""

    def __init__(self, lines, out, *, convention, profile, temperature, pressure, partition,
                 mass, nu_start, dnu, grid_points, precision=capi.FP32, ref_temp=296.0,
                 ref_press=1.0, half_width=0.0, cutoff=-1.0, start_idx=0, n_points=None,
                 accumulate=0, quad_nodes=16, window_rule=None, erf_form=None):
        self.c = job_init(convention, profile, temperature, pressure, partition, mass,
                          nu_start, dnu, grid_points, ref_temp, ref_press, half_width, cutoff)
        self.lines = lines
        self.out = out
        self.c.lines = lines.c_lines()
        self.c.out = out.data_ptr()
        self.c.precision = precision
        self.c.start_idx = start_idx
        self.c.n_points = grid_points - start_idx if n_points is None else n_points
        self.c.accumulate = accumulate
        self.c.quad_nodes = quad_nodes
        if window_rule is not None:
            self.c.window_rule = window_rule
        if erf_form is not None:
            self.c.erf_form = erf_form

    def host_copy(self, host_lines):
        """The same job pointing at host numpy arrays (for the oracle)."""
        j = capi.GexsJob.from_buffer_copy(self.c)
        hl = host_lines
        def p(a):
            return None if a is None else a.ctypes.data_as(C.c_void_p)
        j.lines = capi.GexsLines(p(hl["nu"]), p(hl["elow"]), p(hl["aif"]), p(hl["gns"]),
                                 p(hl.get("gamma")), p(hl.get("n")), len(hl["nu"]))
        j.out = None
        return j


def _job_array(jobs):
    arr = (capi.GexsJob * len(jobs))()
    for i, j in enumerate(jobs):
        arr[i] = j.c if isinstance(j, Job) else j
    return arr


def _cfg(cfg):
    if cfg is None:
        return None
    if isinstance(cfg, capi.GexsLaunchCfg):
        return C.byref(cfg)
    b, w, c = cfg[:3]
    return C.byref(capi.GexsLaunchCfg(b, w, c, cfg[3] if len(cfg) > 3 else 0,
                                      cfg[4] if len(cfg) > 4 else 0))


class Batch:
    def __init__(self, ctx, jobs, cfg=None):
        self._jobs = list(jobs)
        self.h = C.c_void_p()
        arr = _job_array(self._jobs)
        check(lib().gexs_batch_create(ctx.h, arr, len(arr), _cfg(cfg), C.byref(self.h)),
              "gexs_batch_create")

    def launch(self, stream=None):
        check(lib().gexs_batch_launch(self.h, _stream_handle(stream)), "gexs_batch_launch")

    def capture(self, stream):
        check(lib().gexs_batch_capture(self.h, _stream_handle(stream)), "gexs_batch_capture")

    def replay(self, stream=None):
        check(lib().gexs_batch_replay(self.h, _stream_handle(stream)), "gexs_batch_replay")

    def close(self):
        if self.h:
            lib().gexs_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    def __init__(self, device=0):
        self.h = C.c_void_p()
        check(lib().gexs_ctx_create(device, C.byref(self.h)), "gexs_ctx_create")

    def close(self):
        if self.h:
            lib().gexs_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, jobs, cfg=None, stream=None):
        arr = _job_array(jobs)
        check(lib().gexs_run(self.h, arr, len(arr), _cfg(cfg), _stream_handle(stream)), "gexs_run")

    def check(self, stream=None):
        check(lib().gexs_ctx_check(self.h, _stream_handle(stream)), "gexs_ctx_check")

    def count_evals(self, jobs):
        arr = _job_array(jobs)
        out = (C.c_int64 * len(arr))()
        check(lib().gexs_count_evals(self.h, arr, len(arr), out), "gexs_count_evals")
        return [int(v) for v in out]

    def batch(self, jobs, cfg=None):
        return Batch(self, jobs, cfg)

    def autotune(self, jobs):
        arr = _job_array(jobs)
        best = capi.GexsLaunchCfg()
        ms = C.c_float()
        check(lib().gexs_autotune(self.h, arr, len(arr), C.byref(best), C.byref(ms)),
              "gexs_autotune")
        return (best.bins_per_lane, best.warps, best.ctas_per_sm, best.flags), float(ms.value)

    def partition(self, energy, g, temps):
        temps = np.ascontiguousarray(temps, dtype=np.float64)
        q = np.zeros_like(temps)
        check(lib().gexs_partition(self.h, _ptr(energy), _ptr(g), int(energy.shape[0]),
                                   temps.ctypes.data_as(C.POINTER(C.c_double)), len(temps),
                                   q.ctypes.data_as(C.POINTER(C.c_double))), "gexs_partition")
        return q


# ---------------------------------------------------------------- ingest
def _export_states(t, device):
    import torch
    n = int(t.count)
    e = torch.empty(n, dtype=torch.float64, device=device)
    g = torch.empty(n, dtype=torch.int32, device=device)
    j = torch.empty(n, dtype=torch.int32, device=device)
    if n:
        check(lib().gexs_state_table_export(C.byref(t), _ptr(e), _ptr(g), _ptr(j)),
              "gexs_state_table_export")
    lib().gexs_state_table_free(C.byref(t))
    return {"energy": e, "g": g, "J": j}


def _export_lines(t, device):
    import torch
    n = int(t.count)
    d = {k: torch.empty(n, dtype=torch.float64, device=device)
         for k in ("nu", "elow", "aif", "gamma", "n")}
    d["gns"] = torch.empty(n, dtype=torch.int32, device=device)
    if n:
        check(lib().gexs_line_table_export(C.byref(t), _ptr(d["nu"]), _ptr(d["elow"]),
                                           _ptr(d["aif"]), _ptr(d["gns"]), _ptr(d["gamma"]),
                                           _ptr(d["n"])), "gexs_line_table_export")
    lib().gexs_line_table_free(C.byref(t))
    return d


def parse_exomol(ctx, states_text, trans_text, broad_text=b"", broad_mode=capi.BROAD_DEFAULTS,
                 default_gamma=0.1, default_n=0.1, sort_by_nu=True, device="cuda"):
    """ExoMol .states/.trans (and .broad) text parsed on the GPU (gexs_exomol_*):
    returns (states dict, lines dict) of torch device tensors."""
    st = capi.GexsStateTable()
    check(lib().gexs_exomol_parse_states(ctx.h, states_text, len(states_text), C.byref(st)),
          "gexs_exomol_parse_states")
    lt = capi.GexsLineTable()
    rc = lib().gexs_exomol_parse_trans(ctx.h, C.byref(st), trans_text, len(trans_text),
                                       broad_text, len(broad_text), broad_mode, default_gamma,
                                       default_n, 1 if sort_by_nu else 0, C.byref(lt))
    if rc != capi.GEXS_OK:
        lib().gexs_state_table_free(C.byref(st))
        check(rc, "gexs_exomol_parse_trans")
    return _export_states(st, device), _export_lines(lt, device)


def parse_hitran(ctx, text, pressure=1.0, air_mixture=1.0, ref_partition_296=1.0,
                 sort_by_nu=True, device="cuda"):
    """HITRAN .par text parsed on the GPU (gexs_hitran_parse): lines dict of
    torch device tensors."""
    lt = capi.GexsLineTable()
    check(lib().gexs_hitran_parse(ctx.h, text, len(text), pressure, air_mixture,
                                  ref_partition_296, 1 if sort_by_nu else 0, C.byref(lt)),
          "gexs_hitran_parse")
    return _export_lines(lt, device)


def load_exomol(ctx, states_path, trans_path, broad_path=None, broad_mode=capi.BROAD_DEFAULTS,
                default_gamma=0.1, default_n=0.1, sort_by_nu=True, device="cuda"):
    """gexs_exomol_load: read the files on the host, parse on the GPU."""
    st, lt = capi.GexsStateTable(), capi.GexsLineTable()
    check(lib().gexs_exomol_load(ctx.h, states_path.encode(), trans_path.encode(),
                                 broad_path.encode() if broad_path else None, broad_mode,
                                 default_gamma, default_n, 1 if sort_by_nu else 0,
                                 C.byref(st), C.byref(lt)), "gexs_exomol_load")
    return _export_states(st, device), _export_lines(lt, device)


class Manager:
    """The drop-in BaseManager (B200Manager) through its flat C wrappers;
    host numpy arrays in and out, exactly as BaseProfile passes them."""

    def __init__(self, profile, device=0, convention=capi.CONV_REF_GPU, precision=capi.FP64,
                 memory_bytes=0, devices=None):
        """devices (a list) makes the multi-GPU manager, one bin range per
        entry (gexs_manager_create_multi); otherwise one device."""
        self.h = C.c_void_p()
        if devices is not None:
            arr = (C.c_int * len(devices))(*devices)
            check(lib().gexs_manager_create_multi(profile, arr, len(devices), convention,
                                                  precision, memory_bytes, C.byref(self.h)),
                  "gexs_manager_create_multi")
            return
        check(lib().gexs_manager_create(profile, device, convention, precision, memory_bytes,
                                        C.byref(self.h)), "gexs_manager_create")

    def close(self):
        if self.h:
            lib().gexs_manager_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _p(a):
        return None if a is None else a.ctypes.data_as(C.c_void_p)

    def initialize_vectors(self, npoints, num_cs):
        check(lib().gexs_manager_initialize_vectors(self.h, npoints, num_cs), "InitializeVectors")

    def initialize_constants(self, half_width, temperature, partition, dfreq, meanmass,
                             pressure=10.0, ref_temp=296.0, ref_press=1.0):
        check(lib().gexs_manager_initialize_constants(self.h, half_width, temperature, partition,
                                                      dfreq, meanmass, pressure, ref_temp,
                                                      ref_press), "InitializeConstants")

    def transfer_freq(self, freq, intens):
        check(lib().gexs_manager_transfer_freq(self.h, self._p(freq), self._p(intens), len(freq)),
              "TransferFreq")

    def transfer_vectors(self, energies, nu, aif, gns, gamma=None, n=None):
        check(lib().gexs_manager_transfer_vectors(self.h, len(nu), self._p(energies), self._p(nu),
                                                  self._p(aif), self._p(gns), self._p(gamma),
                                                  self._p(n)), "TransferVectors")

    def execute(self, n, n_ener, start_idx, temperature, pressure, partition):
        check(lib().gexs_manager_execute(self.h, n, n_ener, start_idx, temperature, pressure,
                                         partition), "ExecuteCrossSection")

    def transfer_results(self, freq, intens, i):
        check(lib().gexs_manager_transfer_results(self.h, self._p(freq), self._p(intens),
                                                  len(intens), i), "TransferResults")

    def ntrans(self):
        v = C.c_size_t()
        check(lib().gexs_manager_ntrans(self.h, C.byref(v)), "GetNtrans")
        return int(v.value)

    def ready(self):
        v = C.c_int()
        check(lib().gexs_manager_ready(self.h, C.byref(v)), "ReadyForWork")
        return bool(v.value)


class Server:
    """Continuous-batching request loop (include/gexs_serve.h)."""

    def __init__(self, device=0, hbm_budget=0, max_inflight=0, streams=0):
        self.h = C.c_void_p()
        check(lib().gexs_server_create(device, int(hbm_budget), max_inflight, streams,
                                       C.byref(self.h)), "gexs_server_create")

    def close(self):
        if self.h:
            lib().gexs_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _p(a):
        return None if a is None else a.ctypes.data_as(C.c_void_p)

    @staticmethod
    def _any(a):
        if a is None:
            return None
        if hasattr(a, "data_ptr"):
            return C.c_void_p(a.data_ptr())
        return a.ctypes.data_as(C.c_void_p)

    def add_list(self, lines, state_energy, state_g, mass, compact=False):
        """lines: dict of arrays nu, elow, aif, gns[, gamma, n] (numpy host
        arrays or contiguous torch tensors, host or device), or a LineList.
        compact=True keeps the list resident in the 24-byte layout (FP64 nu,
        float E'', g'A, gamma, n; gexs_server_add_lines)."""
        lid = C.c_int()
        se = np.ascontiguousarray(state_energy, dtype=np.float64)
        sg = np.ascontiguousarray(state_g, dtype=np.int32)
        a = self._any
        if compact or isinstance(lines, LineList):
            ll = lines if isinstance(lines, LineList) else LineList(
                lines["nu"], lines["elow"], lines["aif"], lines["gns"], lines.get("gamma"),
                lines.get("n"), compact=True)
            cl = ll.c_lines()
            check(lib().gexs_server_add_lines(self.h, C.byref(cl), a(se), a(sg), len(se),
                                              float(mass), C.byref(lid)), "gexs_server_add_lines")
            return lid.value
        check(lib().gexs_server_add_list(
            self.h, a(lines["nu"]), a(lines["elow"]), a(lines["aif"]), a(lines["gns"]),
            a(lines.get("gamma")), a(lines.get("n")), int(lines["nu"].shape[0]), a(se), a(sg),
            len(se), float(mass), C.byref(lid)), "gexs_server_add_list")
        return lid.value

    @staticmethod
    def request(list_id, profile, temperature, pressure, nu_start, dnu, grid_points,
                precision=capi.FP32, convention=capi.CONV_PHYSICAL, cutoff=-1.0, quad_nodes=16,
                half_width=0.0, ref_temp=296.0, ref_press=1.0):
        return capi.GexsRequest(list_id, profile, precision, convention, quad_nodes, 0,
                                temperature, pressure, nu_start, dnu, int(grid_points), cutoff,
                                half_width, ref_temp, ref_press)

    def submit(self, req):
        t = C.c_uint64()
        st = lib().gexs_server_submit(self.h, C.byref(req), C.byref(t))
        check(st, "gexs_server_submit")
        return t.value

    def try_submit(self, req):
        t = C.c_uint64()
        st = lib().gexs_server_submit(self.h, C.byref(req), C.byref(t))
        return st, t.value

    def wait(self, ticket, grid_points, timeout_ms=-1):
        out = np.empty(int(grid_points), dtype=np.float64)
        info = capi.GexsRequestInfo()
        check(lib().gexs_server_wait(self.h, ticket, timeout_ms, self._p(out), C.byref(info)),
              "gexs_server_wait")
        return out, info

    def wait_status(self, ticket, timeout_ms):
        info = capi.GexsRequestInfo()
        return lib().gexs_server_wait(self.h, ticket, timeout_ms, None, C.byref(info))

    def poll(self, ticket):
        return lib().gexs_server_poll(self.h, ticket)

    def partition(self, list_id, temperature):
        """(Q(T), True when it came from the resident table)"""
        q, tab = C.c_double(), C.c_int()
        check(lib().gexs_server_partition(self.h, list_id, temperature, C.byref(q), C.byref(tab)),
              "gexs_server_partition")
        return q.value, bool(tab.value)

    def stats(self):
        v = [C.c_int64() for _ in range(4)]
        check(lib().gexs_server_stats(self.h, *[C.byref(x) for x in v]), "gexs_server_stats")
        return {"submitted": v[0].value, "completed": v[1].value, "batches": v[2].value,
                "inflight_bytes": v[3].value}

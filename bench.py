#!/usr/bin/env python
"""Cross-section benchmark: Voigt line-profile evaluations per second.

Workload (one step = one cross-section): the Voigt form of the 1e8-line
configuration - 2e5 synthetic states (J 0-80), 1e8 transitions with nu0 in
[100, 30000] cm^-1, pressure broadening gamma_ref ~ U(0.03, 0.1), n ~
U(0.4, 0.8), T_ref 296 K; T = 1500 K, P = 1 bar, 18 amu; grid 100-30000
cm^-1 at 0.01 (2,990,001 points), cutoff 25 cm^-1; FP32 profile
arithmetic with FP64 centres, S(T), Q(T) and Kahan-compensated bins.

value  = line-profile evaluations / s over all ranks (the exact count of
         (line, bin) pairs inside the cutoff window), device time of the
         tile kernel with inputs resident in HBM (4.4 GB of lines > L2);
e2e    = the same through the drop-in manager's C ABI (gexs_manager_*):
         host->device copy of the line list and the grid seed from pinned
         memory, the launch, and the device->host read of the result;
also   = plain FP64 per-(T,P) GPU path on the same workload, the 64-pair
         uneven-grid batch (FP32, one persistent launch replayed from a CUDA
         graph) against the plain FP64 path pair by pair, roofline, the
         reference's own CPU path timed on a bounded sample, and the
         reference's own GPU kernel (built for sm_100a) on a bounded sample
         of the same list against ours on the same lines and bins
         (--no-cpu skips both reference legs).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
import argparse
import faulthandler
import json
import os
import subprocess
import sys
import time

import numpy as np

# a crash in native code prints the Python stack of every thread to stderr
faulthandler.enable()
_T0 = time.perf_counter()


def log(msg):
    """progress on stderr (stdout carries only the JSON line)"""
    sys.stderr.write("[bench %7.1f s] %s\n" % (time.perf_counter() - _T0, msg))
    sys.stderr.flush()

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Voigt line-evals/s @1e8 lines; 64-(T,P) batch vs plain FP64; serve p50/p99"
UNIT = "line-evals/s"
T_K, P_BAR, MASS, CUT = 1500.0, 1.0, 18.0, 25.0
NU0, NU1, DNU = 100.0, 30000.0, 0.01
# Humlicek FLOP per evaluation by region (complex mul 6, add 2, Re-only
# division 7 + 1 divide, Horner step 7; divide, exp and cos count 1 each)
FLOPS_REGION = [15.0, 29.0, 71.0, 113.0]


def grid_points():
    return int(round((NU1 - NU0) / DNU)) + 1


def world():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), \
        int(os.environ.get("LOCAL_RANK", "0"))


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_id):
        self.p = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200",
                                       "-i", dev_id], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "samples": len(sm),
                "reasons": sorted(reasons)}


def device_id_for_smi(torch, dev):
    try:
        return "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v for v in vis.split(",") if v.strip()]
        return ids[dev] if dev < len(ids) else str(dev)


# --------------------------------------------------------- CPU baseline
def gpu_reference_sample(torch, ctx, L, q, dev, k=1_000_000, reps=3):
    """The reference's own GPU path on this B200: GpuManager with the v2 Voigt
    kernel (Managers/Accel/GPU/GPUManager.cpp, compute/CUDA/cross_kernal_v2.cu
    :403-457, one CTA per bin scanning the list), built for sm_100a as
    oracle/_ref/gexsref_gpu, on k consecutive lines around the median nu0 of
    the workload's own list, over the bins within its 100 cm^-1 window.  The
    same lines and grid run through our reference-GPU convention (inclusive
    100 cm^-1 window, the same (line, bin) pairs, counted exactly) in the
    FP32 form; the FP64 form gives the agreement.  A bounded sample: the
    reference kernel's scan grows with lines x bins, so the full list would
    take minutes per pair."""
    from gexs_b200 import Job, LineList, _capi as capi
    from oracle import pyoracle as po
    if not po.ref_gpu_available():
        return {"unavailable": "oracle/_ref/gexsref_gpu not built"}
    n = int(L["nu"].shape[0])
    a = max(0, n // 2 - k // 2)
    b = min(n, a + k)
    S = {kk: v[a:b].cpu().numpy() for kk, v in L.items()}
    lo = float(S["nu"][0]) - 100.0 - 1.0
    nb = int((float(S["nu"][-1]) + 100.0 + 1.0 - lo) / DNU) + 1
    budget = (b - a) * 52 + nb * 16 + (64 << 20)
    sig, ms = po.ref_gpu_voigt(S, lo, DNU, nb, T_K, P_BAR, q, MASS, 296.0, 1.0, 0.0,
                               reps=reps, budget_bytes=budget)
    ref_ms = min(ms[1:]) if len(ms) > 1 else ms[0]
    lines = LineList(*[L[kk][a:b] for kk in ("nu", "elow", "aif", "gns", "gamma", "n")])
    res = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for prec, name in ((capi.FP32, "fp32"), (capi.FP64, "fp64")):
        out = torch.zeros(nb, dtype=torch.float64, device=dev)
        j = Job(lines, out, convention=capi.CONV_REF_GPU, profile=capi.VOIGT, temperature=T_K,
                pressure=P_BAR, partition=q, mass=MASS, nu_start=lo, dnu=DNU, grid_points=nb,
                precision=prec, ref_temp=296.0, ref_press=1.0)
        ctx.run([j])
        ctx.check()
        ts = []
        for _ in range(3):
            e0.record(); ctx.run([j]); e1.record(); e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        o = out.cpu().numpy()
        m = o > 1e-6 * o.max()
        res[name] = {"ms": min(ts),
                     "max_rel_vs_reference": float(np.max(np.abs(sig[m] - o[m]) / o[m]))}
        if prec == capi.FP64:
            evals = ctx.count_evals([j])[0]
    return {"sample": "%d consecutive lines around the median nu0 of the workload's list, "
                      "%d bins (its 100 cm^-1 window), reference-GPU convention" % (b - a, nb),
            "evals": evals, "reference_ms": ref_ms, "reference_evals_per_s": evals / (ref_ms * 1e-3),
            "ours_fp32_ms": res["fp32"]["ms"], "ours_fp32_evals_per_s": evals / (res["fp32"]["ms"] * 1e-3),
            "ours_fp64_ms": res["fp64"]["ms"],
            "speedup_fp32": ref_ms / res["fp32"]["ms"], "speedup_fp64": ref_ms / res["fp64"]["ms"],
            "max_rel_fp64_vs_reference": res["fp64"]["max_rel_vs_reference"],
            "max_rel_fp32_vs_reference": res["fp32"]["max_rel_vs_reference"],
            "reference_build": "reference sources compiled for sm_100a; __shfl_xor mapped to "
                               "__shfl_xor_sync (oracle/ref_gpu_shim.h), nothing else changed"}


def _synth():
    """The numpy workload generator (gexs_b200/synth.py) loaded by file path,
    so the reference arm imports nothing of the gexs_b200 package (whose
    import would map libgexs_b200.so)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "gexs_workload_synth", os.path.join(ROOT, "gexs_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def reference_window_evals(nu, f0, dnu, nb, cut):
    """(line, bin) pairs the reference CPU loop visits: bins [ib, ie) with
    ib = max(round((nu-cut-f0)/dnu), 0), ie = min(round((nu+cut-f0)/dnu), nb)
    (Managers/CPU/OpenMPManager.cpp:399-400; C round, half away from zero),
    for every line (all synthetic A > 0, so no line is skipped at :402)."""
    nu = np.where(nu == 0.0, 1e-6, nu)

    def cround(x):
        return np.copysign(np.floor(np.abs(x) + 0.5), x)
    ib = np.maximum(cround((nu - cut - f0) / dnu), 0.0)
    ie = np.minimum(cround((nu + cut - f0) / dnu), float(nb))
    return int(np.sum(np.maximum(ie - ib, 0.0)))


class ReferenceSample:
    """The reference CPU path (OpenMPManager::ComputeVoigtTP + humlic,
    compiled from the reference sources at -O3 -march=x86-64-v3 into
    oracle/_ref/libgexsref_fast.so; the FP64 port in oracle/ when that
    build is absent) on a bounded sample of the Voigt workload: k
    consecutive lines around the median nu0 of a 2e6-line list with the
    workload's distribution (2e5 states, J 0-80, nu0 100-30000) over the
    bins of their window, all host threads.  The list is generated once; k
    is sized once so that one pass takes about target_s seconds."""

    def __init__(self, target_s, seed_states=1002, seed_lines=2002):
        from oracle import pyoracle as po
        self.po = po
        if not os.path.exists(po.ORACLE_LIB) and not po.ref_available(fast=True):
            po.build(with_reference=False)
        self.kind = "reference" if po.ref_available(fast=True) else "port"
        self.threads = len(os.sched_getaffinity(0))
        sy = _synth()
        st = sy.make_states(200000, 80, seed_states)
        self.L = sy.make_lines(st, 2000000, NU0, NU1, seed_lines, broadening_seed=seed_lines + 1000)
        self.q = (po.ref_partition(st.energy, st.g, T_K, fast=True) if self.kind == "reference"
                  else po.partition(st.energy, st.g, T_K))
        k = 2000
        dt = self._prepare(k)
        while dt < 0.5 and k < len(self.L["nu"]) // 2:
            k *= 4
            dt = self._prepare(k)
        k = int(min(len(self.L["nu"]) - 2, k * max(1.0, target_s / max(dt, 1e-3))))
        self._prepare(k, timed=False)

    def _prepare(self, k, timed=True):
        mid = len(self.L["nu"]) // 2
        sl = slice(mid - k // 2, mid - k // 2 + k)
        self.S = {kk: np.ascontiguousarray(v[sl]) for kk, v in self.L.items()}
        self.lo = float(self.S["nu"][0]) - CUT - 1.0
        self.nb = int((float(self.S["nu"][-1]) + CUT + 1.0 - self.lo) / DNU) + 1
        self.freq = self.lo + np.arange(self.nb, dtype=np.float64) * DNU
        self.k = k
        # reference CPU convention at P = 1 bar: cutoff min(25 P, 100) = 25
        self.evals = reference_window_evals(self.S["nu"], self.lo, DNU, self.nb,
                                            min(25.0 * P_BAR, 100.0))
        return self.run() if timed else 0.0

    def run(self):
        """one pass; returns its wall time in s"""
        t0 = time.perf_counter()
        if self.kind == "reference":
            self.po.ref_voigt_tp(self.freq, self.S, T_K, P_BAR, self.q, MASS, 296.0, DNU,
                                 nthreads=self.threads, fast=True)
        else:
            self.po.cross_section(self._port_job(), nthreads=self.threads)
        return time.perf_counter() - t0

    def _port_job(self):
        from gexs_b200 import _capi as capi
        from gexs_b200.engine import job_init
        from tests.helpers import host_job
        j = job_init(capi.CONV_REF_CPU, capi.VOIGT, T_K, P_BAR, self.q, MASS, self.lo, DNU,
                     self.nb, ref_temp=296.0)
        return host_job(j, self.S)

    def describe(self, dt):
        return ("%d consecutive lines around the median nu0 of a 2e6-line list with the "
                "workload's distribution, %d bins; %.4g evaluations per pass, %.2f s per pass "
                "(reference CPU conventions: HWHM Doppler scaling, cutoff min(25P,100)=25)"
                % (self.k, self.nb, self.evals, dt))


def cpu_reference_sample(target_s=12.0):
    """(evals/s, threads, sample description, kind) of one pass."""
    R = ReferenceSample(target_s)
    dt = R.run()
    return R.evals / dt, R.threads, R.describe(dt), R.kind


def reference_arm(args):
    ws, rank, _ = world()
    if rank != 0:
        return 0
    try:
        from oracle import pyoracle as po
        if not po.ref_available(fast=True) and not os.path.exists(po.ORACLE_LIB):
            po.build(with_reference=False)
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": "CPU checker build failed: %s" % e}))
        return 0
    # the whole run (warm-up + timed passes) stays within about three minutes
    per = max(0.5, min(args.cpu_seconds, 180.0 / (args.steps + args.warmup)))
    R = ReferenceSample(per)
    for _ in range(args.warmup):
        R.run()
    times = [R.run() for _ in range(args.steps)]
    total = float(np.sum(times))
    value = R.evals * args.steps / total
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "Voigt, 1e8-line list distribution, T=1500 K, P=1 bar, "
                                   "0.01 cm^-1 grid, cutoff 25 (bounded CPU sample per step)",
                       "evals_per_step": R.evals, "lines_per_step": R.k,
                       "bins_per_step": R.nb},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": R.threads, "kind": R.kind,
                             "sample": R.describe(total / args.steps)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "timed": "wall clock of each pass of the reference CPU loop on the sample"}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------- our arm
def region_flops(L, q):
    """FLOP per evaluation from the oracle's region histogram on a sample of
    8000 lines (uniform in line index) on the full grid."""
    from gexs_b200 import _capi as capi
    from gexs_b200.engine import job_init
    from oracle import pyoracle as po
    from tests.helpers import host_job
    n = L["nu"].shape[0]
    idx = np.linspace(0, n - 1, 8000).astype(np.int64)
    import torch
    ti = torch.as_tensor(idx, device=L["nu"].device)
    S = {k: np.ascontiguousarray(v[ti].cpu().numpy()) for k, v in L.items()}
    j = job_init(capi.CONV_PHYSICAL, capi.VOIGT, T_K, P_BAR, q, MASS, NU0, DNU, grid_points(),
                 cutoff=CUT)
    hist = np.array(po.region_hist(host_job(j, S)), dtype=np.float64)
    frac = hist / hist.sum()
    return float(np.dot(frac, FLOPS_REGION)), [float(f) for f in frac]


def oracle_subband(torch, L, q, outs, nbins=2000):
    """Error of the device results against the FP64 oracle (oracle/,
    checker only) on `nbins` bins around the median nu0 of the list: the
    oracle evaluates the same job restricted to those bins (start_idx,
    n_points) over the lines that can reach them.  outs: {name: (device
    grid, precision)}."""
    from gexs_b200 import _capi as capi
    from gexs_b200.engine import job_init
    from oracle import pyoracle as po
    from tests.helpers import host_job, fp32_errors
    nu = L["nu"]
    mid = float(nu[nu.shape[0] // 2])
    j0 = int(round((mid - NU0) / DNU)) - nbins // 2
    fa, fb = NU0 + j0 * DNU, NU0 + (j0 + nbins - 1) * DNU
    a = int(torch.searchsorted(nu, torch.tensor(fa - CUT - 1.0, dtype=nu.dtype, device=nu.device)))
    b = int(torch.searchsorted(nu, torch.tensor(fb + CUT + 1.0, dtype=nu.dtype, device=nu.device)))
    S = {k: np.ascontiguousarray(v[a:b].cpu().numpy()) for k, v in L.items()}
    j = job_init(capi.CONV_PHYSICAL, capi.VOIGT, T_K, P_BAR, q, MASS, NU0, DNU, grid_points(),
                 cutoff=CUT)
    j.start_idx, j.n_points = j0, nbins
    ref = po.cross_section(host_job(j, S), nthreads=len(os.sched_getaffinity(0)))[j0:j0 + nbins]
    res = {"bins": nbins, "lines": b - a, "nu_range": [fa, fb]}
    for name, (o, prec) in outs.items():
        got = o[j0:j0 + nbins].cpu().numpy()
        if prec == capi.FP64:
            res[name + "_max_rel_vs_oracle"] = float(np.max(np.abs(got - ref) / np.abs(ref)))
        else:
            rel, band = fp32_errors(got, ref)
            res[name + "_max_rel_vs_oracle_bins_gt_1e-6_peak"] = rel
            res[name + "_band_rel_vs_oracle"] = band
    return res


def batch64(ctx, torch, dev):
    """The 64-(T,P) uneven-grid batch over the 1e6-line list: FP32 batched
    (autotuned, graph-replayed persistent launch) vs plain FP64 per pair."""
    from gexs_b200 import synth, _capi as capi
    from gexs_b200.engine import Job, LineList
    st = synth.make_states(20000, 40, 1001)
    L = synth.make_lines(st, 1000000, NU0, 10000.0, 2001, broadening_seed=3001)
    lines = LineList.from_dict(L, device=dev)
    se = torch.as_tensor(st.energy, device=dev)
    sg = torch.as_tensor(st.g, device=dev)
    temps = np.logspace(np.log10(100.0), np.log10(3000.0), 8)
    press = np.logspace(-5.0, 2.0, 8)
    rng = np.random.Generator(np.random.PCG64(4003))
    dnus = rng.choice([0.1, 0.01, 0.005], size=64)
    qs = ctx.partition(se, sg, np.repeat(temps, 8))
    j32, j64 = [], []
    for i in range(64):
        T, P, d = temps[i // 8], press[i % 8], float(dnus[i])
        G = int(round((30000.0 - NU0) / d)) + 1
        kw = dict(convention=capi.CONV_PHYSICAL, profile=capi.VOIGT, temperature=T, pressure=P,
                  partition=float(qs[i]), mass=MASS, nu_start=NU0, dnu=d, grid_points=G,
                  cutoff=CUT)
        j32.append(Job(lines, torch.zeros(G, dtype=torch.float64, device=dev),
                       precision=capi.FP32, **kw))
        j64.append(Job(lines, torch.zeros(G, dtype=torch.float64, device=dev),
                       precision=capi.FP64, **kw))
    evals = sum(ctx.count_evals(j32))
    cfg, tune_ms = ctx.autotune(j32)
    b = ctx.batch(j32, cfg)
    s = torch.cuda.Stream(device=dev)
    b.capture(s)
    b.replay(s)
    s.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t32 = []
    for _ in range(2):
        e0.record(s); b.replay(s); e1.record(s); e1.synchronize()
        t32.append(e0.elapsed_time(e1))
    ctx.check(s)
    cur = torch.cuda.current_stream(dev)
    ctx.run(j64[:1])
    ctx.check()
    e0.record(cur)
    for j in j64:
        ctx.run([j], stream=cur)
    e1.record(cur)
    e1.synchronize()
    ctx.check()
    t64 = e0.elapsed_time(e1)
    worst, band = 0.0, 0.0
    for a, c in zip(j32, j64):
        x, r = a.out, c.out
        pk = float(r.max())
        if pk <= 0:
            continue
        m = r > 1e-6 * pk
        worst = max(worst, float(((x[m] - r[m]).abs() / r[m]).max()))
        band = max(band, abs(float(x.sum()) - float(r.sum())) / float(r.sum()))
    b.close()
    return {"pairs": 64, "lines": lines.count, "evals": evals,
            "fp32_batched_ms": min(t32), "fp64_plain_ms": t64, "speedup": t64 / min(t32),
            "fp32_evals_per_s": evals / (min(t32) * 1e-3),
            "max_rel_err_vs_fp64": worst, "max_band_err_vs_fp64": band,
            "launch_cfg": {"bins_per_lane": cfg[0], "warps": cfg[1],
                           "long_stages": bool(len(cfg) > 3 and cfg[3] & capi.LAUNCH_LONG_STAGES)},
            "grids": {"0.1": int(np.sum(dnus == 0.1)), "0.01": int(np.sum(dnus == 0.01)),
                      "0.005": int(np.sum(dnus == 0.005))}}


def batch_64_pairs_full_list(ctx, torch, dev, lines, st, fpe, fp64_peak, cfg):
    """64 (T, P) cross-sections of the 1e8-line list on the 2,990,001-bin grid
    (T log-spaced 100-3000 K x P log-spaced 1e-5-100 bar, 0.01 cm^-1 over
    100-30000, cutoff 25): the FP32 form as one batch (gexs_batch, lines
    derived on load: prep arrays for 64 pairs would take 154 GB) captured in
    a CUDA graph and replayed, timed with CUDA events on its stream; the
    plain FP64 form one launch per pair on the 8 pairs (T_i, P_i) of the
    diagonal, its time per evaluation scaled to the 64 pairs' evaluations,
    with the FP32 form's error against it on those 8 pairs."""
    from gexs_b200 import _capi as capi
    from gexs_b200.engine import Job
    temps = np.logspace(np.log10(100.0), np.log10(3000.0), 8)
    press = np.logspace(-5.0, 2.0, 8)
    qs = ctx.partition(torch.as_tensor(st.energy, device=dev),
                       torch.as_tensor(st.g, dtype=torch.int32, device=dev), np.repeat(temps, 8))
    G = grid_points()
    kw = dict(convention=capi.CONV_PHYSICAL, profile=capi.VOIGT, mass=MASS, nu_start=NU0, dnu=DNU,
              grid_points=G, cutoff=CUT)
    j32 = [Job(lines, torch.zeros(G, dtype=torch.float64, device=dev), precision=capi.FP32,
               temperature=float(temps[i // 8]), pressure=float(press[i % 8]),
               partition=float(qs[i]), **kw) for i in range(64)]
    evals = sum(ctx.count_evals(j32))
    # lines derived on load load the producers more: the 4-stage ring of
    # 128-line stages serves this batch better (13.00 s against 13.16 s with
    # 256-line stages, measured on one B200)
    bcfg = tuple(cfg[:3]) + (capi.LAUNCH_DERIVE_ON_LOAD,) + tuple(cfg[4:])
    b = ctx.batch(j32, bcfg)
    s = torch.cuda.Stream(device=dev)
    b.capture(s)
    b.replay(s)
    s.synchronize()
    ctx.check(s)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    b.replay(s)
    e1.record(s)
    e1.synchronize()
    ctx.check(s)
    t32 = e0.elapsed_time(e1)
    b.close()
    diag = [i * 8 + i for i in range(8)]
    cur = torch.cuda.current_stream(dev)
    out64 = torch.zeros(G, dtype=torch.float64, device=dev)
    worst, band, t64, ev64 = 0.0, 0.0, 0.0, 0
    for n, i in enumerate(diag):
        j = Job(lines, out64, precision=capi.FP64, temperature=float(temps[i // 8]),
                pressure=float(press[i % 8]), partition=float(qs[i]), **kw)
        if n == 0:
            ctx.run([j], stream=cur)
            ctx.check(cur)
        e0.record(cur); ctx.run([j], stream=cur); e1.record(cur); e1.synchronize()
        ctx.check(cur)
        t64 += e0.elapsed_time(e1)
        ev64 += ctx.count_evals([j])[0]
        x, r = j32[i].out, out64
        m = r > 1e-6 * float(r.max())
        worst = max(worst, float(((x[m] - r[m]).abs() / r[m]).max()))
        band = max(band, abs(float(x.sum()) - float(r.sum())) / float(r.sum()))
    t64_all = t64 * evals / ev64
    del j32
    torch.cuda.empty_cache()
    fp64_tf = fpe * ev64 / (t64 * 1e-3) / 1e12
    return {"pairs": 64, "lines": lines.count, "grid_points": G, "evals": evals,
            "fp32_batched_ms": t32, "fp32_evals_per_s": evals / (t32 * 1e-3),
            "fp64_plain_ms_8_pairs": t64, "fp64_plain_ms_64_pairs_scaled": t64_all,
            "speedup": t64_all / t32,
            "max_rel_err_vs_fp64_8_pairs": worst, "max_band_err_vs_fp64_8_pairs": band,
            "fp64_roofline": {"achieved_tflops": fp64_tf, "peak_tflops": fp64_peak,
                              "frac": fp64_tf / fp64_peak if fp64_peak else None,
                              "flop_per_eval": fpe,
                              "peak_source": "measured FP64 FMA rate (gexs_probe_fp64_tflops)"},
            "launch_cfg": list(bcfg),
            "fp64_scaling": "time per evaluation of the 8 diagonal pairs times the 64 pairs' "
                            "evaluations (every pair has the same window, so the same count)"}


def serve_bench(torch, dev, local_rank, args):
    """Request loop under Poisson arrivals (continuous batching).

    Three resident synthetic lists of 1e7, 1e8 and 5e8 lines times
    --serve-scale (18, 16, 44 amu; generated as the 1e8-line workload, the
    largest from 1e6 states J 0-120), kept in the compact layout (FP64 nu0,
    float E'', g'A, gamma, n: 24 B per line).  One seeded set of --serve-requests
    requests is used for every rate: list uniform, T log-U(100, 3000) K, P
    log-U(1e-6, 100) bar, dnu log-U(0.001, 0.1) cm^-1, 1e4-1e7 points (at
    most the span 100-20000 allows), start uniform in 100-20000 minus the
    span, Doppler or Voigt, FP32 form.  The set is first run one request at
    a time; its mean service time s sets the rate of offered load L as L/s.
    It is then submitted all at once, untimed, so that the server's memory
    pool has grown to what its budget admits before any timed rate.
    Per rate the same set arrives as a Poisson stream; each request has its
    own waiter, so a result is fetched as soon as it is done.  latency =
    result copied into the caller's buffer minus submission (device done
    minus submission also given); throughput = requests / (last fetch -
    first submission)."""
    import threading
    from gexs_b200 import synth, _capi as capi
    from gexs_b200.engine import Server, Context, Job, LineList
    scale = args.serve_scale
    specs = [(int(1e7 * scale), 18.0, 1), (int(1e8 * scale), 16.0, 2), (int(5e8 * scale), 44.0, 3)]
    srv = Server(local_rank, hbm_budget=0, streams=4)
    keep, lists = [], []
    t_gen = time.perf_counter()
    for n, mass, k in specs:
        big = k == 3
        st = synth.make_states(1000000 if big else 200000, 120 if big else 80, 1010 + k)
        L = synth.make_lines_torch(st, n, NU0, NU1, 2010 + k, broadening_seed=3010 + k, device=dev)
        lid = srv.add_list(L, st.energy, st.g, mass, compact=True)
        keep.append(LineList(L["nu"], L["elow"], L["aif"], L["gns"], L["gamma"], L["n"], device=dev))
        lists.append((lid, mass, n))
        del L
        torch.cuda.empty_cache()
    t_gen = time.perf_counter() - t_gen
    rng = np.random.Generator(np.random.PCG64(4000))

    def draw():
        li = int(rng.integers(0, 3))
        T = float(10 ** rng.uniform(2.0, np.log10(3000.0)))
        P = float(10 ** rng.uniform(-6.0, 2.0))
        d = float(10 ** rng.uniform(-3.0, -1.0))
        G = int(10 ** rng.uniform(4.0, 7.0))
        G = min(G, int(19900.0 / d))
        nu0 = float(rng.uniform(100.0, 20000.0 - G * d))
        prof = capi.VOIGT if rng.random() < 0.5 else capi.DOPPLER
        return li, Server.request(lists[li][0], prof, T, P, nu0, d, G, precision=capi.FP32,
                                  cutoff=CUT)

    reqs = [draw() for _ in range(args.serve_requests)]
    # evaluations of the request set, counted on the generated copies, which
    # are then freed: the server's budget (0.9 of the memory free when it was
    # created) must not also cover them
    ctx = Context(local_rank)
    ev = 0
    for li, rq in reqs:
        j = Job(keep[li], torch.empty(1, dtype=torch.float64, device=dev),
                convention=capi.CONV_PHYSICAL, profile=rq.profile, temperature=rq.temperature,
                pressure=rq.pressure, partition=1.0, mass=lists[li][1], nu_start=rq.nu_start,
                dnu=rq.dnu, grid_points=rq.grid_points, cutoff=CUT, n_points=rq.grid_points)
        ev += ctx.count_evals([j])[0]
    del keep, ctx, j
    torch.cuda.empty_cache()

    def run(rate, seed):
        n = len(reqs)
        lat, dlat, infos = [0.0] * n, [0.0] * n, [None] * n
        errors = []

        def waiter(i, ticket, G):
            try:
                _, info = srv.wait(ticket, G)
                lat[i] = info.fetched_ms - info.submit_ms
                dlat[i] = info.done_ms - info.submit_ms
                infos[i] = info
            except Exception as e:  # pragma: no cover
                errors.append(str(e))
        r2 = np.random.Generator(np.random.PCG64(seed))
        gaps = r2.exponential(1.0 / rate, n) if rate else np.zeros(n)
        threads = []
        t0 = time.perf_counter()
        due = t0
        for i, (_, rq) in enumerate(reqs):
            due += float(gaps[i])
            dt = due - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            th = threading.Thread(target=waiter, args=(i, srv.submit(rq), rq.grid_points))
            th.start()
            threads.append(th)
        for th in threads:
            th.join()
        wall = time.perf_counter() - t0
        if len(errors) == n:
            raise RuntimeError(errors[0])
        ok = [i for i in range(n) if infos[i] is not None]
        return (wall, np.array([lat[i] for i in ok]), np.array([dlat[i] for i in ok]),
                [infos[i] for i in ok], errors)

    log("serving: %d requests, serial pass" % len(reqs))
    # warm-up (module loads, pools), then the set one request at a time
    for _, rq in reqs[:3]:
        srv.wait(srv.submit(rq), rq.grid_points)
    t0 = time.perf_counter()
    for _, rq in reqs:
        srv.wait(srv.submit(rq), rq.grid_points)
    service = (time.perf_counter() - t0) / len(reqs)
    # the whole set at once, untimed: the memory pool grows to what the
    # budget admits at a time, so no timed rate pays for mapping new pages
    for t_, (_, rq) in [(srv.submit(rq), (li, rq)) for li, rq in reqs]:
        srv.wait(t_, rq.grid_points)
    rates = []
    for k, load in enumerate(args.serve_loads):
        rate = load / service
        log("serving: offered load %.2f" % load)
        wall, lat, dlat, infos, errors = run(rate, 4100 + k)
        rates.append({"offered_load": load, "offered_req_per_s": rate, "requests": len(reqs),
                      "failed": len(errors), "first_error": errors[0] if errors else None,
                      "p50_ms": float(np.percentile(lat, 50)),
                      "p99_ms": float(np.percentile(lat, 99)),
                      "mean_ms": float(lat.mean()),
                      "device_done_p50_ms": float(np.percentile(dlat, 50)),
                      "device_done_p99_ms": float(np.percentile(dlat, 99)),
                      "throughput_req_per_s": len(infos) / wall,
                      "evals_per_s": ev / wall if not errors else None,
                      "mean_batch": float(np.mean([i.batch_size for i in infos])),
                      "max_batch": int(max(i.batch_size for i in infos))})
    stats = srv.stats()
    srv.close()
    return {"lists": [{"lines": n, "mass_amu": m} for _, m, n in lists],
            "list_layout": "resident compact: FP64 nu0 + float E'', g'A, gamma, n (24 B/line), "
                           "%.1f GB of lines" % (24.0 * sum(n for _, _, n in lists) / 1e9),
            "list_scale": scale, "list_generation_s": t_gen,
            "serial_service_ms": 1e3 * service, "evals_per_request_set": ev,
            "rates": rates, "batches": stats["batches"],
            "requests": "one seeded set of %d for every rate: T log-U(100,3000) K, P "
                        "log-U(1e-6,100) bar, dnu log-U(0.001,0.1), 1e4-1e7 points in "
                        "100-20000 cm^-1, Doppler|Voigt, FP32 form" % len(reqs),
            "latency": "result in the caller's buffer minus submission; one waiter per request"}


def quad_suite(args):
    """Voigt-Quad against Humlicek on the 5e8-line list (resident compact:
    FP64 nu0, float E'', g'A, gamma, n): 1e6 states (J 0-120),
    nu0 10-20000 cm^-1, T = 2500 K, P = 1e-3, 1, 100 bar, 0.01 cm^-1 over
    10-20000 (1,999,001 points), cutoff 25, FP32 form timed per
    (P, method); errors of the FP32 form against the FP64 form of the same
    quadrature (which matches the CPU oracle to 1e-10) and of GH against
    Humlicek, on a 20 cm^-1 sub-band at 5000 cm^-1."""
    import torch
    from gexs_b200 import Context, Job, LineList, synth, _capi as capi
    from oracle import pyoracle as po
    dev = "cuda:0"
    torch.cuda.set_device(0)
    n = args.quad_lines
    st = synth.make_states(1000000, 120, 1004)
    L = synth.make_lines_torch(st, n, 10.0, 20000.0, 2004, broadening_seed=3004, device=dev)
    # resident as the configuration states: FP64 nu0, float E'', g'A, gamma, n (24 B/line)
    lines = LineList(L["nu"], L["elow"], L["aif"], L["gns"], L["gamma"], L["n"], device=dev,
                     compact=True)
    del L
    torch.cuda.empty_cache()
    T = 2500.0
    ctx = Context(0)
    q = float(ctx.partition(torch.as_tensor(st.energy, device=dev),
                            torch.as_tensor(st.g, dtype=torch.int32, device=dev), [T])[0])
    nu0, d = 10.0, 0.01
    G = int(round((20000.0 - nu0) / d)) + 1
    out = torch.zeros(G, dtype=torch.float64, device=dev)
    ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sub0 = int(round((5000.0 - nu0) / d))
    res = []
    for P in (1e-3, 1.0, 100.0):
        row = {"pressure_bar": P}
        subs = {}
        for name, prof, nodes in (("humlicek", capi.VOIGT, 16), ("gh16", capi.VOIGT_QUAD, 16),
                                  ("gh32", capi.VOIGT_QUAD, 32)):
            kw = dict(convention=capi.CONV_PHYSICAL, profile=prof, temperature=T, pressure=P,
                      partition=q, mass=18.0, nu_start=nu0, dnu=d, grid_points=G, cutoff=CUT,
                      quad_nodes=nodes)
            j = Job(lines, out, precision=capi.FP32, **kw)
            evals = ctx.count_evals([j])[0]
            ctx.run([j]); ctx.check()
            ev[0].record(); ctx.run([j]); ev[1].record(); ev[1].synchronize()
            ms = ev[0].elapsed_time(ev[1])
            row[name] = {"ms": ms, "evals_per_s": evals / (ms * 1e-3)}
            o32 = torch.zeros(G, dtype=torch.float64, device=dev)
            o64 = torch.zeros(G, dtype=torch.float64, device=dev)
            for o, prec in ((o32, capi.FP32), (o64, capi.FP64)):
                js = Job(lines, o, precision=prec, start_idx=sub0, n_points=2000, **kw)
                ctx.run([js])
            ctx.check()
            a, b = o32[sub0:sub0 + 2000], o64[sub0:sub0 + 2000]
            m = b > 1e-6 * b.max()
            row[name]["fp32_max_rel_vs_fp64"] = float(((a[m] - b[m]).abs() / b[m]).max())
            subs[name] = b
        h = subs["humlicek"]
        m = h > 1e-6 * h.max()
        for g in ("gh16", "gh32"):
            row[g]["max_rel_vs_humlicek_fp64"] = float(((subs[g][m] - h[m]).abs() / h[m]).max())
        row["evals_per_pass"] = evals
        res.append(row)
    return {"lines": lines.count, "grid_points": G, "temperature": T, "rows": res}


def order_suite(args):
    """Work-item order of a batch: --order-pairs (T, P) pairs (T log-spaced
    100-3000 K x P log-spaced 1e-5-100 bar) of the --lines list on the
    2,990,001-bin grid, FP32 Voigt with lines derived on load, launched with
    items tile-major (the default) and job-major (GEXS_LAUNCH_JOB_MAJOR).
    Default: each order as a graph-captured batch, one warm replay and
    --steps timed replays (CUDA events), and whether the grids are bitwise
    equal.  --order-plain: two plain launches per order (tile, job, tile,
    job) and nothing timed, for an ncu capture of the last two."""
    import torch
    from gexs_b200 import Context, Job, LineList, synth, _capi as capi
    dev = "cuda:0"
    torch.cuda.set_device(0)
    st = synth.make_states(200000, 80, 1002)
    L = synth.make_lines_torch(st, args.lines, NU0, NU1, 2002, broadening_seed=3002, device=dev)
    lines = LineList(L["nu"], L["elow"], L["aif"], L["gns"], L["gamma"], L["n"], device=dev)
    ctx = Context(0)
    n = args.order_pairs
    k = next(d for d in range(int(np.sqrt(n)), 0, -1) if n % d == 0)
    temps = np.logspace(np.log10(100.0), np.log10(3000.0), k)
    press = np.logspace(-5.0, 2.0, n // k)
    qs = ctx.partition(torch.as_tensor(st.energy, device=dev),
                       torch.as_tensor(st.g, dtype=torch.int32, device=dev), np.repeat(temps, n // k))
    G = grid_points()

    def jobs():
        return [Job(lines, torch.zeros(G, dtype=torch.float64, device=dev),
                    convention=capi.CONV_PHYSICAL, profile=capi.VOIGT,
                    temperature=float(temps[i // (n // k)]), pressure=float(press[i % (n // k)]),
                    partition=float(qs[i]), mass=MASS, nu_start=NU0, dnu=DNU, grid_points=G,
                    precision=capi.FP32, cutoff=CUT) for i in range(n)]

    flags = capi.LAUNCH_DERIVE_ON_LOAD
    orders = (("tile_major", (4, 4, 0, flags)), ("job_major", (4, 4, 0, flags | capi.LAUNCH_JOB_MAJOR)))
    res = {"suite": "order", "pairs": n, "lines": args.lines, "grid_points": G,
           "launch_cfg": [4, 4, 0, flags]}
    if args.order_plain:
        J = jobs()
        for _ in range(2):
            for _, c in orders:
                ctx.run(J, cfg=c)
        ctx.check()
        torch.cuda.synchronize()
        return res
    first = None
    for name, c in orders:
        J = jobs()
        b = ctx.batch(J, c)
        s = torch.cuda.Stream(device=dev)
        b.capture(s)
        b.replay(s)
        s.synchronize()
        ctx.check(s)
        ts = []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            b.replay(s)
            e1.record(s)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        ctx.check(s)
        b.close()
        res[name + "_ms"] = ts
        if first is None:
            first = [j.out for j in J]
        else:
            res["bitwise_equal"] = all(torch.equal(x, j.out) for x, j in zip(first, J))
        del J
    return res


def ingest_suite(args):
    """ExoMol ingest: seeded .states (2e5 states, J 0-80) and .trans (the
    --ingest-lines transitions, 30-7000 cm^-1) text in the ExoMol layout,
    parsed on the GPU from host bytes (gexs_exomol_parse_states/trans: H2D
    copy, newline index, parse, state lookup, stable nu sort), against the
    reference's own ExomolStateReader (compiled from its sources) on a
    bounded sample of the same file, single-threaded as in the reference."""
    import subprocess
    import tempfile
    import torch
    from gexs_b200 import Context, synth
    from gexs_b200.engine import parse_exomol
    from oracle import pyoracle as po
    st = synth.make_states(200000, 80, 1006)
    u, l, a = synth.make_exomol_transitions(st, args.ingest_lines, 30.0, 7000.0, 2006)
    stext = synth.exomol_states_text(st)
    ttext = synth.exomol_trans_text(u, l, a)
    ctx = Context(0)
    parse_exomol(ctx, stext, ttext[:1 << 20].rsplit(b"\n", 1)[0] + b"\n")   # warm-up
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S, L = parse_exomol(ctx, stext, ttext, sort_by_nu=True)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    n = int(L["nu"].numel())
    best = min(times)
    res = {"suite": "ingest", "transitions": n, "states": len(st.energy),
           "text_bytes": len(ttext) + len(stext), "gpu_s": best,
           "gpu_lines_per_s": n / best, "gpu_text_gbs": (len(ttext) + len(stext)) / best / 1e9,
           "timed": "host bytes -> device text -> sorted device line table, wall clock with "
                    "device syncs (includes the H2D copy of the text)"}
    if po.ref_reader_available():
        k = min(n, 2_000_000)
        cut = ttext[:k * (len(ttext) // max(len(u), 1))]
        cut = cut[:cut.rfind(b"\n") + 1]
        with tempfile.TemporaryDirectory() as td:
            sp, tp = os.path.join(td, "s.states"), os.path.join(td, "s.trans")
            open(sp, "wb").write(stext)
            open(tp, "wb").write(cut)
            t0 = time.perf_counter()
            subprocess.run([po.REF_READER_BIN, sp, tp, "-", "0.1", "0.1", os.path.join(td, "o")],
                           check=True, stdout=subprocess.DEVNULL)
            dt = time.perf_counter() - t0
        nref = cut.count(b"\n")
        res["reference_cpu"] = {"lines_per_s": nref / dt, "lines": nref, "s": dt, "threads": 1,
                                "note": "states load + transition stream of the reference reader, "
                                        "one process (the reference reads on one thread)"}
        res["speedup_vs_reference"] = res["gpu_lines_per_s"] / res["reference_cpu"]["lines_per_s"]
    return res


def e2e_manager(torch, dev, L, q, steps, warmup, local_rank):
    """Same workload through the drop-in manager's C ABI with host buffers."""
    from gexs_b200 import _capi as capi
    from gexs_b200.engine import Manager
    G = grid_points()
    n = int(L["nu"].shape[0])
    pin = {k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True) for k, v in L.items()}
    for k in pin:
        pin[k].copy_(L[k])
    h = {k: v.numpy() for k, v in pin.items()}
    freq = NU0 + np.arange(G, dtype=np.float64) * DNU
    zeros = torch.zeros(G, dtype=torch.float64, pin_memory=True).numpy()
    res = torch.zeros(G, dtype=torch.float64, pin_memory=True).numpy()
    lb = sum(v.numel() * v.element_size() for v in pin.values())
    m = Manager(capi.VOIGT, device=local_rank, convention=capi.CONV_PHYSICAL, precision=capi.FP32,
                memory_bytes=lb + 2 * G * 8 + (256 << 20))
    m.initialize_vectors(G, 1)
    m.initialize_constants(0.0, T_K, q, DNU, MASS, P_BAR, 296.0, 1.0)
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        m.transfer_freq(freq, zeros)
        m.transfer_vectors(h["elow"], h["nu"], h["aif"], h["gns"], h["gamma"], h["n"])
        m.execute(G, n, 0, T_K, P_BAR, q)
        m.transfer_results(freq, res, 0)
        if i >= warmup:
            times.append(time.perf_counter() - t0)
    m.close()
    return float(np.sum(times)), lb + G * 8, G * 8, res.copy()


def our_arm(args):
    import torch
    ws, rank, local_rank = world()
    dist = None
    if ws > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = "cuda:%d" % local_rank
    torch.cuda.set_device(local_rank)
    from gexs_b200 import Context, Job, LineList, synth, _capi as capi

    log("generating the %d-line list" % args.lines)
    st = synth.make_states(200000, 80, 1002)
    L = synth.make_lines_torch(st, args.lines, NU0, NU1, 2002, broadening_seed=3002, device=dev)
    lines = LineList(L["nu"], L["elow"], L["aif"], L["gns"], L["gamma"], L["n"], device=dev)
    G = grid_points()
    out = torch.zeros(G, dtype=torch.float64, device=dev)
    ctx = Context(local_rank)
    # Q(T) by the product's own device reduction (gexs_partition)
    q = float(ctx.partition(torch.as_tensor(st.energy, device=dev),
                            torch.as_tensor(st.g, dtype=torch.int32, device=dev), [T_K])[0])
    start_idx, n_points = 0, G
    if args.shard == "grid" and ws > 1:
        from gexs_b200 import shard
        start_idx, n_points = shard.balanced_slices(L["nu"].cpu().numpy(), NU0, DNU, G, CUT,
                                                    ws)[rank]
    job = Job(lines, out, convention=capi.CONV_PHYSICAL, profile=capi.VOIGT, temperature=T_K,
              pressure=P_BAR, partition=q, mass=MASS, nu_start=NU0, dnu=DNU, grid_points=G,
              precision=capi.FP32, cutoff=CUT, start_idx=start_idx, n_points=n_points)
    evals = ctx.count_evals([job])[0]
    evals_full = evals
    if (start_idx, n_points) != (0, G):
        jf = Job(lines, out, convention=capi.CONV_PHYSICAL, profile=capi.VOIGT, temperature=T_K,
                 pressure=P_BAR, partition=q, mass=MASS, nu_start=NU0, dnu=DNU, grid_points=G,
                 precision=capi.FP32, cutoff=CUT)
        evals_full = ctx.count_evals([jf])[0]
    cfg, _ = ctx.autotune([job]) if args.autotune else \
        (tuple(int(v) for v in args.cfg.split(",")), 0.0)
    stream = torch.cuda.current_stream(dev)

    log("warm-up")
    for _ in range(args.warmup):
        ctx.run([job], cfg=cfg, stream=stream)
    ctx.check(stream)
    sampler = ClockSampler(device_id_for_smi(torch, local_rank))
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ctx.run([job], cfg=cfg, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    ctx.check(stream)
    ms = e0.elapsed_time(e1)
    ms_max, evals_all = ms, evals
    if dist:
        from gexs_b200 import shard
        ms_max = shard.max_over_ranks(dist, ms, device=dev)
        evals_all = shard.sum_over_ranks(dist, evals, device=dev)
    value = evals_all * args.steps / (ms_max * 1e-3)
    launch_ms = ms / args.steps

    log("timed region done; plain FP64 path")
    # plain FP64 per-(T,P) path on the same workload
    out64 = torch.zeros(G, dtype=torch.float64, device=dev)
    j64 = Job(lines, out64, convention=capi.CONV_PHYSICAL, profile=capi.VOIGT, temperature=T_K,
              pressure=P_BAR, partition=q, mass=MASS, nu_start=NU0, dnu=DNU, grid_points=G,
              precision=capi.FP64, cutoff=CUT)
    ctx.run([j64], stream=stream)
    ctx.check(stream)
    e0.record(stream); ctx.run([j64], stream=stream); e1.record(stream); e1.synchronize()
    fp64_ms = e0.elapsed_time(e1)
    pk = float(out64.max())
    msk = out64 > 1e-6 * pk
    fp32_err = float(((out[msk] - out64[msk]).abs() / out64[msk]).max())
    band_err = abs(float(out.sum()) - float(out64.sum())) / float(out64.sum())
    integral = float(out64.sum()) * DNU
    vs_oracle = None
    if rank == 0 and not args.no_cpu and (start_idx, n_points) == (0, G):
        log("oracle sub-band")
        vs_oracle = oracle_subband(torch, L, q, {"fp32": (out, capi.FP32),
                                                 "fp64": (out64, capi.FP64)})
    del out64, j64

    log("e2e through the manager")
    # e2e through the manager C ABI, host buffers
    e2e_s, h2d, d2h, e2e_res = e2e_manager(torch, dev, L, q, args.steps, min(args.warmup, 1),
                                           local_rank)
    e2e_match = float(np.max(np.abs(e2e_res - out.cpu().numpy())) / max(pk, 1e-300))
    e2e_max = e2e_s
    if dist:
        e2e_max = shard.max_over_ranks(dist, e2e_s, device=dev)
    # the manager computes one full cross-section per rank
    e2e_value = evals_full * ws * args.steps / e2e_max

    result = None
    if rank == 0:
        log("probes and FLOP accounting")
        peak = 0.0
        import ctypes as C
        from gexs_b200._capi import lib
        pv = C.c_double()
        if lib().gexs_probe_fp32_tflops(local_rank, C.byref(pv)) == 0:
            peak = pv.value
        peak64 = None
        if lib().gexs_probe_fp64_tflops(local_rank, C.byref(pv)) == 0:
            peak64 = pv.value
        rcp = None
        if lib().gexs_probe_rcp_gops(local_rank, C.byref(pv)) == 0:
            rcp = pv.value
        fpe, frac = region_flops(L, q)
        achieved = evals * fpe / (launch_ms * 1e-3) / 1e12
        line_bytes = lines.nbytes()
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic_voigt_fp32.json")
        if os.path.exists(tp):
            try:
                traffic = json.load(open(tp)).get("bytes_per_launch_scaled")
            except Exception:
                traffic = None
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong" if (args.shard == "grid" and ws > 1) else "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "Voigt FP32-profile cross-section, 1e8-line synthetic list "
                                   "(2e5 states, J 0-80, nu0 100-30000), T=1500 K, P=1 bar, "
                                   "grid 100-30000 @0.01 (2,990,001 pts), cutoff 25",
                       "lines": lines.count, "grid_points": G, "evals_per_step": evals,
                       "per_rank": ("a line-density-balanced slice of one cross-section"
                                    if (args.shard == "grid" and ws > 1)
                                    else "one full cross-section per rank"),
                       "parallelism": "replicas x%d" % ws if args.shard != "grid" else
                                      "grid-slices x%d" % ws,
                       "l2": "inputs (%.1f GB of lines) larger than L2" % (line_bytes / 1e9),
                       "launch_cfg": {"bins_per_lane": cfg[0], "warps": cfg[1],
                                      "long_stages": bool(len(cfg) > 3 and
                                                          cfg[3] & capi.LAUNCH_LONG_STAGES)}},
            # per step: put_blob_kernel (launch table), prep_kernel (S(T),
            # width, y per line), slice_plan_kernel and slice_scan_kernel
            # (line slices), voigt_ws_kernel (region I), zero_ints_kernel
            # (core work counter), core_slice_plan_kernel and
            # slice_scan_kernel (core slices), core_kernel (regions II-IV)
            "gpu_launches": 9 * args.steps,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                         "traffic": traffic,
                         "peak_source": "measured FP32 FMA rate of this GPU "
                                        "(gexs_probe_fp32_tflops); MEASURED_PEAKS.json has "
                                        "no FP32 figure",
                         "flop_per_eval": fpe, "region_fractions": frac,
                         "launch_ms": launch_ms,
                         "timed": "one cross-section per step: prep_kernel + voigt_ws_kernel "
                                  "(region I) + core_kernel (regions II-IV), CUDA events on "
                                  "the launching stream; per-kernel shares in the ncu launch "
                                  "list under profiles/",
                         "line_stream_gbs": line_bytes / (launch_ms * 1e-3) / 1e9,
                         "fp64_peak_tflops": peak64,
                         "mufu": {"rcp_gops_measured": rcp,
                                  "region1_evals_per_s": evals * frac[0] / (launch_ms * 1e-3),
                                  "frac": (evals * frac[0] / (launch_ms * 1e-3)) / (rcp * 1e9)
                                          if rcp else None,
                                  "note": "region I takes one MUFU reciprocal per evaluation; "
                                          "frac = its evaluations/s over the measured "
                                          "rcp.approx.f32 rate"}},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "path": "gexs_manager_* C ABI, pinned host",
                    "max_abs_diff_vs_device_run_over_peak": e2e_match},
            "fp64_plain": {"ms": fp64_ms, "evals_per_s": evals / (fp64_ms * 1e-3),
                           "fp32_speedup": fp64_ms / launch_ms,
                           "roofline_frac": (evals * fpe / (fp64_ms * 1e-3) / 1e12) / peak64
                           if peak64 else None,
                           "roofline_note": "algorithmic FLOP per evaluation x evaluations/s "
                                            "over the measured FP64 FMA rate"},
            "accuracy": {"fp32_max_rel_vs_fp64_bins_gt_1e-6_peak": fp32_err,
                         "fp32_band_rel_vs_fp64": band_err, "integrated_fp64": integral,
                         "vs_oracle_subband": vs_oracle},
            "clocks": clocks,
        }
    if not args.no_cpu and rank == 0 and ws == 1:
        log("reference GPU kernel")
        result["reference_gpu_kernel"] = gpu_reference_sample(torch, ctx, L, q, dev)
    if not args.no_batch and rank == 0:
        log("64-pair batch on the 1e6-line list")
        result["batch64"] = batch64(ctx, torch, dev)
        log("64 pairs of the 1e8-line list")
        result["batch_64_pairs_1e8_lines"] = batch_64_pairs_full_list(
            ctx, torch, dev, lines, st, result["roofline"]["flop_per_eval"],
            result["roofline"].get("fp64_peak_tflops"), cfg)
    if not args.no_serve and rank == 0:
        log("serving loop")
        del lines, job, out, L
        torch.cuda.empty_cache()
        result["serve"] = serve_bench(torch, dev, local_rank, args)
    if not args.no_cpu and rank == 0 and ws == 1:
        log("CPU baseline")
        v, cores, sample, kind = cpu_reference_sample(target_s=args.cpu_seconds)
        result["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
                                  "sample": sample}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--lines", type=int, default=100_000_000)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the reference legs (CPU sample, reference GPU kernel)")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--suite", default="main", choices=["main", "quad", "ingest", "serve", "order"],
                    help="quad: Gauss-Hermite 16/32 vs Humlicek on the 5e8-line list; "
                         "ingest: ExoMol text parsed on the GPU vs the reference reader; "
                         "order: a batch in tile-major and job-major item order")
    ap.add_argument("--ingest-lines", type=int, default=20_000_000)
    ap.add_argument("--quad-lines", type=int, default=500_000_000)
    ap.add_argument("--shard", default="replica", choices=["replica", "grid"],
                    help="N>1: one cross-section per rank (weak) or slices of one (strong)")
    ap.add_argument("--serve-scale", type=float, default=0.1,
                    help="scale of the three resident line lists (1 = 1e7, 1e8, 5e8 lines)")
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--serve-loads", type=float, nargs="+", default=[0.3, 0.6, 0.9, 1.2])
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--cfg", default="4,4,0,2",
                    help="launch shape bins_per_lane,warps,ctas_per_sm[,flags] of the timed kernel")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--order-pairs", type=int, default=64,
                    help="order suite: (T, P) pairs of the batch")
    ap.add_argument("--order-plain", action="store_true",
                    help="order suite: plain launches only (for an ncu capture)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    if args.suite == "ingest":
        print(json.dumps(ingest_suite(args)), flush=True)
        return 0
    if args.suite == "serve":
        import torch
        torch.cuda.set_device(0)
        r = serve_bench(torch, "cuda:0", 0, args)
        print(json.dumps({"suite": "serve", **r}), flush=True)
        return 0
    if args.suite == "order":
        print(json.dumps(order_suite(args)), flush=True)
        return 0
    if args.suite == "quad":
        r = quad_suite(args)
        print(json.dumps({"suite": "voigt-quad", "unit": UNIT, **r}), flush=True)
        return 0
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())

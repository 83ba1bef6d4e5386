"""The manager's overlapped transfer (B200Manager: lists of 2^21 lines or
more are copied in pieces on a copy stream and the first launch runs as grid
segments that start as soon as their lines have arrived) gives bit for bit
the sums of one launch over the whole pair: the same job through
Context.run on the same device lines, seeded the same way.  Covers the
segmented first launch, a second launch on the same lines (plain path), a
pair with an unaligned start_idx and a shorter line prefix, a second
TransferVectors of a different list, FP32 and FP64 forms, the inclusive
and the rounded window rule."""
import numpy as np
import pytest
import torch

from gexs_b200 import Context, Job, LineList, synth, _capi as capi
from gexs_b200.engine import Manager

pytestmark = pytest.mark.gpu

NU0, DNU, NPTS = 100.0, 0.05, 598001
MASS, REF_T, REF_P = 18.0, 296.0, 1.0


def _lines(n, seed):
    st = synth.make_states(20000, 40, seed)
    L = synth.make_lines_torch(st, n, NU0, NU0 + DNU * (NPTS - 1), seed + 1,
                               broadening_seed=seed + 2, device="cuda")
    host = {k: v.cpu().pin_memory() for k, v in L.items()}
    return L, host


def _reference(ctx, L, seeds, conv, precision, hw, T, P, q, start, npts, nener):
    dev = {k: v[:nener] for k, v in L.items()}
    lines = LineList(dev["nu"], dev["elow"], dev["aif"], dev["gns"], dev["gamma"], dev["n"])
    out = torch.as_tensor(seeds).to("cuda")
    j = Job(lines, out, convention=conv, profile=capi.VOIGT, temperature=T, pressure=P,
            partition=q, mass=MASS, nu_start=NU0, dnu=DNU, grid_points=NPTS, precision=precision,
            ref_temp=REF_T, ref_press=REF_P, half_width=hw, start_idx=start, n_points=npts,
            accumulate=1)
    ctx.run([j])
    ctx.check()
    return out.cpu().numpy()


@pytest.mark.parametrize("conv,precision,hw", [(capi.CONV_PHYSICAL, capi.FP32, 0.0),
                                               (capi.CONV_REF_GPU, capi.FP64, 20.0),
                                               (capi.CONV_REF_CPU, capi.FP64, 0.0)])
def test_overlapped_transfer_is_bitwise_one_launch(conv, precision, hw):
    n = 3_000_000
    L, h = _lines(n, 501)
    freq = NU0 + np.arange(NPTS, dtype=np.float64) * DNU
    rng = np.random.Generator(np.random.PCG64(7))
    seeds = rng.uniform(0.0, 1e-22, NPTS)
    pairs = [(1500.0, 1.0, 0, NPTS, n), (800.0, 0.1, 12345, NPTS - 20000, n - 777)]
    qs = [1234.5, 567.8]
    m = Manager(capi.VOIGT, 0, conv, precision, memory_bytes=(n * 44) + 3 * NPTS * 8 + (64 << 20))
    m.initialize_vectors(NPTS, 2)
    m.transfer_freq(freq, seeds)
    m.initialize_constants(hw, 296.0, qs[0], DNU, MASS, 1.0, REF_T, REF_P)
    m.transfer_vectors(h["elow"].numpy(), h["nu"].numpy(), h["aif"].numpy(), h["gns"].numpy(),
                       h["gamma"].numpy(), h["n"].numpy())
    got = []
    for i, ((T, P, s0, npts, ne), q) in enumerate(zip(pairs, qs)):
        m.execute(npts, ne, s0, T, P, q)
        f = np.zeros(NPTS)
        o = np.zeros(NPTS)
        m.transfer_results(f, o, i)          # first: segmented launch; second: plain
        got.append(o)
    # a second list through the same manager
    L2, h2 = _lines(n, 777)
    m.transfer_freq(freq, seeds)
    m.transfer_vectors(h2["elow"].numpy(), h2["nu"].numpy(), h2["aif"].numpy(), h2["gns"].numpy(),
                       h2["gamma"].numpy(), h2["n"].numpy())
    T, P, s0, npts, ne = pairs[0]
    m.execute(npts, ne, s0, T, P, qs[0])
    o2 = np.zeros(NPTS)
    m.transfer_results(np.zeros(NPTS), o2, 0)
    m.close()

    ctx = Context(0)
    for (T, P, s0, npts, ne), q, o in zip(pairs, qs, got):
        want = _reference(ctx, L, seeds, conv, precision, hw, T, P, q, s0, npts, ne)
        assert np.any(o != seeds)
        assert np.array_equal(o.view(np.int64), want.view(np.int64)), \
            float(np.max(np.abs(o - want)))
    T, P, s0, npts, ne = pairs[0]
    want2 = _reference(ctx, L2, seeds, conv, precision, hw, T, P, qs[0], s0, npts, ne)
    assert np.array_equal(o2.view(np.int64), want2.view(np.int64))


def test_overlapped_pairs_queued_together_and_doppler():
    """Three Voigt pairs queued before the first TransferResults (one
    segmented flush with three jobs per segment launch), then a Doppler
    manager on the same list without gamma and n."""
    n = 2_500_000
    L, h = _lines(n, 909)
    freq = NU0 + np.arange(NPTS, dtype=np.float64) * DNU
    seeds = np.zeros(NPTS)
    pairs = [(1500.0, 1.0, 0, NPTS, n), (300.0, 5.0, 4097, NPTS - 9000, n - 5),
             (2500.0, 0.01, 77777, 300000, n)]
    qs = [1000.0, 250.0, 3000.0]
    m = Manager(capi.VOIGT, 0, capi.CONV_PHYSICAL, capi.FP32,
                memory_bytes=(n * 44) + 4 * NPTS * 8 + (64 << 20))
    m.initialize_vectors(NPTS, 3)
    m.transfer_freq(freq, seeds)
    m.initialize_constants(0.0, 296.0, qs[0], DNU, MASS, 1.0, REF_T, REF_P)
    m.transfer_vectors(h["elow"].numpy(), h["nu"].numpy(), h["aif"].numpy(), h["gns"].numpy(),
                       h["gamma"].numpy(), h["n"].numpy())
    for (T, P, s0, npts, ne), q in zip(pairs, qs):
        m.execute(npts, ne, s0, T, P, q)
    got = []
    for i in range(3):
        o = np.zeros(NPTS)
        m.transfer_results(np.zeros(NPTS), o, i)
        got.append(o)
    m.close()
    ctx = Context(0)
    for (T, P, s0, npts, ne), q, o in zip(pairs, qs, got):
        want = _reference(ctx, L, seeds, capi.CONV_PHYSICAL, capi.FP32, 0.0, T, P, q, s0, npts, ne)
        assert np.any(o != 0.0)
        assert np.array_equal(o.view(np.int64), want.view(np.int64))

    d = Manager(capi.DOPPLER, 0, capi.CONV_PHYSICAL, capi.FP32,
                memory_bytes=(n * 28) + 2 * NPTS * 8 + (64 << 20))
    d.initialize_vectors(NPTS, 1)
    d.transfer_freq(freq, seeds)
    d.initialize_constants(0.0, 296.0, qs[0], DNU, MASS, 1.0, REF_T, REF_P)
    d.transfer_vectors(h["elow"].numpy(), h["nu"].numpy(), h["aif"].numpy(), h["gns"].numpy())
    d.execute(NPTS, n, 0, 1200.0, 1.0, qs[0])
    o = np.zeros(NPTS)
    d.transfer_results(np.zeros(NPTS), o, 0)
    d.close()
    lines = LineList(L["nu"], L["elow"], L["aif"], L["gns"])
    out = torch.zeros(NPTS, dtype=torch.float64, device="cuda")
    j = Job(lines, out, convention=capi.CONV_PHYSICAL, profile=capi.DOPPLER, temperature=1200.0,
            pressure=1.0, partition=qs[0], mass=MASS, nu_start=NU0, dnu=DNU, grid_points=NPTS,
            precision=capi.FP32, ref_temp=REF_T, ref_press=REF_P, accumulate=1)
    ctx.run([j])
    ctx.check()
    want = out.cpu().numpy()
    assert np.any(o != 0.0)
    assert np.array_equal(o.view(np.int64), want.view(np.int64))

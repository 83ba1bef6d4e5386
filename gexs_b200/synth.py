"""Seeded synthetic ExoMol-style line lists (the workloads have no public
dataset; these stand in with the stated shapes and distributions).

States: E ~ Exponential(mean 4000 cm^-1) clipped to [0, 30000], J uniform
integer in [0, j_max], g = 2J + 1.  Transitions: the lower state is uniform
over states; the upper state is uniform over states with
E_u in [E_l + nu_min, E_l + nu_max] (lower states with no such upper state
are redrawn); nu0 = E_u - E_l; Einstein A log-uniform in [1e-6, 1e2] s^-1;
g_ns of the line = g of the upper state (Readers/Exomol/
ExomolStateReader.cpp:158-162 takes energy of the lower state and g of the
upper).  Broadening: gamma_ref ~ U(0.03, 0.1) cm^-1/atm, n ~ U(0.4, 0.8).
Lines are returned sorted by nu0.

numpy (PCG64) is used for CPU-sized lists; the torch variant generates the
same distributions on the GPU for 1e8-line lists (different random stream).
"""
import numpy as np


class States:
    def __init__(self, energy, g, j):
        self.energy = energy
        self.g = g
        self.j = j


def make_states(n, j_max, seed, mean_e=4000.0, e_max=30000.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    e = np.clip(rng.exponential(mean_e, n), 0.0, e_max)
    j = rng.integers(0, j_max + 1, n).astype(np.int32)
    return States(e.astype(np.float64), (2 * j + 1).astype(np.int32), j)


def _pick_upper(rng, es, lower_e, nu_min, nu_max):
    lo = np.searchsorted(es, lower_e + nu_min, side="left")
    hi = np.searchsorted(es, lower_e + nu_max, side="right")
    ok = hi > lo
    u = rng.random(lower_e.shape[0])
    up = lo + np.floor(u * np.maximum(hi - lo, 1)).astype(np.int64)
    up = np.minimum(up, len(es) - 1)
    return up, ok


def make_lines(states, ntrans, nu_min, nu_max, seed, broadening_seed=None):
    """Return dict of numpy arrays nu, elow, aif, gns (+ gamma, n when
    broadening_seed is given), sorted by nu."""
    rng = np.random.Generator(np.random.PCG64(seed))
    order = np.argsort(states.energy, kind="stable")
    es = states.energy[order]
    gs = states.g[order]
    n = len(es)
    low = rng.integers(0, n, ntrans)
    up, ok = _pick_upper(rng, es, es[low], nu_min, nu_max)
    for _ in range(64):
        bad = np.nonzero(~ok)[0]
        if bad.size == 0:
            break
        low[bad] = rng.integers(0, n, bad.size)
        u2, ok2 = _pick_upper(rng, es, es[low[bad]], nu_min, nu_max)
        up[bad] = u2
        ok[bad] = ok2
    keep = ok
    low, up = low[keep], up[keep]
    nu = es[up] - es[low]
    aif = 10.0 ** rng.uniform(-6.0, 2.0, nu.shape[0])
    srt = np.argsort(nu, kind="stable")
    out = {
        "nu": np.ascontiguousarray(nu[srt], dtype=np.float64),
        "elow": np.ascontiguousarray(es[low][srt], dtype=np.float64),
        "aif": np.ascontiguousarray(aif[srt], dtype=np.float64),
        "gns": np.ascontiguousarray(gs[up][srt], dtype=np.int32),
    }
    if broadening_seed is not None:
        r2 = np.random.Generator(np.random.PCG64(broadening_seed))
        out["gamma"] = r2.uniform(0.03, 0.1, nu.shape[0]).astype(np.float64)
        out["n"] = r2.uniform(0.4, 0.8, nu.shape[0]).astype(np.float64)
    return out


def make_lines_torch(states, ntrans, nu_min, nu_max, seed, broadening_seed=None,
                     device="cuda"):
    """Same distributions generated with torch on `device` (for 1e8+ lines).
    Returns dict of torch tensors sorted by nu."""
    import torch
    gen = torch.Generator(device=device)
    gen.manual_seed(int(seed))
    order = np.argsort(states.energy, kind="stable")
    es = torch.as_tensor(states.energy[order], device=device)
    gs = torch.as_tensor(states.g[order], device=device)
    n = es.shape[0]
    low = torch.randint(0, n, (ntrans,), generator=gen, device=device)
    el = es[low]
    lo = torch.searchsorted(es, el + nu_min, side="left")
    hi = torch.searchsorted(es, el + nu_max, side="right")
    ok = hi > lo
    for _ in range(64):
        bad = torch.nonzero(~ok).flatten()
        if bad.numel() == 0:
            break
        low[bad] = torch.randint(0, n, (bad.numel(),), generator=gen, device=device)
        el[bad] = es[low[bad]]
        lo[bad] = torch.searchsorted(es, el[bad] + nu_min, side="left")
        hi[bad] = torch.searchsorted(es, el[bad] + nu_max, side="right")
        ok[bad] = hi[bad] > lo[bad]
    u = torch.rand(ntrans, generator=gen, device=device, dtype=torch.float64)
    up = lo + torch.floor(u * (hi - lo).clamp(min=1).double()).long()
    up = up.clamp(max=n - 1)
    keep = torch.nonzero(ok).flatten()
    low, up = low[keep], up[keep]
    nu = es[up] - es[low]
    aif = torch.pow(10.0, torch.empty(nu.shape[0], device=device, dtype=torch.float64)
                    .uniform_(-6.0, 2.0, generator=gen))
    nu_sorted, srt = torch.sort(nu, stable=True)
    out = {"nu": nu_sorted.contiguous(), "elow": es[low][srt].contiguous(),
           "aif": aif[srt].contiguous(), "gns": gs[up][srt].to(torch.int32).contiguous()}
    if broadening_seed is not None:
        g2 = torch.Generator(device=device)
        g2.manual_seed(int(broadening_seed))
        m = nu.shape[0]
        out["gamma"] = torch.empty(m, device=device, dtype=torch.float64).uniform_(0.03, 0.1, generator=g2)
        out["n"] = torch.empty(m, device=device, dtype=torch.float64).uniform_(0.4, 0.8, generator=g2)
    return out


# ------------------------------------------------------------------ ExoMol text
# Fixed-width text in the layout of ExoMol files, formatted with numpy
# (vectorised: 1e7-line files in seconds).  The text itself is the ground
# truth of the ingest tests: the parsers are compared on the bytes.
def _digits(v, width, pad=b" "):
    """Right-aligned decimal of non-negative int64 v in `width` columns."""
    v = np.asarray(v, dtype=np.int64)
    out = np.full((v.shape[0], width), pad[0], dtype=np.uint8)
    rem = v.copy()
    for k in range(width - 1, -1, -1):
        d = (rem % 10).astype(np.uint8)
        nz = (rem > 0) | (k == width - 1)
        out[:, k] = np.where(nz, d + ord("0"), out[:, k])
        rem //= 10
    return out


def _zeros(v, width):
    """Zero-padded decimal of non-negative int64 v in `width` columns."""
    v = np.asarray(v, dtype=np.int64)
    out = np.empty((v.shape[0], width), dtype=np.uint8)
    rem = v.copy()
    for k in range(width - 1, -1, -1):
        out[:, k] = (rem % 10).astype(np.uint8) + ord("0")
        rem //= 10
    return out


def _col(n, ch):
    return np.full((n, 1), ord(ch), dtype=np.uint8)


def _fixed(x, width, prec):
    """Non-negative x as '%{width}.{prec}f'-like text (rounded half up)."""
    scale = 10 ** prec
    v = np.floor(np.asarray(x, dtype=np.float64) * scale + 0.5).astype(np.int64)
    return np.hstack([_digits(v // scale, width - prec - 1), _col(len(v), "."),
                      _zeros(v % scale, prec)])


def _sci(x, mant=4):
    """Positive x as 'd.ddddE+XX'."""
    x = np.asarray(x, dtype=np.float64)
    e = np.floor(np.log10(x)).astype(np.int64)
    m = np.floor(x / np.power(10.0, e) * 10 ** mant + 0.5).astype(np.int64)
    over = m >= 10 ** (mant + 1)
    m = np.where(over, m // 10, m)
    e = np.where(over, e + 1, e)
    under = m < 10 ** mant
    m = np.where(under, m * 10, m)
    e = np.where(under, e - 1, e)
    n = len(x)
    sign = np.where(e < 0, ord("-"), ord("+")).astype(np.uint8)[:, None]
    return np.hstack([_zeros(m // 10 ** mant, 1), _col(n, "."), _zeros(m % 10 ** mant, mant),
                      _col(n, "E"), sign, _zeros(np.abs(e), 2)])


def exomol_states_text(states):
    """`id E g J` lines (ids 1..N in order), as ExoMol .states files."""
    n = len(states.energy)
    rows = np.hstack([_digits(np.arange(1, n + 1), 12), _col(n, " "),
                      _fixed(states.energy, 12, 6), _col(n, " "), _digits(states.g, 6),
                      _col(n, " "), _digits(states.j, 7), _col(n, "\n")])
    return rows.tobytes()


def exomol_trans_text(upper, lower, aif, nu=None):
    """`id_upper id_lower A [nu]` lines (1-based ids), as ExoMol .trans files."""
    n = len(upper)
    parts = [_digits(np.asarray(upper) + 1, 12), _col(n, " "), _digits(np.asarray(lower) + 1, 12),
             _col(n, " "), _sci(aif)]
    if nu is not None:
        parts += [_col(n, " "), _fixed(nu, 12, 6)]
    parts.append(_col(n, "\n"))
    return np.hstack(parts).tobytes()


def exomol_broad_text(j_max, seed, a1_pairs=0):
    """`a0 gamma n J''` lines for J'' = 0..j_max (and some `a1 gamma n J'' J'`)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for j in range(j_max + 1):
        out.append("a0 %.4f %.3f %d" % (rng.uniform(0.03, 0.1), rng.uniform(0.4, 0.8), j))
    for _ in range(a1_pairs):
        j = int(rng.integers(0, j_max + 1))
        out.append("a1 %.4f %.3f %d %d" % (rng.uniform(0.03, 0.1), rng.uniform(0.4, 0.8), j,
                                           j + int(rng.integers(-1, 2))))
    return ("\n".join(out) + "\n").encode()


def make_exomol_transitions(states, ntrans, nu_min, nu_max, seed):
    """Upper/lower indices (0-based) and A of seeded transitions, file order
    (not sorted by nu)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    order = np.argsort(states.energy, kind="stable")
    es = states.energy[order]
    lower = rng.integers(0, len(es), ntrans)
    le = es[lower]
    lo = np.searchsorted(es, le + nu_min, side="left")
    hi = np.searchsorted(es, le + nu_max, side="right")
    ok = hi > lo
    lower, lo, hi = lower[ok], lo[ok], hi[ok]
    up = lo + np.floor(rng.random(len(lower)) * (hi - lo)).astype(np.int64)
    up = np.minimum(up, hi - 1)
    aif = 10.0 ** rng.uniform(-6.0, 2.0, len(lower))
    return order[up].astype(np.int64), order[lower].astype(np.int64), aif


def make_hitran_par(n, seed, nu_min=500.0, nu_max=8000.0, a_zero_every=7):
    """Seeded HITRAN .par text (160-column records, HITRAN 2004 layout):
    nu F12.6, S and A E10.3, gamma_air F5.3, gamma_self F5.3, E'' F10.4,
    n_air F4.2, g' and g'' F7.1; every `a_zero_every`-th record has A = 0
    (the reader then rebuilds A from S)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nu = np.sort(rng.uniform(nu_min, nu_max, n))
    S = 10.0 ** rng.uniform(-28.0, -19.0, n)
    A = 10.0 ** rng.uniform(-6.0, 2.0, n)
    gair = rng.uniform(0.02, 0.099, n)
    gself = rng.uniform(0.1, 0.499, n)
    elow = rng.exponential(1500.0, n)
    nair = rng.uniform(0.4, 0.8, n)
    gup = (2 * rng.integers(0, 60, n) + 1).astype(np.float64)
    glow = (2 * rng.integers(0, 60, n) + 1).astype(np.float64)
    zero = np.zeros(n, dtype=bool)
    if a_zero_every:
        zero[::a_zero_every] = True
    sci_a = _sci(np.where(zero, 1.0, A), 3)
    sci_a[zero] = np.frombuffer(b"0.000E+00", dtype=np.uint8)
    cols = [np.tile(np.frombuffer(b" 11", dtype=np.uint8), (n, 1)),
            _fixed(nu, 12, 6), _col(n, " "), _sci(S, 3), _col(n, " "), sci_a,
            _fixed(gair, 5, 3), _fixed(gself, 5, 3), _fixed(elow, 10, 4), _fixed(nair, 4, 2),
            np.tile(np.frombuffer(b" 0.00000", dtype=np.uint8), (n, 1)),
            np.full((n, 60), ord(" "), dtype=np.uint8),
            np.tile(np.frombuffer(b"000000" + b"0" * 12 + b" ", dtype=np.uint8), (n, 1)),
            _fixed(gup, 7, 1), _fixed(glow, 7, 1), _col(n, "\n")]
    rows = np.hstack(cols)
    assert rows.shape[1] == 161
    return rows.tobytes()

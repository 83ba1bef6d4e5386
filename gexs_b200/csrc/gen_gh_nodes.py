"""Generate gh_nodes.h: Gauss-Hermite nodes and weights (weight function
exp(-t^2)) for 16 and 32 points, positive nodes only, ascending.

Golub-Welsch starting values from numpy.polynomial.hermite.hermgauss are
refined by Newton's method on the physicists' Hermite polynomial H_n in
50-digit mpmath arithmetic; weights are w = 2^(n-1) n! sqrt(pi) /
(n^2 H_{n-1}(t)^2).  Run: python gexs_b200/csrc/gen_gh_nodes.py
"""
import os
import numpy as np
import mpmath as mp

mp.mp.dps = 50


def hermite(n, x):
    h0, h1 = mp.mpf(1), 2 * x
    if n == 0:
        return h0, mp.mpf(0)
    for k in range(1, n):
        h0, h1 = h1, 2 * x * h1 - 2 * k * h0
    return h1, h0  # H_n, H_{n-1}


def nodes(n):
    t0, _ = np.polynomial.hermite.hermgauss(n)
    out = []
    for t in t0[t0 > 0]:
        x = mp.mpf(float(t))
        for _ in range(60):
            hn, hm = hermite(n, x)
            dx = hn / (2 * n * hm)           # H_n' = 2n H_{n-1}
            x -= dx
            if abs(dx) < mp.mpf(10) ** -45:
                break
        _, hm = hermite(n, x)
        w = mp.mpf(2) ** (n - 1) * mp.factorial(n) * mp.sqrt(mp.pi) / (n * n * hm * hm)
        out.append((x, w))
    out.sort()
    return out


def main():
    lines = ["/* Gauss-Hermite nodes t_k > 0 (ascending) and weights w_k for the",
             " * weight function exp(-t^2); generated by gen_gh_nodes.py (50-digit",
             " * Newton refinement of H_n roots).  Used by the GPU kernels and by the",
             " * CPU oracle, which must see identical constants. */",
             "#ifndef GEXS_GH_NODES_H", "#define GEXS_GH_NODES_H",
             "#define GEXS_INV_PI 0.31830988618379067154",
             "#define GEXS_INV_SQRTPI 0.56418958354775628695"]
    for n in (16, 32):
        nw = nodes(n)
        assert len(nw) == n // 2
        for tag, vals in (("T", [x for x, _ in nw]), ("W", [w for _, w in nw])):
            lines.append("#define GEXS_GH%d_%s_LIST \\" % (n, tag))
            lines += ["    %s, \\" % mp.nstr(v, 20, min_fixed=-1, max_fixed=1) for v in vals[:-1]]
            lines.append("    %s" % mp.nstr(vals[-1], 20, min_fixed=-1, max_fixed=1))
            lines.append("static const double GEXS_GH%d_%s[%d] = {GEXS_GH%d_%s_LIST};"
                         % (n, tag, n // 2, n, tag))
    lines.append("#endif")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gh_nodes.h")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()

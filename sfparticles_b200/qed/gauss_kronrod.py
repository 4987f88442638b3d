"""Gauss-Kronrod rules for the QED table generator (build-time script).

Writes sfparticles_b200/csrc/sfp_gk_rules.h: the (2n+1)-point Kronrod
extensions of the n-point Gauss-Legendre rules for n = 7 (15 points, the
rule of QUADPACK's infinite-interval integrator QAGI) and n = 10 (21 points,
the rule of its finite-interval integrator QAGS), which the reference's
scipy.integrate.quad runs.  Computed here from the definition, in 60-digit
arithmetic, then rounded to float64:
  * Gauss nodes: the roots of the Legendre polynomial P_n;
  * Kronrod nodes: the n + 1 roots of the Stieltjes polynomial E_{n+1}, the
    monic polynomial of degree n + 1 orthogonal to x^j P_n(x), j = 0..n;
  * weights: the unique weights on the 2n + 1 nodes that integrate
    x^0 .. x^(2n) over [-1, 1] exactly (then exact to degree 3n + 1);
    the Gauss weights likewise on the n Gauss nodes.
Layout as in QUADPACK's qk15 / qk21: xgk[0..n] the non-negative nodes in
decreasing order, the centre last (odd positions, 1-based even, are the
Gauss nodes), wgk their Kronrod weights, wg the Gauss weights.

    python -m sfparticles_b200.qed.gauss_kronrod      # rewrites the header
"""
from __future__ import annotations

import os

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "csrc", "sfp_gk_rules.h")


def _rule(n):
    import mpmath as mp
    mp.mp.dps = 60
    # Legendre P_n coefficients (ascending powers) and its roots
    P = [mp.mpf(0)] * (n + 1)
    for k in range(n // 2 + 1):
        c = (-1) ** k * mp.binomial(n, k) * mp.binomial(2 * n - 2 * k, n) / mp.mpf(2) ** n
        P[n - 2 * k] = c
    gauss = sorted(mp.polyroots(list(reversed(P)), maxsteps=200, extraprec=200), key=lambda r: -mp.re(r))
    gauss = [mp.re(r) for r in gauss]

    def moment(k):  # integral of x^k over [-1, 1]
        return mp.mpf(0) if k % 2 else mp.mpf(2) / (k + 1)

    def integ_poly(c):  # integral of sum c_k x^k
        return mp.fsum(ck * moment(k) for k, ck in enumerate(c))

    def mul(a, b):
        out = [mp.mpf(0)] * (len(a) + len(b) - 1)
        for i, ai in enumerate(a):
            for j, bj in enumerate(b):
                out[i + j] += ai * bj
        return out

    # Stieltjes polynomial E = x^(n+1) + sum_{k<=n} e_k x^k, orthogonal to x^j P_n
    m = n + 1
    A = mp.matrix(m, m)
    rhs = mp.matrix(m, 1)
    for j in range(m):
        xjP = mul([mp.mpf(0)] * j + [mp.mpf(1)], P)
        for k in range(m):
            A[j, k] = integ_poly(mul([mp.mpf(0)] * k + [mp.mpf(1)], xjP))
        rhs[j] = -integ_poly(mul([mp.mpf(0)] * m + [mp.mpf(1)], xjP))
    e = mp.lu_solve(A, rhs)
    E = [e[k] for k in range(m)] + [mp.mpf(1)]
    kron = [mp.re(r) for r in mp.polyroots(list(reversed(E)), maxsteps=400, extraprec=400)]
    nodes = sorted(gauss + kron, key=lambda r: -r)

    def weights(pts):
        N = len(pts)
        V = mp.matrix(N, N)
        b = mp.matrix(N, 1)
        for k in range(N):
            for j, p in enumerate(pts):
                V[k, j] = p ** k
            b[k] = moment(k)
        return [w for w in mp.lu_solve(V, b)]

    wk = weights(nodes)
    wg = weights(gauss)
    # non-negative half, decreasing, centre last
    half = [(p, w) for p, w in zip(nodes, wk) if p >= -mp.mpf(10) ** -40]
    gset = [(p, w) for p, w in zip(gauss, wg) if p >= -mp.mpf(10) ** -40]
    xgk = [float(p) if abs(p) > mp.mpf(10) ** -40 else 0.0 for p, _ in half]
    wgk = [float(w) for _, w in half]
    wgh = [float(w) for _, w in gset]
    return xgk, wgk, wgh


def write_header(path=HEADER):
    lines = ["// sfp_gk_rules.h -- generated by sfparticles_b200/qed/gauss_kronrod.py; do not edit.",
             "// Gauss-Kronrod rules: xgk (non-negative nodes, decreasing, centre last), wgk",
             "// (Kronrod weights), wg (Gauss weights of the nodes xgk[1], xgk[3], ...),",
             "// as accessors usable in host and device code.",
             "#pragma once", "#ifndef SFP_HD", "#if defined(__CUDACC__)", "#define SFP_HD __host__ __device__ inline",
             "#else", "#define SFP_HD inline", "#endif", "#endif", "", "namespace sfp_gk {", ""]
    for n, name in ((7, "15"), (10, "21")):
        xgk, wgk, wg = _rule(n)
        for arr, nm in ((xgk, f"xgk{name}"), (wgk, f"wgk{name}"), (wg, f"wg{name}")):
            body = ", ".join(float.hex(v) for v in arr)
            lines.append(f"SFP_HD double {nm}(int i) {{")
            lines.append(f"    constexpr double v[{len(arr)}] = {{{body}}};")
            lines.append("    return v[i];")
            lines.append("}")
        lines.append("")
    lines.append("}  // namespace sfp_gk")
    lines.append("")
    with open(path, "w") as f:
        f.write("\n".join(lines))
    return path


if __name__ == "__main__":
    print(write_header())

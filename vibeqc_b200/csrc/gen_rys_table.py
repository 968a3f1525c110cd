"""Generate the Rys quadrature table used by the CUDA integral kernels.

Rys quadrature (Rys, Dupuis and King, J. Comput. Chem. 4, 154 (1983)) needs,
for a Boys argument T, the n nodes u_i in (0, 1) and weights w_i with

    sum_i w_i u_i^k = F_k(T) = int_0^1 t^{2k} exp(-T t^2) dt,   k = 0 .. 2n-1.

For every n <= NMAX this script computes (u_i, w_i) in 80-digit arithmetic:
moments F_k(T) = 1F1(k+1/2; k+3/2; -T) / (2k+1), the three-term recurrence by
Gautschi's Chebyshev algorithm, and the Golub-Welsch eigenproblem of the Jacobi
matrix.  On [0, T_asym(n)) it fits each u_i(T) and w_i(T) with a Chebyshev
series of degree DEG on intervals of width H (nodes at Chebyshev points), and
writes the coefficients as hex doubles into ``rys_table.inc``.  For
T >= T_asym(n) the kernels use the large-T limit u_i = x_i^2 / T,
w_i = W_i / sqrt(T) with (x_i, W_i) the positive Gauss-Hermite nodes/weights of
order 2n; those constants are written too.  T_asym(n) is the smallest grid
point where the limit agrees with the exact quadrature to 1e-15 relative.

Run:  python vibeqc_b200/csrc/gen_rys_table.py   (about a minute on 8 cores)
"""

from __future__ import annotations

import math
import multiprocessing as mp_proc
import sys
from pathlib import Path

import mpmath as mp

NMAX = 7
DEG = 9           # Chebyshev degree per interval
H = 0.5           # interval width in T
DPS = 80
TOL_ASYM = 1e-15


def moments(n2: int, t):
    if t == 0:
        return [mp.mpf(1) / (2 * k + 1) for k in range(n2)]
    return [mp.hyp1f1(k + mp.mpf(0.5), k + mp.mpf(1.5), -t) / (2 * k + 1) for k in range(n2)]


def rys_exact(n: int, t) -> tuple[list, list]:
    mu = moments(2 * n, t)
    alpha = [mp.mpf(0)] * n
    beta = [mp.mpf(0)] * n
    sig_prev = [mp.mpf(0)] * (2 * n)
    sig = list(mu)
    alpha[0] = mu[1] / mu[0]
    beta[0] = mu[0]
    for k in range(1, n):
        new = [mp.mpf(0)] * (2 * n)
        for l in range(k, 2 * n - k):
            new[l] = sig[l + 1] - alpha[k - 1] * sig[l] - beta[k - 1] * sig_prev[l]
        alpha[k] = new[k + 1] / new[k] - sig[k] / sig[k - 1]
        beta[k] = new[k] / sig[k - 1]
        sig_prev, sig = sig, new
    j = mp.matrix(n, n)
    for i in range(n):
        j[i, i] = alpha[i]
        if i + 1 < n:
            j[i, i + 1] = j[i + 1, i] = mp.sqrt(beta[i + 1])
    e, q = mp.eigsy(j)
    nodes = [e[i] for i in range(n)]
    weights = [beta[0] * q[0, i] ** 2 for i in range(n)]
    order = sorted(range(n), key=lambda i: nodes[i])
    return [nodes[i] for i in order], [weights[i] for i in order]


def hermite_half(n: int):
    """Positive nodes x_i and weights W_i of 2n-point Gauss-Hermite, ascending."""
    m = 2 * n
    # Jacobi matrix of the Hermite weight exp(-x^2): alpha = 0, beta_k = k/2
    j = mp.matrix(m, m)
    for i in range(m - 1):
        j[i, i + 1] = j[i + 1, i] = mp.sqrt(mp.mpf(i + 1) / 2)
    e, q = mp.eigsy(j)
    pairs = [(e[i], mp.sqrt(mp.pi) * q[0, i] ** 2) for i in range(m) if e[i] > 0]
    pairs.sort(key=lambda p: p[0])
    return [p[0] for p in pairs], [p[1] for p in pairs]


def asym(n: int, t, xs, ws):
    return [x * x / t for x in xs], [w / mp.sqrt(t) for w in ws]


def cheb_nodes(deg):
    return [mp.cos(mp.pi * (k + mp.mpf(0.5)) / (deg + 1)) for k in range(deg + 1)]


def fit_interval(args):
    n, t0 = args
    mp.mp.dps = DPS
    xs = cheb_nodes(DEG)
    vals = []
    for x in xs:
        t = mp.mpf(t0) + (x + 1) * mp.mpf(H) / 2
        u, w = rys_exact(n, t)
        vals.append(u + w)
    coefs = []
    for s in range(2 * n):
        f = [vals[k][s] for k in range(DEG + 1)]
        row = []
        for jdeg in range(DEG + 1):
            c = mp.mpf(0)
            for k in range(DEG + 1):
                c += f[k] * mp.cos(mp.pi * jdeg * (k + mp.mpf(0.5)) / (DEG + 1))
            c *= mp.mpf(2) / (DEG + 1)
            if jdeg == 0:
                c /= 2
            row.append(float(c))
        coefs.append(row)
    return coefs


def clenshaw(c, x):
    b1 = b2 = 0.0
    for k in range(len(c) - 1, 0, -1):
        b1, b2 = 2 * x * b1 - b2 + c[k], b1
    return x * b1 - b2 + c[0]


def t_asym(n, xs, ws):
    mp.mp.dps = DPS
    t = 10.0
    while True:
        ue, we = rys_exact(n, mp.mpf(t))
        ua, wa = asym(n, mp.mpf(t), xs, ws)
        err = max(
            max(abs((a - b) / b) for a, b in zip(ua, ue)),
            max(abs((a - b) / b) for a, b in zip(wa, we)),
        )
        if err < TOL_ASYM:
            return t
        t += H


def main():
    mp.mp.dps = DPS
    out = Path(__file__).with_name("rys_table.inc")
    herm = {n: hermite_half(n) for n in range(1, NMAX + 1)}
    tas = {n: t_asym(n, *herm[n]) for n in range(1, NMAX + 1)}
    print("T_asym:", tas, flush=True)
    jobs = []
    for n in range(1, NMAX + 1):
        nint = int(round(tas[n] / H))
        jobs += [(n, i * H) for i in range(nint)]
    with mp_proc.Pool() as pool:
        res = pool.map(fit_interval, jobs, chunksize=4)
    table = {}
    for (n, t0), c in zip(jobs, res):
        table.setdefault(n, []).append(c)
    # validation at off-node points
    import random

    rnd = random.Random(1)
    worst = {}
    for n in range(1, NMAX + 1):
        err = 0.0
        for _ in range(60):
            t = rnd.uniform(0, tas[n] - 1e-9)
            i = int(t / H)
            x = 2 * (t - i * H) / H - 1
            ue, we = rys_exact(n, mp.mpf(t))
            ref = [float(v) for v in ue + we]
            got = [clenshaw(c, x) for c in table[n][i]]
            err = max(err, max(abs(g - r) / abs(r) for g, r in zip(got, ref)))
        worst[n] = err
    print("max relative fit error per n:", worst, flush=True)
    lines = [
        "// Generated by gen_rys_table.py -- Rys nodes/weights as Chebyshev series.",
        f"// NMAX={NMAX} DEG={DEG} H={H}; max relative fit error per n: "
        + ", ".join(f"{n}:{worst[n]:.1e}" for n in worst),
        "// Included by vqc_internal.cuh inside namespace vqc (device code only).",
        f"#define RYS_NMAX {NMAX}",
        f"#define RYS_DEG {DEG}",
        f"#define RYS_H {H!r}",
        "template <int N> struct RysIntervals;",
        "template <int N> struct RysOffset;",
    ]
    offs, total = [], 0
    for n in range(1, NMAX + 1):
        offs.append(total)
        total += len(table[n]) * 2 * n * (DEG + 1)
    for n in range(1, NMAX + 1):
        lines.append(
            f"template <> struct RysIntervals<{n}> {{ static constexpr int value = {len(table[n])}; }};"
        )
        lines.append(
            f"template <> struct RysOffset<{n}> {{ static constexpr int value = {offs[n - 1]}; }};"
        )
    lines.append(f"#define RYS_TABLE_SIZE {total}")
    lines.append("static __device__ const double d_rys_table[RYS_TABLE_SIZE] = {")
    for n in range(1, NMAX + 1):
        for c in table[n]:
            for row in c:
                lines.append(",".join(float.hex(v) for v in row) + ",")
    lines.append("};")
    # asymptotic constants: x_i^2 and W_i, [n][i] padded to NMAX
    xx = []
    ww = []
    for n in range(1, NMAX + 1):
        xs, ws = herm[n]
        xx.append([float(x * x) for x in xs] + [0.0] * (NMAX - n))
        ww.append([float(w) for w in ws] + [0.0] * (NMAX - n))
    lines.append("static __device__ const double d_rys_x2[RYS_NMAX][RYS_NMAX] = {")
    lines += ["{" + ",".join(float.hex(v) for v in r) + "}," for r in xx]
    lines.append("};")
    lines.append("static __device__ const double d_rys_w[RYS_NMAX][RYS_NMAX] = {")
    lines += ["{" + ",".join(float.hex(v) for v in r) + "}," for r in ww]
    lines.append("};")
    out.write_text("\n".join(lines) + "\n")
    print(f"wrote {out}: {total} coefficients", flush=True)


if __name__ == "__main__":
    sys.setrecursionlimit(10000)
    main()

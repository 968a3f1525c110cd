"""The int8 sliced whitening B = A W, restated in numpy on a real 3-centre tensor.

``scf.whiten_tensor_cores`` forms B = A W from exact integer pieces
(``csrc/ozaki_gemm.cu``): the columns of A are rebalanced against the rows
of W by powers of two S, every row of A S and of (W / S)^T is scaled by
2^-e (max |x| < 2^e) and cut into ns signed 7-bit slices by repeated
round-to-nearest, and the slice products with s + t <= ns + 1 are summed in
integers and scaled by 2^(e_a + e_b - 7 (s + t)).  This test repeats those
steps on the packed 3-centre tensor and Cholesky whitening factor of a water
dimer (def2-SVP / cc-pVDZ-JKFIT, from the oracle) and checks each row of B
against the FP64 product.  The largest per-row error, relative to the row's
largest element, is 1.6e-12 with the kernel's 7 slices (the GPU test
``test_gpu_ozaki`` requires 1e-10), 2.5e-10 with 6 and 3.4e-8 with 5: 6
slices miss the bar, which is why the kernel keeps 7.
"""

import numpy as np
import pytest

from oracle import oracle
from vibeqc_b200 import basis as bas
from vibeqc_b200.geometry import water_cluster

ANGSTROM = 1 / 0.52917721092


def slice_rows(x: np.ndarray, ns: int):
    """(slices (ns, rows, K) int64, exponents (rows,)) as ``slice_rows_kernel``."""
    mx = np.abs(x).max(axis=1)
    e = np.where(mx > 0, np.frexp(mx)[1], 0)
    y = x * np.ldexp(1.0, -e)[:, None]
    out = np.empty((ns,) + x.shape, dtype=np.int64)
    for s in range(ns):
        y = y * 128.0
        a = np.clip(np.rint(y), -127, 127)
        y = y - a
        out[s] = a.astype(np.int64)
    return out, e


def sliced_product(a: np.ndarray, b: np.ndarray, ns: int) -> np.ndarray:
    """A B^T from the slices of the rows of A and of B (pairs s + t <= ns + 1, 1-based)."""
    sa, ea = slice_rows(a, ns)
    sb, eb = slice_rows(b, ns)
    c = np.zeros((a.shape[0], b.shape[0]))
    for g in range(2, ns + 2):  # one exact integer accumulator per level g = s + t
        acc = np.zeros((a.shape[0], b.shape[0]), dtype=np.int64)
        for s in range(1, g):
            t = g - s
            if s <= ns and t <= ns:
                acc += sa[s - 1] @ sb[t - 1].T
        c += acc.astype(np.float64) * 2.0 ** (-7 * g)
    return c * np.ldexp(1.0, ea[:, None] + eb[None, :])


@pytest.fixture(scope="module")
def dimer():
    mol = water_cluster(2, seed=0)
    z = np.array([bas.atomic_number(e) for e, _ in mol])
    xyz = np.array([p for _, p in mol]) * ANGSTROM
    orb = oracle.OracleBasis(bas.expand_shells(z, "def2-SVP"))
    aux = oracle.OracleBasis(bas.expand_shells(z, "cc-pVDZ-JKFIT"))
    full = oracle.int3c(orb, aux, xyz)
    n = full.shape[0]
    mu, nu = np.tril_indices(n)
    a = full[mu, nu]  # packed rows mu >= nu, (P, X)
    m = oracle.int2c(aux, xyz)
    w = np.linalg.inv(np.linalg.cholesky(m)).T  # W = L^-T, upper triangular
    # the kernel's power-of-two balance of A's columns against W's rows
    scale = np.exp2(np.round(0.5 * (np.log2(np.abs(w).max(axis=1)) - 0.5 * np.log2(np.diag(m)))))
    return a, w, scale


def _row_error(a, w, scale, ns):
    ref = a @ w
    got = sliced_product(a * scale[None, :], (w / scale[:, None]).T, ns)
    return float((np.abs(got - ref).max(axis=1) / np.abs(ref).max(axis=1)).max())


def test_seven_slices_give_fp64_accurate_rows(dimer):
    a, w, scale = dimer
    assert _row_error(a, w, scale, 7) < 1e-10


def test_six_slices_miss_the_row_accuracy_bar(dimer):
    a, w, scale = dimer
    assert _row_error(a, w, scale, 6) > 1e-10

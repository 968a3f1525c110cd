"""Bound on what the 3-centre kernels' primitive-pair skip leaves out.

The value and derivative kernels skip a primitive pair (a, b) of a shell
pair when exp(-ab/(a+b) |AB|^2) |c_a c_b| < 1e-30 (``kPrimPairCut`` in
``csrc/vqc_internal.cuh``; c are the normalised contraction coefficients of
``basis.normalized_coefficients``).  The oracle evaluates every primitive.
Here each contracted shell is split into single-primitive shells, the oracle
gives every primitive pair's own 3-centre block, and the blocks of exactly
the pairs the kernels skip are summed per contracted function pair.  On a
water trimer (def2-SVP / cc-pVDZ-JKFIT) the skip removes 1740 of 4356
primitive pairs and what it leaves out is at most 2.8e-28 (largest integral
5.8); the test holds it below 1e-24.
"""

import numpy as np
import pytest

from oracle import oracle
from vibeqc_b200 import basis as bas
from vibeqc_b200.geometry import water_cluster

CUT = 1e-30  # kPrimPairCut
ANGSTROM = 1 / 0.52917721092


def _primitive_shells(shells):
    """One shell per primitive, with (parent shell, primitive index, coefficient / norm)."""
    out, meta = [], []
    for si, s in enumerate(shells):
        a, c = bas.normalized_coefficients(s)
        for k, (ak, ck) in enumerate(zip(a, c)):
            out.append(bas.Shell(s.atom_index, s.angular_momentum, (bas.Primitive(float(ak), 1.0),)))
            # a single-primitive shell is normalised to one: its coefficient is the
            # primitive norm, so the contracted shell weighs it by ck / norm
            meta.append((si, k, ck / bas.primitive_norm(float(ak), s.angular_momentum), float(ak)))
    return out, meta


def test_skipped_primitive_pairs_are_negligible():
    mol = water_cluster(3, seed=0)
    z = np.array([bas.atomic_number(e) for e, _ in mol])
    xyz = np.array([p for _, p in mol]) * ANGSTROM
    shells = bas.expand_shells(z, "def2-SVP")
    aux = oracle.OracleBasis(bas.expand_shells(z, "cc-pVDZ-JKFIT"))
    full = oracle.int3c(oracle.OracleBasis(shells), aux, xyz)

    pshells, meta = _primitive_shells(shells)
    porb = oracle.OracleBasis(pshells)
    prim = oracle.int3c(porb, aux, xyz)  # (nprimfunc, nprimfunc, X)
    nf = [bas.nfunc(s.angular_momentum, True) for s in pshells]
    off = np.concatenate([[0], np.cumsum(nf)])

    fo = np.concatenate([[0], np.cumsum([bas.nfunc(s.angular_momentum, True) for s in shells])])

    skipped = 0
    left_out = np.zeros_like(full)  # what the kernels omit, per contracted function pair
    for i, (si, _, wi, ai) in enumerate(meta):
        for j, (sj, _, wj, aj) in enumerate(meta):
            r2 = float(((xyz[shells[si].atom_index] - xyz[shells[sj].atom_index]) ** 2).sum())
            ci = wi * bas.primitive_norm(ai, shells[si].angular_momentum)
            cj = wj * bas.primitive_norm(aj, shells[sj].angular_momentum)
            if np.exp(-ai * aj / (ai + aj) * r2) * abs(ci * cj) >= CUT:
                continue
            skipped += 1
            left_out[fo[si]:fo[si + 1], fo[sj]:fo[sj + 1]] += (
                wi * wj * prim[off[i]:off[i + 1], off[j]:off[j + 1]])
    assert skipped > 100  # the skip is not vacuous on this cluster
    assert np.abs(full).max() > 0.1
    assert np.abs(left_out).max() < 1e-24, np.abs(left_out).max()


@pytest.mark.parametrize("n", [2])
def test_primitive_split_reassembles_the_contracted_tensor(n):
    """The split above is exact: summing all primitive blocks gives the oracle tensor."""
    mol = water_cluster(n, seed=1)
    z = np.array([bas.atomic_number(e) for e, _ in mol])
    xyz = np.array([p for _, p in mol]) * ANGSTROM
    shells = bas.expand_shells(z, "def2-SVP")
    aux = oracle.OracleBasis(bas.expand_shells(z, "cc-pVDZ-JKFIT"))
    full = oracle.int3c(oracle.OracleBasis(shells), aux, xyz)
    pshells, meta = _primitive_shells(shells)
    prim = oracle.int3c(oracle.OracleBasis(pshells), aux, xyz)
    nf = [bas.nfunc(s.angular_momentum, True) for s in pshells]
    off = np.concatenate([[0], np.cumsum(nf)])
    fo = np.concatenate([[0], np.cumsum([bas.nfunc(s.angular_momentum, True) for s in shells])])
    rebuilt = np.zeros_like(full)
    for i, (si, _, wi, _) in enumerate(meta):
        for j, (sj, _, wj, _) in enumerate(meta):
            rebuilt[fo[si]:fo[si + 1], fo[sj]:fo[sj + 1]] += (
                wi * wj * prim[off[i]:off[i + 1], off[j]:off[j + 1]])
    assert np.abs(rebuilt - full).max() <= 1e-12 * np.abs(full).max()

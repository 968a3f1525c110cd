"""CUDA integral kernels (through the C ABI) against the CPU oracle.

Same shells, same order (auxiliary shells sorted by l as the plan requires),
same coordinates; FP64 bit-for-bit is not expected (Rys quadrature on the GPU,
McMurchie-Davidson in the oracle) -- agreement to 1e-11 relative to the
largest element is.
"""

import numpy as np
import pytest
import torch

from oracle import oracle
from vibeqc_b200 import geometry
from vibeqc_b200.plan import NativePlan, make_molecule
from vibeqc_b200.scf import compute_integrals

pytestmark = pytest.mark.gpu

CASES = [
    (geometry.water_cluster(1, 11), "def2-svp", "cc-pvdz-jkfit"),
    (geometry.alkane(2, 5), "def2-svp", "def2-tzvp"),       # f auxiliary shells on C
    (geometry.water_cluster(1, 13), "def2-tzvp", "cc-pvdz-jkfit"),  # f orbital shells
    (geometry.water_cluster(2, 4), "cc-pvdz", "cc-pvdz-jkfit"),
]


def _oracle_integrals(mol, spherical=True):
    orb = oracle.OracleBasis(mol.orbital_shells, spherical)
    aux = oracle.OracleBasis(mol.aux_shells, spherical)
    xyz = mol.coordinates
    s, t, v = oracle.int1e(orb, xyz, mol.atomic_numbers.astype(float))
    return s, t, v, oracle.int2c(aux, xyz), oracle.int3c(orb, aux, xyz)


def _unpack(a_packed, n):
    mu = np.arange(n)
    hi = np.maximum(mu[:, None], mu[None, :])
    lo = np.minimum(mu[:, None], mu[None, :])
    return a_packed[hi * (hi + 1) // 2 + lo]


@pytest.mark.parametrize("spherical", [True, False])
def test_integrals_match_oracle_ragged_batch(spherical):
    mols = [make_molecule(a, b, x) for a, b, x in CASES]
    plan = NativePlan(mols, spherical)
    xyz = torch.tensor(plan.coordinates(), dtype=torch.float64, device="cuda")
    mat = {k: torch.empty(plan.mat_total, dtype=torch.float64, device="cuda") for k in "stv"}
    met = torch.empty(plan.met_total, dtype=torch.float64, device="cuda")
    a = torch.empty(plan.a_total, dtype=torch.float64, device="cuda")
    from vibeqc_b200 import _lib

    st = torch.cuda.current_stream().cuda_stream
    _lib.call("vqc_int1e", plan.handle, xyz.data_ptr(), mat["s"].data_ptr(), mat["t"].data_ptr(),
              mat["v"].data_ptr(), st)
    _lib.call("vqc_int2c", plan.handle, xyz.data_ptr(), met.data_ptr(), st)
    _lib.call("vqc_int3c", plan.handle, xyz.data_ptr(), a.data_ptr(), st)
    torch.cuda.synchronize()
    for mol, lay in zip(mols, plan.layout):
        s, t, v, m, a3 = _oracle_integrals(mol, spherical)
        n, x = lay.nao, lay.naux
        sl = slice(lay.mat_offset, lay.mat_offset + n * n)
        for name, ref in (("s", s), ("t", t), ("v", v)):
            got = mat[name][sl].view(n, n).cpu().numpy()
            assert np.abs(got - ref).max() <= 1e-11 * max(1.0, np.abs(ref).max()), name
        got_m = met[lay.met_offset:lay.met_offset + x * x].view(x, x).cpu().numpy()
        assert np.abs(got_m - m).max() <= 1e-11 * np.abs(m).max()
        p = n * (n + 1) // 2
        got_a = a[lay.a_offset:lay.a_offset + p * x].view(p, x).cpu().numpy()
        full = _unpack(got_a, n)
        assert np.abs(full - a3).max() <= 1e-11 * np.abs(a3).max()
    plan.close()


def test_int3c_translation_invariance_large_batch():
    # many molecules in one launch; values must not depend on batch position
    mols = [make_molecule(geometry.water_cluster(2, i), "def2-svp", "cc-pvdz-jkfit") for i in range(6)]
    plan = NativePlan(mols + mols[:1], True)
    xyz = torch.tensor(plan.coordinates(), dtype=torch.float64, device="cuda")
    ints = compute_integrals_any(plan, xyz)
    a = ints.cpu().numpy()
    first = plan.layout[0]
    last = plan.layout[-1]
    size = first.npair * first.naux
    assert np.array_equal(a[first.a_offset:first.a_offset + size], a[last.a_offset:last.a_offset + size])
    plan.close()


def compute_integrals_any(plan, xyz):
    from vibeqc_b200 import _lib

    a = torch.empty(plan.a_total, dtype=torch.float64, device="cuda")
    _lib.call("vqc_int3c", plan.handle, xyz.data_ptr(), a.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return a

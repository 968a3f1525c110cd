"""Unrestricted DF-HF on the GPU against the CPU oracle (energies and analytic forces).

Open-shell doublets and a triplet (OH, NH2, O2, the H atom) in one ragged
batch, each in its own chunk (different alpha/beta counts), on the FP64 path
and the mixed-precision path; a closed-shell water solved unrestricted must
reproduce the restricted result.  The unrestricted oracle is pinned by its
own known answers and finite differences (tests/test_oracle_uhf.py).
"""

import numpy as np
import pytest

from oracle import oracle
from vibeqc_b200 import Calculator, geometry

pytestmark = pytest.mark.gpu

BASIS, AUX = "def2-svp", "cc-pvdz-jkfit"
SYSTEMS = [
    ([("O", (0.0, 0.0, 0.0)), ("H", (0.3, 0.2, 1.85))], 2),
    ([("O", (0.0, 0.0, 0.0)), ("O", (0.05, 0.0, 2.28))], 3),
    ([("N", (0.0, 0.0, 0.0)), ("H", (0.0, 1.52, 1.19)), ("H", (0.1, -1.5, 1.2))], 2),
    ([("H", (0.1, -0.2, 0.3))], 2),
]
# |dE| Eh, max|dF| Eh/Bohr against the FP64 oracle
TOL = {"fp64": (1e-8, 1e-7), "mixed": (1e-6, 1e-5)}


@pytest.fixture(scope="module")
def references():
    return [oracle.df_uhf(a, BASIS, AUX, multiplicity=m) for a, m in SYSTEMS]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_open_shell_batch_matches_oracle(precision, references):
    calc = Calculator(method="uhf", basis=BASIS, auxiliary_basis=AUX, device="cuda",
                      density_fitting="cuda", precision=precision)
    batch = calc.prepare_batch([a for a, _ in SYSTEMS], multiplicities=[m for _, m in SYSTEMS])
    res = batch.execute(strict=True)
    batch.close()
    de_tol, df_tol = TOL[precision]
    for item, ref in zip(res.items, references):
        assert item.converged
        assert abs(item.energy - ref.energy) < de_tol, (item.index, item.energy, ref.energy)
        assert np.abs(item.forces - ref.forces).max() < df_tol


def test_closed_shell_unrestricted_equals_restricted():
    atoms = geometry.water_cluster(2, np.random.default_rng(4))
    kw = dict(basis=BASIS, auxiliary_basis=AUX, device="cuda", density_fitting="cuda")
    r = Calculator(method="rhf", **kw).singlepoint(atoms)
    u = Calculator(method="uhf", **kw).singlepoint(atoms)
    assert u.converged
    assert abs(u.energy - r.energy) < 1e-9
    assert np.abs(u.forces - r.forces).max() < 1e-7


def test_unrestricted_warm_start_replay(references):
    calc = Calculator(method="uhf", basis=BASIS, auxiliary_basis=AUX, device="cuda",
                      density_fitting="cuda")
    atoms, m = SYSTEMS[0]
    batch = calc.prepare_batch([atoms], multiplicities=[m])
    cold = batch.execute(strict=True).items[0]
    warm = batch.execute(strict=True).items[0]
    batch.close()
    assert warm.warm_start_used and not cold.warm_start_used
    assert warm.iterations < cold.iterations
    assert abs(warm.energy - references[0].energy) < 1e-8
    assert np.abs(warm.forces - references[0].forces).max() < 1e-7

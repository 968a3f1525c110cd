"""Forces with a truncated auxiliary metric (rank < X) against the CPU oracle.

With density_fitting_relative_threshold above the metric's smallest
eigenvalues the fitting space loses functions and the forces need the spectral
adjoint of the thresholded pseudoinverse (reference
src/integrals/density_fitting_metric.cpp:50-99), whose restatement in the
oracle reproduces the reference's known answers.  An eigenvalue at the cutoff
is a rank crossing: the forces fail with numerical failure (status 5).
"""

import numpy as np
import pytest

from oracle import oracle
from vibeqc_b200 import Calculator, geometry
from vibeqc_b200.plan import make_molecule

pytestmark = pytest.mark.gpu

ATOMS = geometry.water_cluster(2, np.random.default_rng([0, 7]))


def _metric_eigenvalues():
    mol = make_molecule(ATOMS, "def2-svp", "cc-pvdz-jkfit")
    return np.linalg.eigvalsh(oracle.int2c(oracle.OracleBasis(mol.aux_shells, True), mol.coordinates))


def _cut_in_gap(drop: int) -> float:
    """A relative threshold in the widest eigenvalue gap near `drop` discarded functions.

    Near the cutoff the spectral adjoint's divided differences 1/(l_i (l_i - l_j))
    amplify any difference in the converged densities, so the parity check
    keeps the cutoff away from every eigenvalue.
    """
    lam = _metric_eigenvalues()
    j = max(range(max(1, drop - 3), drop + 4), key=lambda i: lam[i] / lam[i - 1])
    return float(np.sqrt(lam[j - 1] * lam[j]) / lam[-1])


@pytest.mark.parametrize("drop", [2, 40])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_truncated_metric_forces_match_oracle(drop, precision):
    # both sides converge well below the default tolerances, so that the
    # comparison probes the force formulas rather than two SCF endpoints
    tight = dict(energy_tolerance=1e-12, density_tolerance=1e-10)
    threshold = _cut_in_gap(drop)
    ref = oracle.df_rhf(ATOMS, "def2-svp", "cc-pvdz-jkfit", relative_threshold=threshold, **tight)
    assert ref.extra["rank"] < ref.extra["naux"]
    calc = Calculator(method="rhf", basis="def2-svp", auxiliary_basis="cc-pvdz-jkfit", device="cuda",
                      density_fitting="cuda", precision=precision,
                      density_fitting_relative_threshold=threshold, **tight)
    res = calc.singlepoint(ATOMS)
    assert res.basis_metadata["metric_rank"] == ref.extra["rank"]
    assert abs(res.energy - ref.energy) < 1e-8
    # FP64: 2e-7 Eh/Bohr as for the reference goldens; mixed (split-precision
    # products, anchored increments): 1e-6, ten times inside its 1e-5 target
    assert np.abs(res.forces - ref.forces).max() < (2e-7 if precision == "fp64" else 1e-6)
    assert np.abs(res.forces.sum(axis=0)).max() < 1e-8


def test_eigenvalue_at_the_cutoff_fails_the_forces():
    lam = _metric_eigenvalues()
    calc = Calculator(method="rhf", basis="def2-svp", auxiliary_basis="cc-pvdz-jkfit", device="cuda",
                      density_fitting="cuda", density_fitting_relative_threshold=lam[8] / lam[-1])
    with calc.prepare_batch([ATOMS]) as batch:
        res = batch.execute()
        assert res.items[0].status == 5 and "rank crossing" in res.items[0].status_message
        energy_only = batch.execute(properties=("energy",))
        assert energy_only.items[0].succeeded

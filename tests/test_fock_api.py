"""Host-side checks of the fixed-density J/K interface and its oracle (no GPU).

* The specification types validate like the reference's
  (``python/generativeqc/fock.py:33-100``).
* The oracle's dE2/dR at a fixed density matches five-point finite
  differences of E2 (restricted hybrid-like and unrestricted densities).
"""

import numpy as np
import pytest

from oracle import oracle
from vibeqc_b200 import FockBuildSpec, FockTerm, geometry


def test_spec_validation():
    assert FockBuildSpec.hf().exchange.coefficient == -0.5
    assert FockBuildSpec.hf("unrestricted").exchange.coefficient == -1.0
    with pytest.raises(ValueError):
        FockTerm(operator="medium_range")
    with pytest.raises(ValueError):
        FockTerm(coefficient=float("nan"))
    with pytest.raises(TypeError):
        FockTerm(present=1)
    with pytest.raises(ValueError):
        FockBuildSpec(spin="general")
    with pytest.raises(ValueError):
        FockBuildSpec(derivative_order=2)


@pytest.mark.parametrize("spins,ck", [(1, -0.25), (2, -1.0)])
def test_oracle_fixed_density_gradient_matches_finite_differences(spins, ck):
    atoms = geometry.water_cluster(1, np.random.default_rng(3))
    base = oracle.df_rhf(atoms, "def2-svp", "cc-pvdz-jkfit", forces=False).density
    rng = np.random.default_rng(1)
    ds = []
    for _ in range(spins):
        a = rng.normal(size=base.shape)
        ds.append(base / spins + 0.025 * (a + a.T))
    g = oracle.fock_evaluate(atoms, "def2-svp", "cc-pvdz-jkfit", ds, 1.0, ck)["gradient"]

    def e2(ia, ix, step):
        moved = [list(a) for a in atoms]
        p = list(moved[ia][1])
        p[ix] += step
        moved[ia][1] = tuple(p)
        return oracle.fock_evaluate([tuple(a) for a in moved], "def2-svp", "cc-pvdz-jkfit", ds,
                                    1.0, ck, derivative=False)["energy_two_electron"]

    # E2 carries ~1e-10 Eh of noise from the metric pseudoinverse (condition
    # ~1e7); a wide five-point stencil keeps the difference quotient clean
    h = 4e-3
    for ia, ix in [(0, 0), (1, 2)]:
        fd = (-e2(ia, ix, 2 * h) + 8 * e2(ia, ix, h) - 8 * e2(ia, ix, -h) + e2(ia, ix, -2 * h)) / (12 * h)
        assert fd == pytest.approx(g[ia, ix], abs=3e-7)

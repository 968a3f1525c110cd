"""Fixed-density DF J/K source (FockPlan) on the GPU against the CPU oracle.

The J/K source other methods consume (hybrid DFT scales exchange by a_x):
raw J and K, the assembled Fock matrices, E1/E2 and the two-electron
gradient dE2/dR at a fixed density, for restricted and unrestricted spin,
Hartree-Fock and hybrid-like coefficients, full-rank and truncated metrics.
The oracle's fixed-density gradient is pinned by five-point finite
differences (tests/test_fock_api.py).
"""

import numpy as np
import pytest

from oracle import oracle
from vibeqc_b200 import Calculator, FockBuildSpec, FockPlan, FockTerm, geometry

pytestmark = pytest.mark.gpu

BASIS, AUX = "def2-svp", "cc-pvdz-jkfit"
ATOMS = geometry.water_cluster(2, np.random.default_rng([0, 11]))


def _density(seed, n, scale=0.05):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, n))
    return scale * 0.5 * (a + a.T)


@pytest.fixture(scope="module")
def scf_density():
    calc = Calculator(method="rhf", basis=BASIS, auxiliary_basis=AUX, device="cuda",
                      density_fitting="cuda")
    res = oracle.df_rhf(ATOMS, BASIS, AUX, forces=False)
    return calc, res.density, res.energy


def _compare(ev, ref, grad_tol=1e-9):
    scale = max(1.0, np.abs(ref["fock"][0]).max())
    assert ev.coulomb is None or np.abs(ev.coulomb - ref["coulomb"]).max() < 1e-10 * scale
    exch = ev.exchange if ev.exchange.ndim == 3 else ev.exchange[None]
    for k, kr in zip(exch, ref["exchange"]):
        assert np.abs(k - kr).max() < 1e-10 * scale
    fock = ev.fock if ev.fock.ndim == 3 else ev.fock[None]
    for f, fr in zip(fock, ref["fock"]):
        assert np.abs(f - fr).max() < 1e-10 * scale
    assert ev.energy_one_electron == pytest.approx(ref["energy_one_electron"], abs=1e-9)
    assert ev.energy_two_electron == pytest.approx(ref["energy_two_electron"], abs=1e-9)
    if ev.gradient is not None:
        g = ev.gradient.reshape(-1, 3)
        assert np.abs(g - ref["gradient"]).max() < grad_tol * max(1.0, np.abs(ref["gradient"]).max())


def test_hf_restricted_at_the_scf_density(scf_density):
    _, d, e_scf = scf_density
    with FockPlan(ATOMS, BASIS, auxiliary_basis=AUX) as plan:
        ev = plan.evaluate(d, derivative=True)
    ref = oracle.fock_evaluate(ATOMS, BASIS, AUX, [d], 1.0, -0.5)
    _compare(ev, ref)
    assert ev.energy == pytest.approx(e_scf, abs=1e-8)


@pytest.mark.parametrize("ck", [-0.125, 0.0])
def test_hybrid_coefficients_perturbed_density(scf_density, ck):
    _, d, _ = scf_density
    d = d + _density(1, d.shape[0])
    spec = FockBuildSpec(coulomb=FockTerm(coefficient=1.0),
                         exchange=FockTerm(coefficient=ck))
    with FockPlan(ATOMS, BASIS, spec, auxiliary_basis=AUX) as plan:
        ev = plan.evaluate(d, derivative=True)
    _compare(ev, oracle.fock_evaluate(ATOMS, BASIS, AUX, [d], 1.0, ck))


def test_unrestricted_spin_densities(scf_density):
    _, d, _ = scf_density
    n = d.shape[0]
    ds = np.stack([0.5 * d + _density(2, n), 0.5 * d + _density(3, n)])
    spec = FockBuildSpec.hf("unrestricted")
    with FockPlan(ATOMS, BASIS, spec, auxiliary_basis=AUX) as plan:
        ev = plan.evaluate(ds, derivative=True)
    assert ev.fock.shape == (2, n, n) and ev.exchange.shape == (2, n, n)
    _compare(ev, oracle.fock_evaluate(ATOMS, BASIS, AUX, list(ds), 1.0, -1.0))


def test_truncated_metric_gradient(scf_density):
    _, d, _ = scf_density
    thr = 1e-4
    with FockPlan(ATOMS, BASIS, auxiliary_basis=AUX, metric_relative_threshold=thr) as plan:
        assert plan._mf.rank[0] < plan.naux
        ev = plan.evaluate(d, derivative=True)
    ref = oracle.fock_evaluate(ATOMS, BASIS, AUX, [d], 1.0, -0.5, relative_threshold=thr)
    _compare(ev, ref, grad_tol=1e-7)


def test_rejections(scf_density):
    _, d, _ = scf_density
    with pytest.raises(NotImplementedError):
        FockPlan(ATOMS, BASIS, FockBuildSpec.hf(exchange="exact"), auxiliary_basis=AUX)
    with pytest.raises(NotImplementedError):
        FockPlan(ATOMS, BASIS, FockBuildSpec(exchange=FockTerm(coefficient=-0.5,
                                                               operator="long_range", omega=0.3)),
                 auxiliary_basis=AUX)
    with FockPlan(ATOMS, BASIS, auxiliary_basis=AUX) as plan:
        with pytest.raises(ValueError):
            plan.evaluate(d[:-1, :-1])
        nonsym = d.copy()
        nonsym[0, 1] += 1e-3
        plan.evaluate(nonsym)  # values accept nonsymmetric densities
        with pytest.raises(ValueError):
            plan.evaluate(nonsym, derivative=True)

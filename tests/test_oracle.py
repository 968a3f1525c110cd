"""The CPU oracle against the reference's golden vectors and known answers.

Golden energies/forces were produced by the reference's own CPU DF-RHF path
(tests/golden/make_golden.py); the spectral known answers are those of the
reference's native test tests/native/test_density_fitting.cpp:984-1047.
"""

import json
from pathlib import Path

import mpmath
import numpy as np
import pytest

from oracle import oracle

GOLDEN = json.loads((Path(__file__).parent / "golden" / "df_rhf_golden.json").read_text())
FAST = [
    "h2o_def2svp_auxdef2svp",
    "h2o_def2svp_jkfit",
    "h2o_ccpvdz_jkfit",
    "nh3_ccpvdz_jkfit",
    "ethane_def2svp_auxdef2tzvp",
    "h2o_def2tzvp_jkfit",
]


def atoms_of(case):
    return [(s, tuple(p)) for s, p in case["atoms"]]


@pytest.mark.parametrize("name", FAST)
def test_oracle_matches_reference_golden(name):
    case = GOLDEN[name]
    res = oracle.df_rhf(atoms_of(case), case["basis"], case["auxiliary_basis"])
    assert res.converged
    assert abs(res.energy - case["energy"]) < 1e-9
    assert np.abs(res.forces - np.array(case["forces"])).max() < 5e-8


def test_golden_water_smoke_energy_pin():
    # the water/def2-SVP smoke number recorded from the reference
    assert GOLDEN["h2o_def2svp_auxdef2svp"]["energy"] == pytest.approx(-76.17929112830237, abs=1e-10)


@pytest.mark.parametrize("m", [0, 3, 8, 16])
@pytest.mark.parametrize("t", [0.0, 1e-9, 0.3, 7.5, 29.9, 30.1, 55.0])
def test_boys_function(m, t):
    mpmath.mp.dps = 40
    exact = mpmath.hyp1f1(m + 0.5, m + 1.5, -t) / (2 * m + 1)
    got = oracle.boys(m, t)[m]
    assert abs(got - float(exact)) <= 2e-14 * float(exact)


def test_spectral_response_known_answer_inverse():
    # M = diag(1, 0.2), threshold 0.3 drops 0.2; d(M+)[0,1] for dM = offdiag(1) is 1.25
    m = np.diag([1.0, 0.2])
    f = oracle.factor_metric(m, 0.3)
    motion = np.array([[0.0, 1.0], [1.0, 0.0]])
    resp = oracle.metric_response(f, motion, 0.3)
    assert resp[0, 1] == pytest.approx(1.25, abs=1e-13)


def test_spectral_response_known_answer_inverse_sqrt():
    # M = diag(4, 1), threshold 0.3 keeps only 4; d(M^-1/2)[0,1] is 1/6
    m = np.diag([4.0, 1.0])
    f = oracle.factor_metric(m, 0.3)
    motion = np.array([[0.0, 1.0], [1.0, 0.0]])
    resp = oracle.metric_response(f, motion, 0.3, power=-0.5)
    assert resp[0, 1] == pytest.approx(1.0 / 6.0, abs=1e-13)


def test_spectral_response_matches_finite_differences():
    rng = np.random.default_rng(3)
    q, _ = np.linalg.qr(rng.normal(size=(5, 5)))
    lam = np.array([1e-12, 0.003, 0.2, 1.0, 2.5])
    m = (q * lam) @ q.T
    bar = rng.normal(size=(5, 5))
    bar = bar + bar.T
    f = oracle.factor_metric(m, 1e-3)
    adj = oracle.metric_response(f, bar, 1e-3)
    dm = rng.normal(size=(5, 5))
    dm = dm + dm.T
    h = 1e-6
    fp = oracle.factor_metric(m + h * dm, 1e-3).pinv
    fm = oracle.factor_metric(m - h * dm, 1e-3).pinv
    fd = np.sum(bar * (fp - fm)) / (2 * h)
    assert np.sum(adj * dm) == pytest.approx(fd, rel=1e-6)


def test_rank_crossing_rejected():
    m = np.diag([1.0, 1e-10 * (1 + 1e-15)])
    f = oracle.factor_metric(m, 1e-10)
    with pytest.raises(FloatingPointError):
        oracle.metric_response(f, np.eye(2), 1e-10)


def test_nonfinite_metric_rejected():
    with pytest.raises(FloatingPointError):
        oracle.factor_metric(np.array([[1.0, np.nan], [np.nan, 1.0]]))


def test_three_centre_symmetry_and_metric_positive():
    case = GOLDEN["h2o_def2svp_jkfit"]
    from vibeqc_b200 import basis as bas

    z, xyz = oracle.molecule_arrays(atoms_of(case))
    orb = oracle.OracleBasis(bas.expand_shells(z.astype(int), "def2-svp"))
    aux = oracle.OracleBasis(bas.expand_shells(z.astype(int), "cc-pvdz-jkfit"))
    a = oracle.int3c(orb, aux, xyz)
    assert np.abs(a - a.transpose(1, 0, 2)).max() == 0.0
    m = oracle.int2c(aux, xyz)
    assert np.linalg.eigvalsh(m).min() > 0

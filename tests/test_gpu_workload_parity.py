"""Workload molecules on the GPU against fixtures and finite differences.

* Water clusters (H2O)n, n = 2..16 (one per size), taken from the 256-cluster ragged workload
  (def2-SVP / cc-pVDZ-JKFIT), and alkanes C4-C8 from the 64-alkane workload
  (def2-SVP / def2-TZVP): FP64 and mixed-precision energies and forces against
  ``oracle_workload_fixtures.json`` (CPU oracle, itself pinned against the
  reference's own DF-RHF goldens).  Tolerances: FP64 |dE| <= 1e-8 Eh and
  max|dF| <= 5e-7 Eh/Bohr (SCF convergence noise); mixed |dE| <= 1e-6 Eh and
  max|dF| <= 1e-5 Eh/Bohr (the mixed-precision target).
* The config-0 tetramer (H2O)4 cc-pVDZ / cc-pVDZ-JKFIT: FP64 forces against
  the reference's own golden forces.
* Alkanes C_nH_{2n+2}, n in {4, 8, 13, 20} from the 64-alkane workload:
  torch.autograd gradients (the native adjoint) against central finite
  differences with step 1e-3 Bohr on 16 random coordinates per molecule,
  tolerance 2e-6 Eh/Bohr, in FP64 and mixed precision.
"""

import json
from pathlib import Path

import numpy as np
import pytest
import torch

from vibeqc_b200 import Calculator, geometry
from vibeqc_b200.basis import atomic_number
from vibeqc_b200.torch import batched_energy

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).parent / "golden"
FIX = json.loads((GOLDEN / "oracle_workload_fixtures.json").read_text())
REF = json.loads((GOLDEN / "df_rhf_golden.json").read_text())

TOL = {"fp64": (1e-8, 5e-7), "mixed": (1e-6, 1e-5)}


def _atoms(rec):
    return [(s, tuple(p)) for s, p in rec["atoms"]]


@pytest.mark.parametrize("group", ["clusters", "alkanes"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_workload_molecules_match_fixtures(group, precision):
    recs = list(FIX[group].values())
    calc = Calculator(method="rhf", basis=recs[0]["basis"], auxiliary_basis=recs[0]["auxiliary_basis"],
                      device="cuda", density_fitting="cuda", precision=precision)
    with calc.prepare_batch([_atoms(r) for r in recs]) as batch:
        res = batch.execute(strict=True)
    tol_e, tol_f = TOL[precision]
    worst = []
    for rec, item in zip(recs, res.items):
        assert item.converged
        assert item.precision["mode"] == precision
        de = abs(item.energy - rec["energy"])
        df = float(np.abs(item.forces - np.asarray(rec["forces"])).max())
        worst.append((de, df, rec["n"]))
        assert de <= tol_e, (rec["n"], de)
        assert df <= tol_f, (rec["n"], df)
        assert np.abs(item.forces.sum(axis=0)).max() < 1e-8  # translational invariance


def test_config0_tetramer_fp64_forces_match_reference():
    case = REF["h2o4_ccpvdz_jkfit_seed0"]
    calc = Calculator(method="rhf", basis=case["basis"], auxiliary_basis=case["auxiliary_basis"],
                      device="cuda", density_fitting="cuda", precision="fp64")
    res = calc.singlepoint([(s, tuple(p)) for s, p in case["atoms"]])
    assert res.converged
    assert abs(res.energy - case["energy"]) < 1e-8
    assert np.abs(res.forces - np.asarray(case["forces"])).max() < 2e-7


def _alkanes():
    sizes = np.random.default_rng(0).integers(4, 21, size=64)
    batch = geometry.alkane_batch(64, 4, 20, 0)
    out = {}
    for i, n in enumerate(sizes):
        if int(n) in (4, 8, 13, 20) and int(n) not in out:
            out[int(n)] = batch[i]
    return [out[n] for n in sorted(out)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autograd_matches_central_differences_on_workload_alkanes(precision):
    h, ncoord = 1e-3, 16
    rng = np.random.default_rng(2024)
    calc = Calculator(method="rhf", basis="def2-svp", auxiliary_basis="def2-tzvp", device="cuda",
                      density_fitting="cuda", precision=precision, energy_tolerance=1e-12,
                      density_tolerance=1e-9)
    for atoms in _alkanes():
        z = [atomic_number(a[0]) for a in atoms]
        xyz0 = np.array([a[1] for a in atoms], dtype=np.float64)
        with calc.prepare_batch([atoms]) as one:
            c = torch.tensor(xyz0, device="cuda").requires_grad_(True)
            e = batched_energy([c], [z], prepared_batch=one)
            e.sum().backward()
            g = c.grad.cpu().numpy()
        picks = [(int(rng.integers(len(z))), int(rng.integers(3))) for _ in range(ncoord)]
        displaced = []
        for a, d in picks:
            for sgn in (1.0, -1.0):
                x = xyz0.copy()
                x[a, d] += sgn * h
                displaced.append(x)
        # all 2 * ncoord displaced geometries in one ragged execution
        with calc.prepare_batch([atoms] * len(displaced)) as many:
            res = many.execute(displaced, properties=("energy",), strict=True)
        en = np.array([it.energy for it in res.items])
        fd = (en[0::2] - en[1::2]) / (2 * h)
        ana = np.array([g[a, d] for a, d in picks])
        err = np.abs(fd - ana)
        assert err.max() < 2e-6, (len(z), err.max(), picks[int(err.argmax())])

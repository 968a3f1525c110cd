"""Mixed-precision path (tcgen05 3xTF32 K, FP32 J) against the FP64 GPU path.

Tolerances are the targets of this engine: |dE| <= 1e-6 Eh and
max|dF| <= 1e-5 Eh/Bohr against the FP64 plan of the same molecule, and the
same bounds against the reference's golden values.
"""

import json
from pathlib import Path

import numpy as np
import pytest
import torch

from vibeqc_b200.gradient import df_rhf_gradient
from vibeqc_b200.plan import make_molecule
from vibeqc_b200.scf import Chunk, compute_integrals, run_scf

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "df_rhf_golden.json").read_text())


def _run(mol, precision):
    chunk = Chunk([mol], [0])
    xyz = torch.tensor(chunk.plan.coordinates(), dtype=torch.float64, device="cuda")
    ints = compute_integrals(chunk.plan, xyz)
    out = run_scf(chunk, ints, xyz, precision=precision)
    grad = df_rhf_gradient(chunk, ints, out, xyz).cpu().numpy()
    e = float(out["energy"][0])
    conv = bool(out["converged"][0])
    chunk.close()
    return e, -grad, conv


@pytest.mark.parametrize("name", ["h2o_def2svp_jkfit", "nh3_ccpvdz_jkfit", "ethane_def2svp_auxdef2tzvp",
                                  "h2o2_def2svp_jkfit", "h2o4_ccpvdz_jkfit_seed0"])
def test_mixed_matches_fp64_and_reference(name):
    case = GOLDEN[name]
    atoms = [(s, tuple(p)) for s, p in case["atoms"]]
    mol = make_molecule(atoms, case["basis"], case["auxiliary_basis"])
    e64, f64, c64 = _run(mol, "fp64")
    emx, fmx, cmx = _run(mol, "mixed")
    assert c64 and cmx
    assert abs(emx - e64) <= 1e-6
    assert np.abs(fmx - f64).max() <= 1e-5
    assert abs(emx - case["energy"]) <= 1e-6
    assert np.abs(fmx - np.array(case["forces"])).max() <= 1e-5


def test_decane_mixed_matches_fp64():
    """Single all-trans n-decane, def2-SVP (250 AO), FP64 vs mixed on the GPU.

    No carbon JK-fit set is bundled; def2-TZVP (442 functions) stands in as the
    auxiliary basis, fed identically to both precisions.
    """
    from vibeqc_b200 import geometry

    mol = make_molecule(geometry.alkane(10, 0), "def2-svp", "def2-tzvp")
    e64, f64, c64 = _run(mol, "fp64")
    emx, fmx, cmx = _run(mol, "mixed")
    assert c64 and cmx
    assert abs(emx - e64) <= 1e-6
    assert np.abs(fmx - f64).max() <= 1e-5


def test_mixed_request_beyond_kernel_limits_runs_fp64():
    """(H2O)22 in def2-SVP has N = 528 > 512: its chunk runs the FP64 GPU path."""
    from vibeqc_b200 import Calculator, geometry

    calc = Calculator(method="rhf", basis="def2-svp", auxiliary_basis="cc-pvdz-jkfit", device="cuda",
                      density_fitting="cuda", precision="mixed")
    batch = calc.prepare_batch([geometry.water_cluster(22, 0), geometry.water_cluster(3, 0)])
    res = batch.execute(properties=("energy",))
    assert res.items[0].succeeded and res.items[0].precision == {"mode": "fp64", "requested": "mixed"}
    assert res.items[1].succeeded and res.items[1].precision == {"mode": "mixed", "requested": "mixed"}
    batch.close()

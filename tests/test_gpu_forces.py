"""FP64 GPU DF-RHF analytic forces against the reference's golden forces."""

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


@pytest.mark.parametrize(
    "name",
    ["h2o_def2svp_jkfit", "nh3_ccpvdz_jkfit", "ethane_def2svp_auxdef2tzvp", "h2o_def2tzvp_jkfit",
     "h2o2_def2svp_jkfit"],
)
def test_fp64_forces_match_reference(name):
    case = GOLDEN[name]
    atoms = [(s, tuple(p)) for s, p in case["atoms"]]
    mol = make_molecule(atoms, case["basis"], case["auxiliary_basis"])
    chunk = Chunk([mol], [0])
    xyz = torch.tensor(chunk.plan.coordinates(), dtype=torch.float64, device="cuda")
    ints = compute_integrals(chunk.plan, xyz)
    out = run_scf(chunk, ints, xyz, precision="fp64")
    grad = df_rhf_gradient(chunk, ints, out, xyz).cpu().numpy()
    forces = -grad
    ref = np.array(case["forces"])
    assert np.abs(forces - ref).max() < 2e-7, np.abs(forces - ref).max()
    # translational invariance of the analytic gradient
    assert np.abs(grad.sum(axis=0)).max() < 1e-9
    chunk.close()

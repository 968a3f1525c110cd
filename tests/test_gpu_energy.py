"""FP64 GPU DF-RHF energies against the reference's golden energies."""

import json
from pathlib import Path

import numpy as np
import pytest
import torch

from vibeqc_b200.plan import make_molecule
from vibeqc_b200.scf import Chunk, compute_integrals, run_scf

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "df_rhf_golden.json").read_text())


@pytest.mark.parametrize(
    "name",
    ["h2o_def2svp_jkfit", "h2o_ccpvdz_jkfit", "nh3_ccpvdz_jkfit", "ethane_def2svp_auxdef2tzvp",
     "h2o_def2tzvp_jkfit", "h2o2_def2svp_jkfit", "h2o4_ccpvdz_jkfit_seed0"],
)
def test_fp64_energy_matches_reference(name):
    case = GOLDEN[name]
    atoms = [(s, tuple(p)) for s, p in case["atoms"]]
    mol = make_molecule(atoms, case["basis"], case["auxiliary_basis"])
    chunk = Chunk([mol], [0])
    xyz = torch.tensor(chunk.plan.coordinates(), dtype=torch.float64, device="cuda")
    ints = compute_integrals(chunk.plan, xyz)
    out = run_scf(chunk, ints, xyz, precision="fp64")
    assert bool(out["converged"][0])
    assert abs(float(out["energy"][0]) - case["energy"]) < 1e-8
    chunk.close()

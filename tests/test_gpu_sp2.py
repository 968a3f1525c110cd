"""Purification with the X^2 product on the int8 tensor cores against the DGEMM form.

SP2 (Niklasson, PRB 66, 155115 (2002)) needs X^2 to FP64 accuracy in the
anchored phase of the mixed SCF (density tolerance 1e-8); the sliced int8
product (7-bit slices, exact int32 accumulation) must give the same
projector as the batched DGEMM, and a mixed-precision SCF that purifies with
it must reproduce the FP64 path's energies and forces.
"""

import numpy as np
import pytest
import torch

from vibeqc_b200 import Calculator, geometry, tuning
from vibeqc_b200.scf import Chunk, _orthogonalizer, compute_integrals, purify_sp2
from vibeqc_b200.plan import make_molecule

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nclust,nb", [(2, 3), (9, 2)])
def test_int8_square_purification_matches_dgemm(nclust, nb):
    mols = [make_molecule(geometry.water_cluster(nclust, np.random.default_rng([nclust, k])),
                          "def2-svp", "cc-pvdz-jkfit") for k in range(nb)]
    chunk = Chunk(mols, list(range(nb)))
    xyz = torch.as_tensor(chunk.plan.coordinates(), dtype=torch.float64, device="cuda")
    ints = compute_integrals(chunk.plan, xyz)
    xo = _orthogonalizer(ints.s)
    fo = xo.transpose(1, 2) @ ints.h @ xo
    p64 = purify_sp2(fo, chunk.nocc, graphs={}, gemm="fp64")
    p8 = purify_sp2(fo, chunk.nocc, graphs={}, gemm="int8")
    assert (p8 - p64).abs().max().item() < 1e-10
    assert (p8 @ p8 - p8).abs().max().item() < 1e-9
    tr = torch.diagonal(p8, dim1=1, dim2=2).sum(dim=1)
    assert torch.allclose(tr, torch.full_like(tr, float(chunk.nocc)), atol=1e-9)
    chunk.close()


def test_mixed_scf_with_int8_purification_matches_fp64():
    systems = [geometry.water_cluster(n, np.random.default_rng([5, n])) for n in (3, 3, 6)]
    kw = dict(method="rhf", basis="def2-svp", auxiliary_basis="cc-pvdz-jkfit", device="cuda",
              density_fitting="cuda")
    ref = Calculator(precision="fp64", **kw).prepare_batch(systems).execute(strict=True)
    table = tuning.TuningTable({}, {})
    prev = tuning.active_table()
    try:
        tuning.set_active_table(table)
        table.entries = {k: tuning.Schedule(sp2_gemm="int8") for k in
                         ("72/348/15", "144/696/30")}
        got = Calculator(precision="mixed", **kw).prepare_batch(systems).execute(strict=True)
    finally:
        tuning.set_active_table(prev)
    for a, b in zip(got.items, ref.items):
        assert abs(a.energy - b.energy) < 1e-8
        assert np.abs(a.forces - b.forces).max() < 1e-6

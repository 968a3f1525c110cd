"""Bounded 3-centre row tiles (the integral source) against the full tensor.

Every tile of every molecule of a ragged batch must reproduce, bit for bit,
the rows vqc_int3c writes for the whole batch (the same kernels run on a
restricted pair list); concatenated tiles cover the packed tensor exactly;
whitened tiles equal the rows of A W.
"""

import numpy as np
import pytest
import torch

from vibeqc_b200 import geometry
from vibeqc_b200.plan import NativePlan, make_molecule
from vibeqc_b200.scf import compute_integrals, factor_metric
from vibeqc_b200.source import IntegralSource

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("spherical", [True, False])
def test_row_tiles_match_full_tensor(spherical):
    mols = [make_molecule(geometry.water_cluster(3, np.random.default_rng(1)), "def2-tzvp",
                          "cc-pvdz-jkfit"),
            make_molecule(geometry.water_cluster(2, np.random.default_rng(2)), "def2-svp",
                          "cc-pvdz-jkfit")]
    plan = NativePlan(mols, spherical)
    xyz = torch.as_tensor(plan.coordinates(), dtype=torch.float64, device="cuda")
    full = torch.empty(plan.a_total, dtype=torch.float64, device="cuda")
    import vibeqc_b200._lib as lib

    lib.call("vqc_int3c", plan.handle, xyz.data_ptr(), full.data_ptr(),
             torch.cuda.current_stream().cuda_stream)
    src = IntegralSource(plan)
    for m, lay in enumerate(plan.layout):
        a = full[lay.a_offset:lay.a_offset + lay.npair * lay.naux].view(lay.npair, lay.naux)
        tiles = src.tiles(m, max_bytes=lay.npair * lay.naux * 8 // 5)
        assert len(tiles) > 2
        parts = [src.raw_tile(xyz, m, s0, s1) for s0, s1 in tiles]
        got = torch.cat(parts, dim=0)
        assert got.shape == a.shape
        assert torch.equal(got, a)
        # an arbitrary interior tile on its own
        s0, s1 = 1, src.nshells(m) - 1
        r0, r1 = src.row_range(m, s0, s1)
        assert torch.equal(src.raw_tile(xyz, m, s0, s1), a[r0:r1])
    plan.close()


def test_whitened_tiles_equal_rows_of_a_w():
    mols = [make_molecule(geometry.water_cluster(2, np.random.default_rng(5)), "def2-svp",
                          "cc-pvdz-jkfit")]
    plan = NativePlan(mols, True)
    xyz = torch.as_tensor(plan.coordinates(), dtype=torch.float64, device="cuda")
    ints = compute_integrals(plan, xyz)
    mf = factor_metric(ints.metric)
    b_ref = ints.a_packed[0] @ mf.inv_sqrt[0]
    src = IntegralSource(plan)
    rows = [src.whitened_tile(xyz, 0, s0, s1, mf.inv_sqrt[0])
            for s0, s1 in src.tiles(0, max_bytes=1 << 20)]
    got = torch.cat(rows, dim=0)
    assert (got - b_ref).abs().max().item() <= 1e-12 * b_ref.abs().max().item()
    plan.close()


def test_bad_tile_arguments_rejected():
    mols = [make_molecule(geometry.water_cluster(1, np.random.default_rng(0)), "def2-svp",
                          "cc-pvdz-jkfit")]
    plan = NativePlan(mols, True)
    xyz = torch.as_tensor(plan.coordinates(), dtype=torch.float64, device="cuda")
    src = IntegralSource(plan)
    import vibeqc_b200._lib as lib

    buf = torch.empty(1 << 16, dtype=torch.float64, device="cuda")
    with pytest.raises(lib.VqcError):  # shell range beyond the molecule
        lib.call("vqc_int3c_rows", plan.handle, xyz.data_ptr(), 0, 2, 2 + src.nshells(0),
                 buf.data_ptr(), torch.cuda.current_stream().cuda_stream)
    with pytest.raises(lib.VqcError):  # empty range
        lib.call("vqc_int3c_rows", plan.handle, xyz.data_ptr(), 0, 3, 3, buf.data_ptr(),
                 torch.cuda.current_stream().cuda_stream)
    with pytest.raises(lib.VqcError):  # molecule index
        lib.call("vqc_int3c_rows", plan.handle, xyz.data_ptr(), 1, 0, 1, xyz.data_ptr(),
                 torch.cuda.current_stream().cuda_stream)
    plan.close()

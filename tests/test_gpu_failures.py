"""Failure detection without a GPU fault: host-injected failures and a device
wait that is made to run out.

* An item with non-finite coordinates fails alone (status 1); the other items
  of its chunk and batch keep their results.
* An iteration limit reports status 4 per item; strict execution raises.
* The tensor-core kernels' bounded mbarrier wait gives up after its budget,
  reports an error code and leaves the CUDA context usable.
"""

import numpy as np
import pytest
import torch

from vibeqc_b200 import Calculator, _lib, geometry

pytestmark = pytest.mark.gpu


def _calc(**kw):
    return Calculator(method="rhf", basis="def2-svp", auxiliary_basis="cc-pvdz-jkfit",
                      device="cuda", density_fitting="cuda", **kw)


def test_nonfinite_item_fails_alone():
    systems = [geometry.water_cluster(2, s) for s in (1, 2)] + [geometry.water_cluster(3, 3)]
    batch = _calc().prepare_batch(systems)
    clean = batch.execute()
    coords = [np.array([p for _, p in s], dtype=np.float64) for s in systems]
    coords[0][1, 2] = np.nan  # shares its chunk with system 1
    res = batch.execute(coords)
    assert res.items[0].status == 1 and not res.items[0].succeeded
    for i in (1, 2):
        assert res.items[i].succeeded
        assert abs(res.items[i].energy - clean.items[i].energy) < 1e-9
        assert np.abs(res.items[i].forces - clean.items[i].forces).max() < 1e-8
    with pytest.raises(RuntimeError):
        batch.execute(coords, strict=True)
    batch.close()


def test_iteration_limit_reports_not_converged():
    batch = _calc(max_iterations=2).prepare_batch([geometry.water_cluster(2, 4)])
    res = batch.execute()
    assert res.items[0].status == 4 and not res.items[0].converged
    with pytest.raises(RuntimeError):
        batch.execute(strict=True)
    batch.close()


def test_bounded_wait_reports_expiry_and_context_survives():
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _lib.call("vqc_wait_selftest", 50_000, err.data_ptr(), st)  # 50 ms budget
    torch.cuda.synchronize()
    assert int(err.item()) == 31
    x = torch.randn(1000, device="cuda", dtype=torch.float32)
    hi, lo = torch.empty_like(x), torch.empty_like(x)
    _lib.call("vqc_split_tf32", x.data_ptr(), hi.data_ptr(), lo.data_ptr(), x.numel(), st)
    torch.cuda.synchronize()
    assert torch.allclose(hi.double() + lo.double(), x.double(), rtol=1e-6, atol=0)
    with pytest.raises(_lib.VqcError):
        _lib.call("vqc_wait_selftest", 0, err.data_ptr(), st)

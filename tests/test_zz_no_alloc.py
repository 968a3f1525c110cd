"""The no-allocation fitted-density entry point against the workspace one.

The entry point serves callers that cannot allocate device memory (their GPU
memory is owned by another allocator's pool, or they must avoid the
synchronisation cudaFree implies): its partial sums live in a fixed array
inside the library.  Two calls in a row must both reproduce the workspace
entry point, so nothing left in the shared array from a previous call leaks
into a result.  The file name makes pytest collect it last, in the same
process as the other GPU tests and after them; it also passes when run on its
own in a fresh process.
"""

import pytest
import torch

from vibeqc_b200 import _lib

pytestmark = pytest.mark.gpu


def _case(nb, n, x, seed):
    ld = (n + 3) // 4 * 4
    g = torch.Generator(device="cuda").manual_seed(seed)
    b = torch.zeros(nb, n, x, ld, dtype=torch.float32, device="cuda")
    b[..., :n] = torch.randn(nb, n, x, n, generator=g, device="cuda")
    d = torch.randn(nb, n, n, generator=g, device="cuda", dtype=torch.float64)
    return b, 0.5 * (d + d.transpose(1, 2)), ld


@pytest.mark.parametrize("nb,n,x", [(2, 40, 200), (1, 384, 1856), (3, 13, 77)])
def test_noalloc_matches_workspace_entry_point_twice(nb, n, x):
    b, d, ld = _case(nb, n, x, 21)
    st = torch.cuda.current_stream().cuda_stream
    part = torch.empty(nb, n, x, dtype=torch.float64, device="cuda")
    ref = torch.empty(nb, x, dtype=torch.float64, device="cuda")
    _lib.call("vqc_fitted_density_fp32", b.data_ptr(), d.data_ptr(), nb, n, ld, x,
              part.data_ptr(), ref.data_ptr(), st)
    for _ in range(2):  # two calls in a row: the scratch holds no state between calls
        out = torch.full((nb, x), float("nan"), dtype=torch.float64, device="cuda")
        _lib.call("vqc_fitted_density_fp32_noalloc", b.data_ptr(), d.data_ptr(), nb, n, ld, x,
                  out.data_ptr(), st)
        torch.cuda.synchronize()
        assert torch.equal(out, ref)


def test_noalloc_rejects_oversized_request():
    b, d, ld = _case(1, 8, 8, 1)
    out = torch.empty(1, 8, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.VqcError, match="exceeds"):
        _lib.call("vqc_fitted_density_fp32_noalloc", b.data_ptr(), d.data_ptr(), 1000, 2048, ld,
                  4096, out.data_ptr(), torch.cuda.current_stream().cuda_stream)

"""Int8 tensor-core products with FP64 accuracy (vqc_ozaki_slice_rows / vqc_ozaki_gemm).

The slicing (power-of-two row scale, 7-bit round-to-nearest slices) and the
recombination (exact int32 slice products, then FP64 scaling per slice-pair
weight) are deterministic IEEE operations, so a numpy restatement of the same
steps reproduces the GPU result bit for bit.  Against the plain FP64 product
the error is ~2^-7ns of the row/column scales.  The whitening built on them
must agree with the FP64 whitening to 1e-10 of each (non-negligible) row's
largest element.
"""

import numpy as np
import pytest
import torch

from vibeqc_b200 import _lib, geometry
from vibeqc_b200.plan import make_molecule

pytestmark = pytest.mark.gpu


def _np_slices(x, ns, scale=None):
    y = x * scale[None, :] if scale is not None else x.copy()
    mx = np.abs(y).max(axis=1)
    e = np.where(mx > 0, np.frexp(mx)[1], 0).astype(np.int64)
    y = y * np.ldexp(1.0, -e)[:, None]
    out = []
    for _ in range(ns):
        y = y * 128.0
        a = np.clip(np.rint(y), -127.0, 127.0)
        y = y - a
        out.append(a.astype(np.int64))
    return out, e


def _np_gemm(sa, ea, sb, eb, ns):
    acc = np.zeros((sa[0].shape[0], sb[0].shape[0]))
    scale = 1.0 / 16384.0
    for g in range(ns):
        v = sum(sa[s] @ sb[g - s].T for s in range(g + 1))
        acc = acc + v.astype(np.float64) * scale
        scale /= 128.0
    return np.ldexp(acc, ea[:, None] + eb[None, :])


def _gpu(a, b, ns, upper=0, scale=None):
    """a (nmol, m, k), b (nmol, n, k) FP64 -> (nmol, m, n) and the int8 slices."""
    nmol, m, k = a.shape
    n = b.shape[1]
    ldk = (k + 15) // 16 * 16
    da = torch.tensor(a, device="cuda")
    db = torch.tensor(b, device="cuda")
    sa = torch.zeros(nmol, ns, m, ldk, dtype=torch.int8, device="cuda")
    sb = torch.zeros(nmol, ns, n, ldk, dtype=torch.int8, device="cuda")
    ea = torch.empty(nmol, m, dtype=torch.int32, device="cuda")
    eb = torch.empty(nmol, n, dtype=torch.int32, device="cuda")
    sc = None if scale is None else torch.tensor(scale, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _lib.call("vqc_ozaki_slice_rows", da.data_ptr(), nmol, m, k, k, m * k,
              None if sc is None else sc.data_ptr(), ns, sa.data_ptr(), ldk, ea.data_ptr(), st)
    _lib.call("vqc_ozaki_slice_rows", db.data_ptr(), nmol, n, k, k, n * k, None, ns, sb.data_ptr(),
              ldk, eb.data_ptr(), st)
    c = torch.full((nmol, m, n), float("nan"), dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("vqc_ozaki_gemm", sa.data_ptr(), ea.data_ptr(), m, sb.data_ptr(), eb.data_ptr(), n, k,
              ldk, nmol, ns, upper, c.data_ptr(), n, m * n, err.data_ptr(), st)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return c.cpu().numpy(), sa.cpu().numpy()[..., :k], ea.cpu().numpy()


@pytest.mark.parametrize("ns", [7, 3])
@pytest.mark.parametrize("upper", [0, 1])
def test_slices_and_products_match_numpy_restatement_bit_for_bit(ns, upper):
    rng = np.random.default_rng(11 + ns + upper)
    nmol, m, n, k = 2, 300, 200, 200 if upper else 250
    a = rng.standard_normal((nmol, m, k)) * 10.0 ** rng.uniform(-3, 3, size=(nmol, m, 1))
    b = rng.standard_normal((nmol, n, k)) * 10.0 ** rng.uniform(-2, 2, size=(nmol, n, 1))
    if upper:
        b = np.where(np.arange(k)[None, None, :] > np.arange(n)[None, :, None], 0.0, b)
    scale = np.ldexp(1.0, rng.integers(-4, 5, size=(nmol, k))).astype(np.float64)
    c, sa_gpu, ea_gpu = _gpu(a, b, ns, upper, scale)
    for z in range(nmol):
        sa, ea = _np_slices(a[z], ns, scale[z])
        sb, eb = _np_slices(b[z], ns)
        assert (ea_gpu[z] == ea).all()
        for s in range(ns):
            assert (sa_gpu[z, s] == sa[s]).all()
        ref = _np_gemm(sa, ea, sb, eb, ns)
        assert np.array_equal(c[z], ref), np.abs(c[z] - ref).max()
        exact = (a[z] * scale[z][None, :]) @ b[z].T
        bound = np.abs(a[z] * scale[z][None, :]).max(axis=1)[:, None] * np.abs(b[z]).max(axis=1)[None, :]
        assert (np.abs(c[z] - exact) <= 2.0 ** (-7 * ns + 1) * k * bound).all()


def test_tensor_core_whitening_matches_fp64_whitening():
    from vibeqc_b200.scf import (Chunk, compute_integrals, factor_metric, whiten_in_place,
                                 whiten_tensor_cores)

    mols = [make_molecule(geometry.water_cluster(8, np.random.default_rng([0, 8 + i])), "def2-svp",
                          "cc-pvdz-jkfit") for i in range(2)]
    chunk = Chunk(mols, [0, 1])
    xyz = torch.tensor(chunk.plan.coordinates(), dtype=torch.float64, device="cuda")
    ints = compute_integrals(chunk.plan, xyz)
    mf = factor_metric(ints.metric)
    ref = ints.a_packed.clone()
    whiten_in_place(ref, mf)
    b = ints.a_packed.clone()
    whiten_tensor_cores(b, mf, ints.metric)
    # rows above 1e-12 of the tensor's largest element: 1e-10 of their own
    # largest element; every row (including pairs of far-apart tight
    # functions, whose entries are negligible): 1e-10 of the tensor's largest
    rowmax = ref.abs().amax(dim=2)
    big = rowmax > 1e-12 * rowmax.max()
    err = (b - ref).abs().amax(dim=2)
    rel = (err[big] / rowmax[big]).max().item()
    assert rel < 1e-10, rel
    assert err.max().item() < 1e-10 * rowmax.max().item()
    chunk.close()


@pytest.mark.parametrize("n,nmol", [(48, 3), (200, 2), (384, 1)])
def test_symmetric_output_mode_equals_full_product(n, nmol):
    """upper = 2 forms only the tiles on or above the diagonal of X X^T and mirrors
    them; the sliced sums are exactly symmetric, so the result is bit-identical."""
    rng = np.random.default_rng(n)
    x = rng.normal(size=(nmol, n, n))
    x = 0.5 * (x + x.transpose(0, 2, 1))
    ns = 7
    ldk = (n + 15) // 16 * 16
    dx = torch.tensor(x, device="cuda")
    sl = torch.zeros(nmol, ns, n, ldk, dtype=torch.int8, device="cuda")
    ex = torch.empty(nmol, n, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _lib.call("vqc_ozaki_slice_rows", dx.data_ptr(), nmol, n, n, n, n * n, None, ns, sl.data_ptr(),
              ldk, ex.data_ptr(), st)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    full = torch.full((nmol, n, n), float("nan"), dtype=torch.float64, device="cuda")
    sym = torch.full((nmol, n, n), float("nan"), dtype=torch.float64, device="cuda")
    for mode, out in ((0, full), (2, sym)):
        _lib.call("vqc_ozaki_gemm", sl.data_ptr(), ex.data_ptr(), n, sl.data_ptr(), ex.data_ptr(), n,
                  n, ldk, nmol, ns, mode, out.data_ptr(), n, n * n, err.data_ptr(), st)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(full, sym)
    ref = np.einsum("bij,bkj->bik", x, x)
    assert np.abs(sym.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
    with pytest.raises(_lib.VqcError):  # symmetric mode needs A == B
        _lib.call("vqc_ozaki_gemm", sl.data_ptr(), ex.data_ptr(), n, sl.data_ptr(), err.data_ptr(), n,
                  n, ldk, nmol, ns, 2, sym.data_ptr(), n, n * n, err.data_ptr(), st)

"""Tensor-core split-precision GEMMs and the FP32 Coulomb kernel vs FP64 torch.

3xTF32 with round-to-nearest splitting carries ~2^-22 relative product error,
but the tensor core's FP32 accumulation is not round-to-nearest: it leaves a
relative bias of about 2^-24 per accumulation step along a chain, so a chain
of L steps is good to ~L * 2^-25.  The half transform (L <= 144 for N <= 384)
and the Gram product (accumulator drained to FP64 every kFlush K-blocks) both
stay within 5e-6 relative, which the tests pin.  A TF32-only product (2^-11)
would miss that bound by orders of magnitude.
"""

import pytest
import torch

from vibeqc_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nb,n,x,o", [(2, 40, 200, 12), (1, 96, 464, 20), (3, 50, 130, 33),
                                      (1, 384, 300, 80), (2, 72, 520, 100), (1, 136, 260, 128)])
def test_half_transform_and_gram(nb, n, x, o):
    ld = (n + 3) // 4 * 4
    o_pad = (o + 15) // 16 * 16
    g = torch.Generator(device="cuda").manual_seed(7)
    b = torch.zeros(nb, n, x, ld, dtype=torch.float32, device="cuda")
    b[..., :n] = torch.randn(nb, n, x, n, generator=g, device="cuda")
    c = torch.randn(nb, n, o, generator=g, device="cuda", dtype=torch.float64) / n**0.5
    ct = torch.zeros(nb, o, ld, dtype=torch.float32, device="cuda")
    ct[:, :, :n] = c.transpose(1, 2)
    st = torch.cuda.current_stream().cuda_stream
    ct_hi, ct_lo = torch.empty_like(ct), torch.empty_like(ct)
    _lib.call("vqc_split_tf32", ct.data_ptr(), ct_hi.data_ptr(), ct_lo.data_ptr(), ct.numel(), st)
    ldq = (x + 3) // 4 * 4
    u_hi = torch.zeros((nb, n, o, ldq), dtype=torch.float32, device="cuda")
    u_lo = torch.zeros_like(u_hi)
    rho = torch.zeros(nb, x, dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    dm = torch.randn(nb, n, n, generator=g, device="cuda", dtype=torch.float64)
    dm = 0.5 * (dm + dm.transpose(1, 2))
    rho_d = torch.zeros(nb, x, dtype=torch.float64, device="cuda")
    _lib.call("vqc_tc_half_transform", b.data_ptr(), nb, n, ld, x, ct_hi.data_ptr(),
              ct_lo.data_ptr(), c.contiguous().data_ptr(), o, o_pad, ldq, u_hi.data_ptr(),
              u_lo.data_ptr(), rho.data_ptr(), dm.data_ptr(), rho_d.data_ptr(), err.data_ptr(), st)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.isfinite(u_hi).all() and torch.isfinite(u_lo).all()
    # the split parts are TF32-representable (low 13 mantissa bits clear)
    assert ((u_hi.view(torch.int32) & 0x1FFF) == 0).all()
    assert ((u_lo.view(torch.int32) & 0x1FFF) == 0).all()
    b64 = b[..., :n].double()
    c_used = (ct_hi + ct_lo)[:, :, :n].transpose(1, 2).double()  # the C the kernel multiplied
    ref = torch.einsum("bmqn,bni->bmqi", b64, c_used)
    u = u_hi.double() + u_lo.double()  # (nb, mu, i, Q)
    got = u[..., :x].transpose(2, 3)
    scale = ref.abs().max().item()
    assert (got - ref).abs().max().item() <= 5e-6 * scale
    assert (u[..., x:] == 0).all()
    ref_rho = 2.0 * torch.einsum("bmi,bmqi->bq", c, ref)
    assert (rho - ref_rho).abs().max().item() <= 5e-6 * ref_rho.abs().max().item()
    # fitted density formed by the splitters from the exact FP32 B: four-term
    # FP32 partial sums (weights rounded to FP32) accumulated in FP64, so the
    # error is bounded by a few 2^-24 of sum |B| |D| per entry
    ref_rd = torch.einsum("bmqn,bmn->bq", b64, dm)
    bound = torch.einsum("bmqn,bmn->bq", b64.abs(), dm.abs())
    assert ((rho_d - ref_rd).abs() <= 4 * 2.0**-24 * bound).all()

    kdim = o * ldq
    k = torch.zeros(nb, n, n, dtype=torch.float64, device="cuda")
    _lib.call("vqc_tc_gram", u_hi.data_ptr(), u_lo.data_ptr(), nb, n, kdim, k.data_ptr(),
              err.data_ptr(), st)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    uf = u.reshape(nb, n, kdim)
    kref = uf @ uf.transpose(1, 2)
    assert (k - kref).abs().max().item() <= 5e-6 * kref.abs().max().item()
    # off-diagonal tiles are mirrored exactly; diagonal tiles come from separate MMA lanes
    assert (k - k.transpose(1, 2)).abs().max().item() <= 1e-9 * kref.abs().max().item()


def _split(t):
    hi, lo = torch.empty_like(t), torch.empty_like(t)
    _lib.call("vqc_split_tf32", t.data_ptr(), hi.data_ptr(), lo.data_ptr(), t.numel(),
              torch.cuda.current_stream().cuda_stream)
    return hi, lo


@pytest.mark.parametrize("nb,n,kdim", [(2, 40, 256), (1, 200, 1040), (3, 130, 4000)])
def test_gram_sym2_matches_fp64(nb, n, kdim):
    """kout += A B^T + B A^T on top of an existing FP64 value (the anchor K0 / 2)."""
    g = torch.Generator(device="cuda").manual_seed(11)
    a = torch.randn(nb, n, kdim, generator=g, device="cuda", dtype=torch.float32)
    b = 1e-3 * torch.randn(nb, n, kdim, generator=g, device="cuda", dtype=torch.float32)
    ah, al = _split(a)
    bh, bl = _split(b)
    base = torch.randn(nb, n, n, generator=g, device="cuda", dtype=torch.float64)
    base = base + base.transpose(1, 2)
    k = base.clone()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("vqc_tc_gram_sym2", ah.data_ptr(), al.data_ptr(), bh.data_ptr(), bl.data_ptr(), nb, n,
              kdim, k.data_ptr(), err.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    a64, b64 = (ah.double() + al.double()), (bh.double() + bl.double())
    inc = a64 @ b64.transpose(1, 2) + b64 @ a64.transpose(1, 2)
    got = k - base
    # the increment's error scales with |A| |B|, not with the base value
    assert (got - inc).abs().max().item() <= 5e-6 * inc.abs().max().item()
    # diagonal tiles add the two segments in different orders for (r, c) and
    # (c, r): the asymmetry is FP32 accumulation noise of the increment
    assert (k - k.transpose(1, 2)).abs().max().item() <= 5e-6 * inc.abs().max().item()


def test_anchor_combine_modes():
    g = torch.Generator(device="cuda").manual_seed(5)
    rows, x, ldq = 777, 130, 132
    u0 = torch.randn(rows, x, generator=g, device="cuda", dtype=torch.float64)
    du = torch.zeros(rows, ldq, device="cuda", dtype=torch.float32)
    du[:, :x] = 1e-4 * torch.randn(rows, x, generator=g, device="cuda")
    dh, dl = _split(du)
    vh = torch.full((rows, ldq), 7.0, device="cuda", dtype=torch.float32)
    vl = torch.full_like(vh, 7.0)
    st = torch.cuda.current_stream().cuda_stream
    _lib.call("vqc_anchor_combine", u0.data_ptr(), dh.data_ptr(), dl.data_ptr(), vh.data_ptr(),
              vl.data_ptr(), rows, x, ldq, 0.5, 0, st)
    torch.cuda.synchronize()
    want = u0 + 0.5 * (dh[:, :x].double() + dl[:, :x].double())
    got = vh[:, :x].double() + vl[:, :x].double()
    assert ((vh.view(torch.int32) & 0x1FFF) == 0).all()
    assert (got - want).abs().max().item() <= 2.0**-21 * want.abs().max().item()
    assert (vh[:, x:] == 0).all() and (vl[:, x:] == 0).all()
    ref = u0 + (dh[:, :x].double() + dl[:, :x].double())
    _lib.call("vqc_anchor_combine", u0.data_ptr(), dh.data_ptr(), dl.data_ptr(), 0, 0, rows, x,
              ldq, 1.0, 1, st)
    torch.cuda.synchronize()
    assert (u0 - ref).abs().max().item() <= 1e-15 * ref.abs().max().item()


def test_split_tf32_exact_sum():
    x = torch.randn(10007, device="cuda", dtype=torch.float32) * 1e3
    hi, lo = torch.empty_like(x), torch.empty_like(x)
    _lib.call("vqc_split_tf32", x.data_ptr(), hi.data_ptr(), lo.data_ptr(), x.numel(),
              torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert ((hi.view(torch.int32) & 0x1FFF) == 0).all()
    err = (hi.double() + lo.double() - x.double()).abs() / x.double().abs().clamp_min(1e-30)
    assert err.max().item() <= 2.0**-21


@pytest.mark.parametrize("nb,n,x", [(2, 40, 200), (1, 384, 1856), (3, 13, 77)])
def test_coulomb_fp32(nb, n, x):
    ld = (n + 3) // 4 * 4
    g = torch.Generator(device="cuda").manual_seed(3)
    full = torch.randn(nb, n, n, x, generator=g, device="cuda", dtype=torch.float64)
    full = 0.5 * (full + full.transpose(1, 2))
    b = torch.zeros(nb, n, x, ld, dtype=torch.float32, device="cuda")
    b[..., :n] = full.permute(0, 1, 3, 2).float()
    rho = torch.randn(nb, x, generator=g, device="cuda", dtype=torch.float64)
    j = torch.empty(nb, n, n, dtype=torch.float64, device="cuda")
    _lib.call("vqc_coulomb_fp32", b.data_ptr(), rho.data_ptr(), nb, n, ld, x, j.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ref = torch.einsum("bmqn,bq->bmn", b[..., :n].double(), rho)
    assert (j - ref).abs().max().item() <= 1e-12 * ref.abs().max().item() * x**0.5


@pytest.mark.parametrize("nb,n,x", [(2, 40, 200), (1, 384, 1856), (3, 13, 77), (2, 520, 300)])
def test_coulomb_tma(nb, n, x):
    """The TMA-streamed Coulomb build against FP64 torch and the per-row kernel."""
    ld = (n + 3) // 4 * 4
    g = torch.Generator(device="cuda").manual_seed(5)
    full = torch.randn(nb, n, n, x, generator=g, device="cuda", dtype=torch.float32)
    full = 0.5 * (full + full.transpose(1, 2))
    b = torch.zeros(nb, n, x, ld, dtype=torch.float32, device="cuda")
    b[..., :n] = full.permute(0, 1, 3, 2)
    del full
    rho = torch.randn(nb, x, generator=g, device="cuda", dtype=torch.float64)
    j = torch.full((nb, n, n), float("nan"), dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _lib.call("vqc_coulomb_tma", b.data_ptr(), rho.data_ptr(), nb, n, ld, x, j.data_ptr(),
              err.data_ptr(), st)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = torch.einsum("bmqn,bq->bmn", b[..., :n].double(), rho)
    assert (j - ref).abs().max().item() <= 1e-12 * ref.abs().max().item() * x**0.5
    assert torch.equal(j, j.transpose(1, 2))
    if ld <= 512:
        j2 = torch.empty_like(j)
        _lib.call("vqc_coulomb_fp32", b.data_ptr(), rho.data_ptr(), nb, n, ld, x, j2.data_ptr(), st)
        torch.cuda.synchronize()
        assert (j - j2).abs().max().item() <= 1e-12 * ref.abs().max().item() * x**0.5


@pytest.mark.parametrize("nb,n,x", [(2, 40, 200), (1, 384, 1856), (3, 13, 77)])
def test_fitted_density_fp32(nb, n, x):
    ld = (n + 3) // 4 * 4
    g = torch.Generator(device="cuda").manual_seed(4)
    full = torch.randn(nb, n, n, x, generator=g, device="cuda", dtype=torch.float64)
    full = 0.5 * (full + full.transpose(1, 2))
    b = torch.zeros(nb, n, x, ld, dtype=torch.float32, device="cuda")
    b[..., :n] = full.permute(0, 1, 3, 2).float()
    d = torch.randn(nb, n, n, generator=g, device="cuda", dtype=torch.float64)
    d = 0.5 * (d + d.transpose(1, 2))
    rho = torch.full((nb, x), float("nan"), dtype=torch.float64, device="cuda")
    part = torch.full((nb, n, x), float("nan"), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    _lib.call("vqc_fitted_density_fp32", b.data_ptr(), d.data_ptr(), nb, n, ld, x, part.data_ptr(),
              rho.data_ptr(), st)
    torch.cuda.synchronize()
    ref = torch.einsum("bmqn,bmn->bq", b[..., :n].double(), d)
    assert (rho - ref).abs().max().item() <= 1e-12 * ref.abs().max().item() * n
    # deterministic: a second call reproduces every bit
    rho2 = torch.empty_like(rho)
    _lib.call("vqc_fitted_density_fp32", b.data_ptr(), d.data_ptr(), nb, n, ld, x, part.data_ptr(),
              rho2.data_ptr(), st)
    torch.cuda.synchronize()
    assert torch.equal(rho, rho2)


def test_unpack_aux_major_roundtrip():
    nb, n, x = 2, 11, 37
    ld = 12
    p = n * (n + 1) // 2
    g = torch.Generator(device="cuda").manual_seed(5)
    bp = torch.randn(nb, p, x, generator=g, device="cuda", dtype=torch.float64)
    b = torch.full((nb, n, x, ld), 7.0, dtype=torch.float32, device="cuda")
    _lib.call("vqc_unpack_aux_major", bp.data_ptr(), nb, n, x, ld, b.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    mu = torch.arange(n, device="cuda")
    hi = torch.maximum(mu[:, None], mu[None, :])
    lo = torch.minimum(mu[:, None], mu[None, :])
    idx = (hi * (hi + 1) // 2 + lo)
    ref = bp[:, idx, :].permute(0, 1, 3, 2).float()  # (nb, mu, Q, nu)
    assert torch.equal(b[..., :n], ref)
    assert (b[..., n:] == 0).all()


def test_bad_arguments_rejected():
    st = torch.cuda.current_stream().cuda_stream
    with pytest.raises(_lib.VqcError):
        _lib.call("vqc_tc_half_transform", 0, 1, 8, 8, 8, 0, 0, 0, 4, 16, 8, 0, 0, 0, 0, 0, 0, st)
    x = torch.zeros(64, dtype=torch.float32, device="cuda")
    with pytest.raises(_lib.VqcError):  # o_pad above the supported tile
        _lib.call("vqc_tc_half_transform", x.data_ptr(), 1, 8, 8, 8, x.data_ptr(), x.data_ptr(),
                  x.data_ptr(), 140, 144, 8, x.data_ptr(), x.data_ptr(), x.data_ptr(), 0, 0,
                  x.data_ptr(), st)
    with pytest.raises(_lib.VqcError):  # density without its output
        _lib.call("vqc_tc_half_transform", x.data_ptr(), 1, 8, 8, 8, x.data_ptr(), x.data_ptr(),
                  x.data_ptr(), 4, 16, 8, x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(), 0,
                  x.data_ptr(), st)

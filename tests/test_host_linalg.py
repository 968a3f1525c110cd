"""Host-side FP64 linear algebra of the SCF driver, checked on the CPU."""

import numpy as np
import pytest
import torch

from vibeqc_b200 import scf


def _spd(nb, x, cond, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nb):
        q, _ = np.linalg.qr(rng.standard_normal((x, x)))
        lam = np.geomspace(1.0, 1.0 / cond, x)
        out.append((q * lam) @ q.T)
    return torch.tensor(np.array(out))


@pytest.mark.parametrize("x,p", [(37, 50), (300, 700), (513, 129)])
def test_whiten_in_place_matches_dense_product(x, p, monkeypatch):
    monkeypatch.setattr(scf, "WHITEN_COLUMN_BLOCK", 64)
    m = _spd(2, x, 1e5, x)
    mf = scf.factor_metric(m)
    assert mf.kind == "cholesky"
    a = torch.randn(2, p, x, dtype=torch.float64, generator=torch.Generator().manual_seed(3))
    ref = a @ mf.inv_sqrt
    scf.whiten_in_place(a, mf)
    assert torch.allclose(a, ref, rtol=0, atol=1e-12 * ref.abs().max().item())
    # W W^T = M^-1
    ww = mf.inv_sqrt @ mf.inv_sqrt.transpose(1, 2)
    assert torch.allclose(ww @ m, torch.eye(x, dtype=torch.float64).expand(2, x, x), atol=1e-6)


def test_whiten_eigen_factor_dense():
    m = _spd(1, 40, 1e14, 1)  # cutoff active -> eigen factor with reduced rank
    mf = scf.factor_metric(m, relative_threshold=1e-10)
    assert mf.kind == "eigen" and mf.rank[0] < 40
    a = torch.randn(1, 60, 40, dtype=torch.float64)
    ref = a @ mf.inv_sqrt
    scf.whiten_in_place(a, mf)
    assert torch.allclose(a, ref, rtol=0, atol=1e-12 * ref.abs().max().item())


def test_occupied_factor_without_noise_stays_aligned():
    g = torch.Generator().manual_seed(0)
    n, o = 30, 6
    q, _ = torch.linalg.qr(torch.randn(1, n, n, dtype=torch.float64, generator=g))
    c0 = q[:, :, :o]
    # a slightly rotated occupied space
    k = 1e-4 * torch.randn(1, n - o, o, dtype=torch.float64, generator=g)
    c1 = c0 + q[:, :, o:] @ k
    c1, _ = torch.linalg.qr(c1)
    proj = c1 @ c1.transpose(1, 2)
    co = scf.occupied_factor(proj, c0, g, noise_scale=0.0)
    assert torch.allclose(co.transpose(1, 2) @ co, torch.eye(o, dtype=torch.float64)[None], atol=1e-12)
    assert torch.allclose(co @ co.transpose(1, 2), proj, atol=1e-12)
    assert (co - c0).abs().max().item() < 1e-3  # aligned to the guess, O(|rotation|)


@pytest.mark.parametrize("n,o,x,upper", [(13, 3, 40, True), (70, 9, 300, True), (45, 6, 100, False)])
def test_gradient_weights_match_dense_formulas(n, o, x, upper, monkeypatch):
    from vibeqc_b200 import gradient as gr

    monkeypatch.setattr(gr, "WEIGHT_ROW_BLOCK", 8)
    monkeypatch.setattr(gr, "SYM_BLOCK", 64)
    g = torch.Generator().manual_seed(n)
    nb = 2
    c = torch.randn(nb, n, o, dtype=torch.float64, generator=g)
    dens = 2.0 * c @ c.transpose(1, 2)
    rho = torch.randn(nb, x, dtype=torch.float64, generator=g)
    u = torch.randn(nb, n, o, x, dtype=torch.float64, generator=g)
    w = torch.randn(nb, x, x, dtype=torch.float64, generator=g)
    if upper:
        w = torch.triu(w)
    abar, mbar = gr.chunk_weights(c, dens, rho, u, w, upper)
    mu, nu = torch.tril_indices(n, n)
    for m in range(nb):
        # dense restatement: Abar = D (x) cvec - 2 C Gamma C^T, Mbar = -cc^T/2 + Gamma Gamma^T
        cvec = w[m] @ rho[m]
        bij = torch.einsum("mi,mjq->qij", c[m], u[m])
        gam = (w[m] @ bij.reshape(x, o * o)).view(x, o, o)
        full = dens[m][:, :, None] * cvec - 2.0 * torch.einsum("mi,nj,pij->mnp", c[m], c[m], gam)
        ref_abar = full[mu, nu]
        ref_mbar = -0.5 * torch.outer(cvec, cvec) + gam.reshape(x, -1) @ gam.reshape(x, -1).T
        assert torch.allclose(abar[m], ref_abar, rtol=0, atol=1e-11 * ref_abar.abs().max().item())
        assert torch.allclose(mbar[m], ref_mbar, rtol=0, atol=1e-11 * ref_mbar.abs().max().item())


def test_unrestricted_gradient_weights_match_dense_formulas(monkeypatch):
    """Two spin channels c_s = C_s / sqrt(2): Abar = D_t (x) cvec - sum_s C_s Gamma_s C_s^T,
    Mbar = -cc^T/2 + 1/2 sum_s Gamma_s Gamma_s^T (Gamma_s from the unscaled C_s)."""
    from vibeqc_b200 import gradient as gr

    monkeypatch.setattr(gr, "WEIGHT_ROW_BLOCK", 8)
    monkeypatch.setattr(gr, "SYM_BLOCK", 64)
    g = torch.Generator().manual_seed(11)
    nb, n, o, x = 2, 17, 4, 60
    cs = [torch.randn(nb, n, o, dtype=torch.float64, generator=g) for _ in range(2)]
    cs[1][:, :, 3] = 0.0  # beta padded with a zero column
    bfull = torch.randn(nb, n, n, x, dtype=torch.float64, generator=g)
    bfull = 0.5 * (bfull + bfull.transpose(1, 2))
    w = torch.triu(torch.randn(nb, x, x, dtype=torch.float64, generator=g))
    ds = [c @ c.transpose(1, 2) for c in cs]
    dt = ds[0] + ds[1]
    rho = torch.einsum("bmnq,bmn->bq", bfull, dt)
    abar = torch.empty(nb, n * (n + 1) // 2, x, dtype=torch.float64)
    mbar = torch.empty(nb, x, x, dtype=torch.float64)
    for ch, c in enumerate(cs):
        ct = c / 2 ** 0.5
        u = torch.einsum("bmnq,bni->bmiq", bfull, ct)
        gr.chunk_weights(ct, dt, rho, u, w, True, abar, mbar, k_scale=2.0, coulomb=ch == 0)
    mu, nu = torch.tril_indices(n, n)
    for m in range(nb):
        cvec = w[m] @ rho[m]
        full = dt[m][:, :, None] * cvec
        ref_mbar = -0.5 * torch.outer(cvec, cvec)
        for c in cs:
            bij = torch.einsum("mi,mnq,nj->qij", c[m], bfull[m], c[m])
            gam = (w[m] @ bij.reshape(x, o * o)).view(x, o, o)
            full = full - torch.einsum("mi,nj,pij->mnp", c[m], c[m], gam)
            ref_mbar = ref_mbar + 0.5 * gam.reshape(x, -1) @ gam.reshape(x, -1).T
        ref_abar = full[mu, nu]
        assert torch.allclose(abar[m], ref_abar, rtol=0, atol=1e-11 * ref_abar.abs().max().item())
        assert torch.allclose(mbar[m], ref_mbar, rtol=0, atol=1e-11 * ref_mbar.abs().max().item())


def test_uhf_post_block_matches_plain_restatement():
    from vibeqc_b200 import uhf

    g = torch.Generator().manual_seed(5)
    nb, n, x, hist = 2, 7, 4, 3

    def sym(*shape):
        a = torch.randn(*shape, dtype=torch.float64, generator=g)
        return 0.5 * (a + a.transpose(-1, -2))

    h, s = sym(nb, n, n), sym(nb, n, n) + 4 * torch.eye(n, dtype=torch.float64)
    xo = torch.randn(nb, n, n, dtype=torch.float64, generator=g)
    enuc = torch.randn(nb, dtype=torch.float64, generator=g)
    post = uhf._UHFPost(nb, n, x, hist, False, "cpu")
    post.load(h, s, xo, enuc)
    errs, focks = [], []
    for it in range(5):
        j, ka, kb, da, db = (sym(nb, n, n) for _ in range(5))
        f, energy, cmax, f_ext = post.run(j, ka, kb, da, db)
        fa, fb = h + j - ka, h + j - kb
        e_ref = (0.5 * ((da + db) * h).sum(dim=(1, 2)) + 0.5 * (da * fa).sum(dim=(1, 2))
                 + 0.5 * (db * fb).sum(dim=(1, 2)) + enuc)
        assert torch.allclose(energy, e_ref, atol=1e-12)
        res = [fs @ ds @ s - s @ ds @ fs for fs, ds in ((fa, da), (fb, db))]
        assert torch.allclose(cmax, torch.maximum(res[0].abs().amax(dim=(1, 2)),
                                                  res[1].abs().amax(dim=(1, 2))))
        errs.append(torch.cat([xo.transpose(1, 2) @ r @ xo for r in res], dim=1))
        focks.append(torch.cat([fa, fb], dim=1))
        errs, focks = errs[-hist:], focks[-hist:]
        ref = _reference_diis(errs, focks) if len(errs) > 1 else focks[-1]
        got = torch.cat([f_ext[0], f_ext[1]], dim=1)
        assert torch.allclose(got, ref, atol=1e-9 * ref.abs().max().item())


def _reference_diis(errs, focks):
    """Pulay extrapolation over the given vectors (plain restatement)."""
    nh = len(errs)
    e = torch.stack(errs, dim=1)
    f = torch.stack(focks, dim=1)
    gram = torch.einsum("bimn,bjmn->bij", e, e)
    nb = e.shape[0]
    bmat = -torch.ones(nb, nh + 1, nh + 1, dtype=e.dtype)
    bmat[:, nh, nh] = 0.0
    bmat[:, :nh, :nh] = gram
    rhs = torch.zeros(nb, nh + 1, 1, dtype=e.dtype)
    rhs[:, nh, 0] = -1.0
    w = torch.linalg.solve(bmat, rhs)[:, :nh, 0]
    return torch.einsum("bh,bhmn->bmn", w, f)


@pytest.mark.parametrize("with_rho", [False, True])
def test_scf_post_ring_diis_matches_list_diis(with_rho):
    g = torch.Generator().manual_seed(7)
    nb, n, x, hist = 3, 9, 5, 4

    def sym(*shape):
        a = torch.randn(*shape, dtype=torch.float64, generator=g)
        return a + a.transpose(-1, -2)

    h, s_ = sym(nb, n, n), sym(nb, n, n) + 20 * torch.eye(n, dtype=torch.float64)
    xo = torch.randn(nb, n, n, dtype=torch.float64, generator=g)
    enuc = torch.randn(nb, dtype=torch.float64, generator=g)
    post = scf._SCFPost(nb, n, x, hist, with_rho, "cpu")
    post.load(h, s_, xo, enuc)
    errs, focks = [], []
    for it in range(7):  # wraps the ring
        j, k, d = sym(nb, n, n), sym(nb, n, n), sym(nb, n, n)
        rho = torch.randn(nb, x, dtype=torch.float64, generator=g)
        f, energy, cmax, f_ext = post.run(j, k, d, rho if with_rho else None)
        f_ref = h + j - 0.5 * k
        fds = f_ref @ d @ s_
        comm = fds - fds.transpose(1, 2)
        errs.append(xo.transpose(1, 2) @ comm @ xo)
        focks.append(f_ref)
        errs, focks = errs[-hist:], focks[-hist:]
        ext_ref = _reference_diis(errs, focks) if len(errs) > 1 else f_ref
        if with_rho:
            e_ref = (torch.einsum("bmn,bmn->b", d, h) + 0.5 * (rho * rho).sum(1)
                     - 0.25 * torch.einsum("bmn,bmn->b", d, k) + enuc)
        else:
            e_ref = 0.5 * torch.einsum("bmn,bmn->b", d, h + f_ref) + enuc
        assert torch.allclose(f, f_ref, atol=1e-12)
        assert torch.allclose(energy, e_ref, atol=1e-10)
        assert torch.allclose(cmax, comm.abs().amax(dim=(1, 2)), atol=1e-10)
        assert torch.allclose(f_ext, ext_ref, rtol=1e-8, atol=1e-8)


def test_chunk_precision_respects_mixed_kernel_limits():
    from vibeqc_b200.calculator import chunk_precision

    assert chunk_precision("mixed", 384, 80) == "mixed"
    assert chunk_precision("mixed", 512, 128) == "mixed"
    assert chunk_precision("mixed", 513, 80) == "fp64"   # FP32 B rows beyond 512
    assert chunk_precision("mixed", 400, 129) == "fp64"  # MMA N beyond 128
    assert chunk_precision("fp64", 100, 10) == "fp64"

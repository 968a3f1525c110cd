"""Analytic DF-RHF nuclear gradient on the GPU.

Reverse weights (reference ``src/scf/density_fitting.cpp:464-594`` and
``docs/developer/df_derivatives.md:89-104``), with (c_J, c_K) = (1, 1/4):

    Abar[mu nu, P] = D[mu nu] c[P] - 1/2 sum_Q Minv[P Q] (D A_Q D)[mu nu]
                   = D[mu nu] c[P] - 2 sum_ij C[mu i] C[nu j] Gamma[ij, P]
    Mbar           = -Minv Mbar+ Minv,   Mbar+ = rho rho^T / 2 - Q / 4
                   = -c c^T / 2 + sum_ij Gamma[ij, P] Gamma[ij, Q]

with c = Minv rho, Gamma[ij, P] = sum_Q M^{-1/2}[P Q] B[ij, Q] and
B[ij, Q] = sum_{mu nu} C[mu i] C[nu j] B[mu nu, Q].  The contractions with the
derivative integrals run in the native kernels (vqc_grad3c/2c/1e); forces are
F = -(g_1e + g_DF + dE_nn/dR) (``src/scf/rhf.cpp:856-868``).

At full rank Mbar = -Minv Mbar+ Minv.  When the eigenvalue cutoff removed
auxiliary functions (rank < X), the energy depends on M through the
thresholded pseudoinverse and Mbar is its spectral adjoint (Daleckii-Krein
divided differences; reference ``src/integrals/density_fitting_metric.cpp:
50-99`` and ``src/tensor/symmetric_matrix_function.cpp:62``), which needs
Mbar+ in the raw basis, including the components along discarded
eigenvectors: the raw 3-centre tensor is recomputed for such chunks.  An
eigenvalue within 128 eps lambda_max of the cutoff is a rank crossing and the
forces fail (numerical failure), as in the reference.
"""

from __future__ import annotations

import torch

from . import _lib
from .jk import unpack_index
from .timing import TIMER


WEIGHT_ROW_BLOCK = 32  # AO rows per block of the packed Abar assembly
SYM_BLOCK = 256  # row block of the triangular and symmetric products


def _upper_times(w: torch.Tensor, g: torch.Tensor) -> torch.Tensor:
    """W @ g per molecule for upper-triangular W (b, X, X): row block r needs rows >= r0 of g."""
    x = w.shape[1]
    out = torch.empty(g.shape[0], x, g.shape[2], dtype=g.dtype, device=g.device)
    for r0 in range(0, x, SYM_BLOCK):
        r1 = min(x, r0 + SYM_BLOCK)
        out[:, r0:r1] = torch.bmm(w[:, r0:r1, r0:], g[:, r0:])
    return out


def _sym_gram(g: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
    """g g^T per molecule from the upper block triangle (mirrored)."""
    x = g.shape[1]
    for r0 in range(0, x, SYM_BLOCK):
        r1 = min(x, r0 + SYM_BLOCK)
        blk = torch.bmm(g[:, r0:r1], g[:, r0:].transpose(1, 2))
        out[:, r0:r1, r0:] = blk
        out[:, r1:, r0:r1] = blk[:, :, r1 - r0:].transpose(1, 2)
    return out


_BLOCK_INDEX: dict = {}


def _block_rows(n: int, m0: int, m1: int, device) -> torch.Tensor:
    """Positions of the packed rows (mu in [m0, m1), nu <= mu) in a (m1-m0, m1) block."""
    key = (n, m0, m1, str(device))
    idx = _BLOCK_INDEX.get(key)
    if idx is None:
        mu = torch.arange(m0, m1, device=device)
        nu = torch.arange(m1, device=device)
        keep = nu[None, :] <= mu[:, None]
        idx = ((mu[:, None] - m0) * m1 + nu[None, :])[keep]
        _BLOCK_INDEX[key] = idx
    return idx


def chunk_weights(c: torch.Tensor, dens: torch.Tensor, rho: torch.Tensor, u: torch.Tensor,
                  w: torch.Tensor, upper: bool, abar: torch.Tensor | None = None,
                  mbar: torch.Tensor | None = None, k_scale: float = 1.0,
                  coulomb: bool = True):
    """Packed Abar (b, N(N+1)/2, X) and Mbar (b, X, X) for b molecules at once.

    c (b, N, o) occupied factors (D = 2 c c^T), rho (b, X) whitened fitted
    densities, u (b, N, o, X) = B C (whitened), w (b, X, X) whitening factors
    (upper triangular when ``upper``).  Abar rows are the packed pairs
    mu >= nu in row-major order; each block of AO rows mu is one batched GEMM
    over nu < m1 followed by the rank-one D (x) c term, so the full N*N*X
    tensor is never formed.  Every product is a batched GEMM over the b
    molecules (a handful of launches per chunk instead of per molecule).

    ``k_scale`` multiplies the exchange terms (1 for the restricted energy;
    2 for one spin channel of an unrestricted one, whose factor is
    C_s / sqrt(2)).  With ``coulomb`` False only the exchange terms of c are
    added to the given ``abar`` and ``mbar`` (a further spin channel).
    """
    b, n, o, x = u.shape
    # C^T B_Q C: [i][j][Q] from one GEMM, then [Q][i][j]
    bij = torch.bmm(c.transpose(1, 2), u.reshape(b, n, o * x)).view(b, o, o, x)
    bij = bij.permute(0, 3, 1, 2).reshape(b, x, o * o)
    gam = _upper_times(w, bij) if upper else torch.bmm(w, bij)  # Gamma[P, ij]
    del bij
    # T[i][nu][P] = sum_j C[nu, j] Gamma[P, i, j]
    t = torch.bmm(gam.view(b, x * o, o), c.transpose(1, 2))  # [P][i][nu]
    t1 = t.view(b, x, o, n).permute(0, 2, 3, 1).reshape(b, o, n * x)
    del t
    if abar is None:
        abar = torch.empty(b, n * (n + 1) // 2, x, dtype=u.dtype, device=u.device)
    if mbar is None:
        mbar = torch.empty(b, x, x, dtype=u.dtype, device=u.device)
    if coulomb:
        cvec = torch.bmm(w, rho[:, :, None])[:, :, 0]  # raw-basis fitting coefficients Minv rho
        mu_all, nu_all = torch.tril_indices(n, n, device=u.device)
        dpairs = dens[:, mu_all, nu_all]
    for m0 in range(0, n, WEIGHT_ROW_BLOCK):
        m1 = min(n, m0 + WEIGHT_ROW_BLOCK)
        blk = torch.bmm(c[:, m0:m1], t1[:, :, : m1 * x]).view(b, -1, x)  # (mu) x (nu < m1, P)
        p0, p1 = m0 * (m0 + 1) // 2, m1 * (m1 + 1) // 2
        rows = blk[:, _block_rows(n, m0, m1, u.device)]
        if coulomb:
            abar[:, p0:p1] = torch.baddbmm(rows, dpairs[:, p0:p1, None], cvec[:, None, :],
                                           beta=-2.0 * k_scale, alpha=1.0)
        else:
            abar[:, p0:p1].add_(rows, alpha=-2.0 * k_scale)
    if coulomb:
        _sym_gram(gam, mbar)
        if k_scale != 1.0:
            mbar.mul_(k_scale)
        mbar.baddbmm_(cvec[:, :, None], cvec[:, None, :], alpha=-0.5)
    else:
        g2 = torch.empty_like(mbar)
        _sym_gram(gam, g2)
        mbar.add_(g2, alpha=k_scale)
    return abar, mbar


WEIGHT_GROUP_BYTES = 4 << 30  # molecules per batched weight group: ~4 GB of (o, N, X) temporaries


DOUBLE_EPS = 2.220446049250313e-16


def spectral_metric_adjoint(lam: torch.Tensor, vec: torch.Tensor, keep: torch.Tensor,
                            mbar_plus: torch.Tensor, relative_threshold: float) -> torch.Tensor:
    """Adjoint of M -> thresholded pseudoinverse for one molecule (FP64, on the device).

    f(l) = 1/l on the retained eigenvalues and 0 on the discarded ones;
    Mbar = V ((V^T Mbar+ V) o G) V^T with G_ij = (f(l_i) - f(l_j)) / (l_i - l_j)
    and f' on (numerically) equal pairs.  Raises on an eigenvalue within
    128 eps lambda_max of the cutoff (reference
    ``density_fitting_metric.cpp:74-83``).
    """
    lmax = float(lam[-1])
    cut = relative_threshold * lmax
    if bool(((lam - cut).abs() <= 128 * DOUBLE_EPS * lmax).any()):
        raise _lib.VqcError(5, "DF metric rank crossing: eigenvalue is unresolved at the cutoff")
    safe = torch.where(keep, lam, torch.ones_like(lam))
    fl = torch.where(keep, 1.0 / safe, torch.zeros_like(lam))
    dl = lam[:, None] - lam[None, :]
    same = dl.abs() <= 1e-14 * lmax
    gam = (fl[:, None] - fl[None, :]) / torch.where(same, torch.ones_like(dl), dl)
    deriv = torch.where(keep, -1.0 / (safe * safe), torch.zeros_like(lam))
    gam = torch.where(same, 0.5 * (deriv[:, None] + deriv[None, :]), gam)
    return vec @ ((vec.transpose(0, 1) @ mbar_plus @ vec) * gam) @ vec.transpose(0, 1)


def _raw_mbar_plus(a_raw_packed: torch.Tensor, channels, n: int) -> torch.Tensor:
    """Mbar+ = rho rho^T / 2 - sum_(c, k) k sum_ij A_ij A_ij^T in the raw auxiliary basis.

    ``channels``: (c (N, o), k) pairs for one molecule, D = 2 c c^T per channel
    (k = 1 restricted; k = 2 per spin channel C_s / sqrt(2) of an unrestricted
    density); A_ij[P] = sum_{mu nu} c[mu i] c[nu j] (mu nu|P) and
    rho = sum over channels of 2 sum_i A_ii.
    """
    x = a_raw_packed.shape[1]
    a_full = a_raw_packed[unpack_index(n, a_raw_packed.device)]  # (N*N, X)
    rho = torch.zeros(x, dtype=a_full.dtype, device=a_full.device)
    quad = torch.zeros(x, x, dtype=a_full.dtype, device=a_full.device)
    for c, k in channels:
        o = c.shape[1]
        ui = (c.transpose(0, 1) @ a_full.view(n, n * x)).view(o, n, x)  # [i][nu][P]
        aij = torch.einsum("nj,inp->ijp", c, ui).reshape(o * o, x)
        rho += 2.0 * aij.view(o, o, x).diagonal(dim1=0, dim2=1).sum(dim=1)
        quad += k * (aij.transpose(0, 1) @ aij)
    return 0.5 * torch.outer(rho, rho) - quad


def df_rhf_gradient(chunk, ints, scf_out: dict, xyz: torch.Tensor) -> torch.Tensor:
    """Positive energy gradient, (natom_total_of_chunk, 3)."""
    dens = scf_out["density"]
    c = scf_out["orbitals"]  # AO occupied factor, dens = 2 c c^T
    # energy-weighted density of the converged closed shell: W = D F D / 2
    wdens = 0.5 * dens @ scf_out["fock"] @ dens
    if scf_out.get("exact_half") is not None:
        half = scf_out["exact_half"]  # FP64 U = B C already formed for the energy
    else:
        half = scf_out["jk"].half_transform(c)  # fitted density and U = B C
    return _df_gradient(chunk, scf_out, xyz, dens, wdens, [(c, half, 1.0)])


def df_uhf_gradient(chunk, ints, scf_out: dict, xyz: torch.Tensor) -> torch.Tensor:
    """Positive unrestricted energy gradient, (natom_total_of_chunk, 3).

    Reverse weights as the reference's unrestricted weighted gradient
    (``src/scf/density_fitting.cpp:919-944``): Coulomb on D_a + D_b, exchange
    per spin density; energy-weighted density W = sum_s D_s F_s D_s.
    """
    ds = scf_out["spin_densities"]
    cs = scf_out["orbitals"]  # channel factors C_s / sqrt(2), D_s = 2 c_s c_s^T
    dens = ds[0] + ds[1]
    wdens = sum(d @ f @ d for d, f in zip(ds, scf_out["fock"]))
    halves = scf_out.get("exact_half")
    if halves is None:
        halves = [scf_out["jk"].half_transform(c) for c in cs]
    return _df_gradient(chunk, scf_out, xyz, dens, wdens,
                        [(c, half, 2.0) for c, half in zip(cs, halves)])


def _df_gradient(chunk, scf_out, xyz, dens, wdens, channels) -> torch.Tensor:
    """Weights from ``channels`` [(c, (rho, U = B c), k_scale)], then the derivative contractions."""
    plan = chunk.plan
    nb, n, x = chunk.nb, chunk.nao, chunk.naux
    dev = xyz.device
    mf = scf_out["metric"]
    jk = scf_out["jk"]
    truncated = [m for m in range(nb) if mf.rank[m] < x]
    o = channels[0][0].shape[2]
    wctx = TIMER.stage("grad_weights")
    wctx.__enter__()
    rho_all = sum(half[0] for _, half, _ in channels)
    abar = torch.empty(nb, n * (n + 1) // 2, x, dtype=torch.float64, device=dev)
    mbar = torch.empty(nb, x, x, dtype=torch.float64, device=dev)
    tri = mf.kind == "cholesky"
    grp = max(1, WEIGHT_GROUP_BYTES // max(1, 8 * n * o * x))
    for g0 in range(0, nb, grp):  # groups of molecules: bounded temporaries
        g1 = min(nb, g0 + grp)
        for ch, (c, (_, u_all), k) in enumerate(channels):
            chunk_weights(c[g0:g1], dens[g0:g1], rho_all[g0:g1], u_all[g0:g1], mf.inv_sqrt[g0:g1],
                          tri, abar[g0:g1], mbar[g0:g1], k_scale=k, coulomb=ch == 0)
    if truncated:
        # the whitened tensor is no longer needed: recompute the raw one for
        # the spectral response of the truncated metrics
        channels = [(c, None, k) for c, _, k in channels]
        jk.release_all()
        from .scf import compute_integrals

        a_raw = compute_integrals(plan, xyz).a_packed
        for m in truncated:
            mbp = _raw_mbar_plus(a_raw[m], [(c[m], k) for c, _, k in channels], n)
            mbar[m] = spectral_metric_adjoint(mf.eigenvalues[m], mf.eigenvectors[m], mf.keep[m], mbp,
                                              scf_out["relative_threshold"])
        del a_raw
    wctx.__exit__(None, None, None)
    grad = torch.zeros(plan.natom * 3, dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    with TIMER.stage("grad1e"):
        _lib.call("vqc_grad1e", plan.handle, xyz.data_ptr(), dens.contiguous().data_ptr(),
                  wdens.contiguous().data_ptr(), grad.data_ptr(), st)
    with TIMER.stage("grad3c"):
        _lib.call("vqc_grad3c", plan.handle, xyz.data_ptr(), abar.data_ptr(), grad.data_ptr(), st)
    with TIMER.stage("grad2c"):
        _lib.call("vqc_grad2c", plan.handle, xyz.data_ptr(), mbar.contiguous().data_ptr(),
                  grad.data_ptr(), st)
    grad = grad.view(-1, 3)
    from .scf import nuclear_repulsion

    off = 0
    for i, z in enumerate(scf_out["charges"]):
        na = len(z)
        _, gn = nuclear_repulsion(z, xyz[off:off + na])
        grad[off:off + na] += gn
        off += na
    return grad


def df_gradient_host(molecule, bar_a, bar_m, *, spherical: bool = True,
                     maximum_bytes: int = 1 << 32, maximum_tile_elements: int = 0,
                     schedule: int = 0, out=None):
    """DF part of an energy gradient from fixed external weights, host in and out.

    The contract of the reference's ``generativeqc_system_df_gradient_cuda``
    (``include/generativeqc/generativeqc.h:1312-1333``) through
    ``vqc_df_gradient``: ``bar_a`` full (N, N, X) and ``bar_m`` full (X, X)
    FP64 arrays (either may be None for a zero channel; nonsymmetric weights
    are allowed and every element counts once), auxiliary functions in the
    molecule's order (shells sorted by angular momentum).  Returns
    ``(gradient (natom, 3), resources dict)``; when ``out`` is given the
    gradient is written into it, and only on success.
    """
    import ctypes

    import numpy as np

    from .plan import batch_descriptor

    desc, keep = batch_descriptor([molecule], spherical)
    xyz = np.ascontiguousarray(molecule.coordinates, dtype=np.float64)
    natom = xyz.shape[0]
    a = None if bar_a is None else np.ascontiguousarray(bar_a, dtype=np.float64)
    m = None if bar_m is None else np.ascontiguousarray(bar_m, dtype=np.float64)
    from . import basis as bas

    n = bas.count_functions(molecule.orbital_shells, spherical)
    x = bas.count_functions(molecule.aux_shells, spherical)
    count_a = n * n * x if a is None else a.size
    count_m = x * x if m is None else m.size
    grad = np.zeros((natom, 3)) if out is None else out
    if grad.dtype != np.float64 or not grad.flags.c_contiguous or grad.size != 3 * natom:
        raise ValueError("out must be a C-contiguous float64 array of 3 * natom values")
    res = _lib.DfGradientResources()
    res.struct_size = ctypes.sizeof(_lib.DfGradientResources)
    res.abi_version = _lib.ABI_VERSION
    ptr = lambda v: None if v is None else v.ctypes.data  # noqa: E731
    _lib.call("vqc_df_gradient", ctypes.byref(desc), ptr(xyz), ptr(a), count_a, ptr(m), count_m,
              schedule, maximum_bytes, maximum_tile_elements, grad.ctypes.data, grad.size,
              ctypes.byref(res))
    del keep
    rec = {name: int(getattr(res, name)) for name, _ in _lib.DfGradientResources._fields_[2:]}
    return grad.reshape(natom, 3), rec

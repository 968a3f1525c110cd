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

The full-rank form of Mbar is used; a metric whose eigenvalue cutoff removed
functions is rejected for forces (numerical failure), as the thresholded
spectral response needs the discarded components of the raw 3-centre tensor.
"""

from __future__ import annotations

import torch

from . import _lib
from .jk import unpack_index
from .timing import TIMER


def _packed_rows(n: int, device) -> torch.Tensor:
    """Row-major (mu >= nu) positions in the N*N square for every packed row."""
    mu, nu = torch.tril_indices(n, n, device=device)
    return mu * n + nu


def df_rhf_gradient(chunk, ints, scf_out: dict, xyz: torch.Tensor) -> torch.Tensor:
    """Positive energy gradient, (natom_total_of_chunk, 3)."""
    plan = chunk.plan
    nb, n, x, o = chunk.nb, chunk.nao, chunk.naux, chunk.nocc
    dev = xyz.device
    mf = scf_out["metric"]
    if any(r < x for r in mf.rank):
        raise _lib.VqcError(5, "analytic forces need a full-rank auxiliary metric")
    d0 = scf_out["density"]
    jk = scf_out["jk"]
    # final Fock at the returned density -> orbitals, energy-weighted density
    c_prev = scf_out.get("orbitals")
    j, k = jk.build(d0, c_prev[:, :, :o]) if c_prev is not None else jk.build(d0, None)
    f = ints.h + j - 0.5 * k
    xo = scf_out["orthogonalizer"]
    eps, cp = torch.linalg.eigh(xo.transpose(1, 2) @ f @ xo)
    c = (xo @ cp)[:, :, :o]
    dens = 2.0 * c @ c.transpose(1, 2)
    wdens = 2.0 * (c * eps[:, None, :o]) @ c.transpose(1, 2)

    wctx = TIMER.stage("grad_weights")
    wctx.__enter__()
    b = jk.whitened_fp64()  # (nb, N*N, X) whitened, FP64
    rho_w = torch.bmm(dens.reshape(nb, 1, n * n), b)[:, 0, :]  # (nb, X)
    cvec = torch.bmm(mf.inv_sqrt, rho_w[:, :, None])[:, :, 0]  # raw-basis c = Minv rho
    # B[ij, Q]: half transform then quarter transform
    b4 = b.view(nb, n, n, x)
    u = torch.matmul(b4.transpose(2, 3), c[:, None, :, :])  # (nb, N(mu), X, o(j))
    bij = torch.einsum("bmi,bmqj->bqij", c, u)  # (nb, X, o, o)
    del u
    gam = torch.bmm(mf.inv_sqrt, bij.reshape(nb, x, o * o)).view(nb, x, o, o)
    # Abar (full square), then packed rows
    t1 = torch.einsum("bnj,bpij->bpin", c, gam)  # (nb, X, o, N)
    abar_sq = torch.einsum("bmi,bpin->bmnp", c, t1)  # (nb, N, N, X)
    del t1
    abar_sq = dens[:, :, :, None] * cvec[:, None, None, :] - 2.0 * abar_sq
    rows = _packed_rows(n, dev)
    abar = abar_sq.reshape(nb, n * n, x)[:, rows, :].contiguous()
    del abar_sq
    gflat = gam.reshape(nb, x, o * o)
    mbar = -0.5 * cvec[:, :, None] * cvec[:, None, :] + torch.bmm(gflat, gflat.transpose(1, 2))

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

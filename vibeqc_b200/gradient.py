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
    dens = scf_out["density"]
    c = scf_out["orbitals"]  # AO occupied factor, dens = 2 c c^T
    f = scf_out["fock"]
    jk = scf_out["jk"]
    # energy-weighted density of the converged closed shell: W = D F D / 2
    wdens = 0.5 * dens @ f @ dens

    wctx = TIMER.stage("grad_weights")
    wctx.__enter__()
    if scf_out.get("exact_half") is not None:
        rho_all, u_all = scf_out["exact_half"]  # FP64 U = B C already formed for the energy
    else:
        rho_all, u_all = jk.half_transform(c)  # fitted density and U = B C
    rows = _packed_rows(n, dev)
    abar = torch.empty(nb, rows.numel(), x, dtype=torch.float64, device=dev)
    mbar = torch.empty(nb, x, x, dtype=torch.float64, device=dev)
    for m in range(nb):  # per molecule: bounded temporaries
        cvec = mf.inv_sqrt[m] @ rho_all[m]  # raw-basis c = Minv rho
        u = u_all[m].to(torch.float64)  # (N(mu), X, o(j))
        bij = torch.einsum("mi,mqj->qij", c[m], u)  # (X, o, o)
        del u
        gam = (mf.inv_sqrt[m] @ bij.reshape(x, o * o)).view(x, o, o)
        t1 = torch.einsum("nj,pij->inp", c[m], gam).reshape(o, n * x)  # (o, N*X)
        sq = (c[m] @ t1).view(n * n, x)  # (N*N, X) = sum_i C[mu i] T[i, nu, P]
        del t1
        sq = dens[m].reshape(n * n, 1) * cvec[None, :] - 2.0 * sq
        abar[m] = sq[rows]
        del sq
        gflat = gam.reshape(x, o * o)
        mbar[m] = -0.5 * torch.outer(cvec, cvec) + gflat @ gflat.T
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

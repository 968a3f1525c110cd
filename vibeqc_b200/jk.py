"""Coulomb (J) and exchange (K) builders over the whitened DF tensor B.

``fp64``: the plain FP64 GPU path (cuBLAS DGEMM/DGEMV through torch), the
comparator the mixed path is measured against.  J = B (B^T d) as in
``src/scf/cuda/df_coulomb.cpp:24``; occupied-factor K = 2 sum_Q (B_Q C)(B_Q C)^T
as in ``src/scf/cuda/df_occupied_exchange.cpp:191-300``.
"""

from __future__ import annotations

import torch

from .timing import TIMER


def unpack_index(n: int, device) -> torch.Tensor:
    mu = torch.arange(n, device=device)
    hi = torch.maximum(mu[:, None], mu[None, :])
    lo = torch.minimum(mu[:, None], mu[None, :])
    return (hi * (hi + 1) // 2 + lo).reshape(-1)


class FP64Builder:
    """Full (mu, nu, Q) FP64 storage; J by GEMV, K by two DGEMMs."""

    precision = "fp64"

    def __init__(self, b_packed: torch.Tensor, n: int, x: int, nocc: int):
        idx = unpack_index(n, b_packed.device)
        self.n, self.x, self.nocc = n, x, nocc
        self.b = b_packed[:, idx, :].contiguous()  # (nb, N*N, X)
        self.nbuild = 0

    def build(self, d: torch.Tensor, c_occ: torch.Tensor):
        nb, n, x, o = d.shape[0], self.n, self.x, self.nocc
        b = self.b
        with TIMER.stage("J_fp64"):
            rho = torch.bmm(d.reshape(nb, 1, n * n), b)  # (nb, 1, X)
            j = torch.bmm(b, rho.transpose(1, 2)).reshape(nb, n, n)
        with TIMER.stage("K_fp64"):
            # U[b, mu, Q, i] = sum_nu B[mu, nu, Q] C[nu, i]
            b4 = b.view(nb, n, n, x)
            u = torch.matmul(b4.transpose(2, 3), c_occ[:, None, :, :])  # (nb, N, X, o)
            u = u.reshape(nb, n, x * o)
            k = 2.0 * torch.bmm(u, u.transpose(1, 2))
        self.nbuild += 1
        return j, k

    def whitened_fp64(self) -> torch.Tensor:
        return self.b


def make_builder(precision: str, b_packed: torch.Tensor, n: int, x: int, nocc: int):
    if precision == "fp64":
        return FP64Builder(b_packed, n, x, nocc)
    raise ValueError(f"unknown precision {precision!r}")

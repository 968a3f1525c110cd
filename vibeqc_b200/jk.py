"""Coulomb (J) and exchange (K) builders over the whitened DF tensor B.

``fp64``: the plain FP64 GPU path (cuBLAS DGEMM/DGEMV through torch), the
comparator the mixed path is measured against.  J = B (B^T d) as in
``src/scf/cuda/df_coulomb.cpp:24``; occupied-factor K = 2 sum_Q (B_Q C)(B_Q C)^T
as in ``src/scf/cuda/df_occupied_exchange.cpp:191-300``.

``mixed``: B stored once in FP32 (aux-major per AO row); the exchange half
transform U = B C and the Gram product K = 2 U U^T run on the tcgen05 tensor
cores in split precision (3xTF32: round-to-nearest hi/lo parts, FP32
accumulation drained to FP64); the fitted density rho = B^T d and J = B rho
stream the FP32 B with FP64 accumulation.  The FP64 tensor stays resident for
the finishing iterations, the final energy and the gradient.
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

    def build_exact(self, d: torch.Tensor, c_occ: torch.Tensor):
        return self.build(d, c_occ)


    def half_transform(self, c_occ: torch.Tensor):
        """(rho_whitened (nb, X), U (nb, N, X, o)) for D = 2 C C^T."""
        nb, n, x, o = c_occ.shape[0], self.n, self.x, self.nocc
        b4 = self.b.view(nb, n, n, x)
        u = torch.matmul(b4.transpose(2, 3), c_occ[:, None, :, :])  # (nb, N, X, o)
        rho = 2.0 * torch.einsum("bmi,bmqi->bq", c_occ, u)
        return rho, u


def _round_up(v: int, m: int) -> int:
    return (v + m - 1) // m * m


class MixedBuilder:
    """FP32 B (aux-major per AO row) with tcgen05 3xTF32 exchange."""

    precision = "mixed"

    def __init__(self, b_packed: torch.Tensor, n: int, x: int, nocc: int):
        from . import _lib

        self._lib = _lib
        nb = b_packed.shape[0]
        self.nb, self.n, self.x, self.nocc = nb, n, x, nocc
        self.ld = _round_up(n, 4)
        self.o_pad = _round_up(nocc, 16)
        if self.o_pad > 128:
            raise _lib.VqcError(1, "mixed exchange supports at most 128 occupied orbitals")
        dev = b_packed.device
        self.b = torch.empty(nb, n, x, self.ld, dtype=torch.float32, device=dev)
        self.st = torch.cuda.current_stream().cuda_stream
        _lib.call("vqc_unpack_aux_major", b_packed.contiguous().data_ptr(), nb, n, x, self.ld,
                  self.b.data_ptr(), self.st)
        # U[mol][mu][i][Q] split into TF32 hi/lo parts; Q rows padded to ldq
        self.ldq = _round_up(x, 4)
        self.u_hi = torch.zeros(nb, n, nocc, self.ldq, dtype=torch.float32, device=dev)
        self.u_lo = torch.zeros_like(self.u_hi)
        self.rho = torch.empty(nb, x, dtype=torch.float64, device=dev)
        # the FP64 whitened tensor stays resident (full rows, as on the FP64
        # path) for the FP64 finishing iterations, the final energy and the
        # gradient weights
        self.b64 = b_packed[:, unpack_index(n, dev), :].contiguous()  # (nb, N*N, X)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.nbuild = 0

    def _check(self):
        if int(self.err.item()) != 0:
            raise self._lib.VqcError(6, f"tensor-core kernel wait expired (code {int(self.err.item())})")

    def _half(self, c_occ: torch.Tensor):
        nb, n, o = self.nb, self.n, self.nocc
        ct = torch.zeros(nb, o, self.ld, dtype=torch.float32, device=c_occ.device)
        ct[:, :, :n] = c_occ.transpose(1, 2)
        ct_hi = torch.empty_like(ct)
        ct_lo = torch.empty_like(ct)
        self._lib.call("vqc_split_tf32", ct.data_ptr(), ct_hi.data_ptr(), ct_lo.data_ptr(),
                       ct.numel(), self.st)
        c64 = c_occ.contiguous()
        with TIMER.stage("K_half_tc"):
            self._lib.call("vqc_tc_half_transform", self.b.data_ptr(), nb, n, self.ld, self.x,
                           ct_hi.data_ptr(), ct_lo.data_ptr(), c64.data_ptr(), o, self.o_pad,
                           self.ldq, self.u_hi.data_ptr(), self.u_lo.data_ptr(), 0,
                           self.err.data_ptr(), self.st)

    def build(self, d: torch.Tensor, c_occ: torch.Tensor):
        nb, n = self.nb, self.n
        self._half(c_occ)
        j = torch.empty(nb, n, n, dtype=torch.float64, device=d.device)
        with TIMER.stage("J_fp32"):
            # fitted density from the FP32 B with FP64 accumulation (no
            # tensor-core accumulation error in J), then J = B rho
            dd = d.contiguous()
            self._lib.call("vqc_fitted_density_fp32", self.b.data_ptr(), dd.data_ptr(), nb, n,
                           self.ld, self.x, self.rho.data_ptr(), self.st)
            self._lib.call("vqc_coulomb_fp32", self.b.data_ptr(), self.rho.data_ptr(), nb, n,
                           self.ld, self.x, j.data_ptr(), self.st)
        k = torch.zeros(nb, n, n, dtype=torch.float64, device=d.device)
        with TIMER.stage("K_gram_tc"):
            self._lib.call("vqc_tc_gram", self.u_hi.data_ptr(), self.u_lo.data_ptr(), nb, n,
                           self.nocc * self.ldq, k.data_ptr(), self.err.data_ptr(), self.st)
        self.nbuild += 1
        self._check()
        return j, 2.0 * k

    def build_exact(self, d: torch.Tensor, c_occ: torch.Tensor):
        """FP64 K and FP64-density J for the finishing iterations.

        K = 2 U U^T with U = B C in FP64 from the FP64 tensor; J streams the
        FP32 B with the exact fitted density (the energy reported at the end is
        re-evaluated fully in FP64, so the FP32 storage of B in J only shifts
        the converged density at second order in the energy).
        """
        nb, n, x, o = self.nb, self.n, self.x, self.nocc
        rho, u = self.half_transform(c_occ)
        j = torch.empty(nb, n, n, dtype=torch.float64, device=d.device)
        with TIMER.stage("J_fp32"):
            self._lib.call("vqc_coulomb_fp32", self.b.data_ptr(), rho.data_ptr(), nb, n,
                           self.ld, x, j.data_ptr(), self.st)
        with TIMER.stage("K_exact_fp64"):
            uf = u.reshape(nb, n, x * o)
            k = 2.0 * torch.bmm(uf, uf.transpose(1, 2))
        self.nbuild += 1
        return j, k

    def half_transform(self, c_occ: torch.Tensor):
        """FP64 (rho_whitened (nb, X), U (nb, N, X, o)) from the FP64 whitened tensor.

        Used by the finishing iterations, the final energy and the gradient
        weights, so the reported energy and forces carry no FP32 storage or
        tensor-core error.
        """
        nb, n, x = self.nb, self.n, self.x
        with TIMER.stage("exact_half_fp64"):
            b4 = self.b64.view(nb, n, n, x)
            u = torch.matmul(b4.transpose(2, 3), c_occ[:, None, :, :])  # (nb, N, X, o)
            rho = 2.0 * torch.einsum("bmi,bmqi->bq", c_occ, u)
        return rho, u


def make_builder(precision: str, b_packed: torch.Tensor, n: int, x: int, nocc: int):
    if precision == "fp64":
        return FP64Builder(b_packed, n, x, nocc)
    if precision == "mixed":
        return MixedBuilder(b_packed, n, x, nocc)
    raise ValueError(f"unknown precision {precision!r}")

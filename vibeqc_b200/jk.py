"""Coulomb (J) and exchange (K) builders over the whitened DF tensor B.

``fp64``: the plain FP64 GPU path (cuBLAS DGEMM/DGEMV through torch), the
comparator the mixed path is measured against.  J = B (B^T d) as in
``src/scf/cuda/df_coulomb.cpp:24``; occupied-factor K = 2 sum_Q (B_Q C)(B_Q C)^T
as in ``src/scf/cuda/df_occupied_exchange.cpp:191-300``.

``mixed``: B stored once in FP32 (aux-major per AO row); the exchange half
transform U = B C and the Gram product K = 2 U U^T run on the tcgen05 tensor
cores in split precision (3xTF32: round-to-nearest hi/lo parts, FP32
accumulation drained to FP64); the fitted density rho = B^T d and J = B rho
stream the FP32 B with FP64 accumulation.  Once the SCF is close to
convergence the builds switch to increments about an FP64 anchor (see
``MixedBuilder.anchor``), so the converged J, K, energy and the gradient
operands carry FP64 accuracy.
"""

from __future__ import annotations

import torch

from .timing import TIMER


# algorithmic work of the tensor-core exchange since the last reset (host-side
# tallies, read by the benchmark): bytes the half transform must move (FP32 B
# read once, split U written), its launches, and the exchange flops counted
# once (half transform 2 N^2 X o, Gram X o N (N + 1) per term); "half_min_bytes"
# is the floor of a symmetric-packed kernel: the mu >= nu half of the FP32 B
# read once and U written once in FP32
COUNTERS = {"half_bytes": 0, "half_min_bytes": 0, "half_launches": 0, "k_flops": 0}


def reset_counters() -> None:
    for k in COUNTERS:
        COUNTERS[k] = 0


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

    def build(self, d: torch.Tensor, c_occ: torch.Tensor, with_j: bool = True):
        nb, n, x, o = d.shape[0], self.n, self.x, self.nocc
        b = self.b
        j = None
        if with_j:
            with TIMER.stage("J_fp64"):
                rho = torch.bmm(d.reshape(nb, 1, n * n), b)  # (nb, 1, X)
                j = torch.bmm(b, rho.transpose(1, 2)).reshape(nb, n, n)
        with TIMER.stage("K_fp64"):
            # U[i][mu][Q] = sum_nu C[nu, i] B[nu, mu Q] (B symmetric in mu, nu),
            # K = 2 sum_i U_i U_i^T
            ui = torch.bmm(c_occ.transpose(1, 2), b.view(nb, n, n * x)).view(nb * o, n, x)
            k = 2.0 * torch.bmm(ui, ui.transpose(1, 2)).view(nb, o, n, n).sum(dim=1)
            del ui
        self.nbuild += 1
        return j, k

    def build_exact(self, d: torch.Tensor, c_occ: torch.Tensor, with_j: bool = True):
        return self.build(d, c_occ, with_j)

    def half_transform(self, c_occ: torch.Tensor):
        """(rho_whitened (nb, X), U (nb, N, o, X)) for D = 2 C C^T."""
        return fp64_half(self.b, c_occ, self.n, self.x)

    def release_all(self) -> None:
        """Drop the whitened tensor (no further builds)."""
        self.b = None


def fp64_half(b_full: torch.Tensor, c_occ: torch.Tensor, n: int, x: int):
    """FP64 U[mu][i][Q] = sum_nu B[mu nu, Q] C[nu, i] and rho = 2 sum C U.

    B is symmetric in (mu, nu), so B viewed as (nu, mu*Q) rows is one plain
    GEMM per molecule, C^T (o x N) times (N x N*X); the result [i][mu][Q] is
    permuted once to [mu][i][Q].
    """
    nb, o = c_occ.shape[0], c_occ.shape[2]
    ui = torch.bmm(c_occ.transpose(1, 2), b_full.view(nb, n, n * x)).view(nb, o, n, x)
    rho = 2.0 * torch.einsum("bmi,bimq->bq", c_occ, ui)
    return rho, ui.transpose(1, 2).contiguous()


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
        if self.ld > 512:
            raise _lib.VqcError(1, "mixed J/K support at most 512 orbital basis functions")
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
        # the FP64 whitened tensor stays resident (full rows: the anchor's half
        # transform is then one plain GEMM per molecule, measured 2.6x faster
        # than gathering from the packed rows)
        self.b64 = b_packed[:, unpack_index(n, dev), :].contiguous()  # (nb, N*N, X)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.v_hi = self.v_lo = None
        self._anc: dict = {}  # anchor state per channel (spin)
        self.nbuild = 0

    def _check(self):
        if int(self.err.item()) != 0:
            raise self._lib.VqcError(6, f"tensor-core kernel wait expired (code {int(self.err.item())})")

    def _half(self, c_occ: torch.Tensor, cvec: torch.Tensor | None = None,
              rho: torch.Tensor | None = None, dens: torch.Tensor | None = None,
              rho_dens: torch.Tensor | None = None):
        """U = B c_occ into u_hi/u_lo; rho += 2 sum_{mu,i} U cvec (when given);
        rho_dens += B^T vec(dens) from the same pass over B (when given)."""
        nb, n, o = self.nb, self.n, self.nocc
        ct = torch.zeros(nb, o, self.ld, dtype=torch.float32, device=c_occ.device)
        ct[:, :, :n] = c_occ.transpose(1, 2)
        ct_hi = torch.empty_like(ct)
        ct_lo = torch.empty_like(ct)
        self._lib.call("vqc_split_tf32", ct.data_ptr(), ct_hi.data_ptr(), ct_lo.data_ptr(),
                       ct.numel(), self.st)
        c64 = (c_occ if cvec is None else cvec).contiguous()
        COUNTERS["half_bytes"] += nb * n * self.x * self.ld * 4 + nb * n * o * self.ldq * 8
        COUNTERS["half_min_bytes"] += nb * (n * (n + 1) // 2 * self.x * 4 + n * o * self.x * 4)
        COUNTERS["half_launches"] += 1
        COUNTERS["k_flops"] += 2 * nb * n * n * self.x * o
        with TIMER.stage("K_half_tc"):
            self._lib.call("vqc_tc_half_transform", self.b.data_ptr(), nb, n, self.ld, self.x,
                           ct_hi.data_ptr(), ct_lo.data_ptr(), c64.data_ptr(), o, self.o_pad,
                           self.ldq, self.u_hi.data_ptr(), self.u_lo.data_ptr(),
                           0 if rho is None else rho.data_ptr(),
                           0 if dens is None else dens.data_ptr(),
                           0 if rho_dens is None else rho_dens.data_ptr(),
                           self.err.data_ptr(), self.st)

    def build(self, d: torch.Tensor, c_occ: torch.Tensor, with_j: bool = True):
        nb, n = self.nb, self.n
        j = None
        if with_j:
            # the fitted density rho = B^T vec(D) comes from the half
            # transform's own pass over the FP32 B (FP32 partial sums of the
            # exact FP32 values accumulated in FP64, no tensor-core
            # accumulation error in J), then J = B rho
            dd = d.contiguous()
            self.rho.zero_()
            self._half(c_occ, dens=dd, rho_dens=self.rho)
            j = torch.empty(nb, n, n, dtype=torch.float64, device=d.device)
            with TIMER.stage("J_fp32"):
                self._lib.call("vqc_coulomb_tma", self.b.data_ptr(), self.rho.data_ptr(), nb, n,
                               self.ld, self.x, j.data_ptr(), self.err.data_ptr(), self.st)
        else:
            self._half(c_occ)
        k = torch.zeros(nb, n, n, dtype=torch.float64, device=d.device)
        COUNTERS["k_flops"] += nb * self.x * self.nocc * n * (n + 1)
        with TIMER.stage("K_gram_tc"):
            self._lib.call("vqc_tc_gram", self.u_hi.data_ptr(), self.u_lo.data_ptr(), nb, n,
                           self.nocc * self.ldq, k.data_ptr(), self.err.data_ptr(), self.st)
        self.nbuild += 1
        self._check()
        return j, 2.0 * k

    def half_transform(self, c_occ: torch.Tensor):
        """FP64 (rho_whitened (nb, X), U (nb, N, o, X)) from the FP64 whitened tensor."""
        with TIMER.stage("exact_half_fp64"):
            return fp64_half(self.b64, c_occ, self.n, self.x)

    def release_all(self) -> None:
        """Drop every copy of the whitened tensor (no further builds)."""
        self.release_tensor_core_buffers()
        self.b64 = None

    def release_tensor_core_buffers(self) -> None:
        """Free the FP32 tensor and the split U/V buffers once the SCF is done."""
        self.b = self.u_hi = self.u_lo = None
        self.v_hi = self.v_lo = None

    # -- incremental builds about an FP64 anchor ---------------------------
    #
    # J and K are linear in D.  At the anchor D0 = 2 C0 C0^T they are formed
    # in FP64 (rho0, J0 = B rho0, U0 = B C0, K0 = 2 U0 U0^T).  Later
    # iterations take C close to C0 (the occupied factor is aligned to C0),
    # dC = C - C0, and only the increments run on the tensor cores:
    #     dU = B dC,  rho = rho0 + 4 sum (C0 + dC/2) dU,  J = J0 + B (rho - rho0)
    #     K = K0 + 2 (V dU^T + dU V^T),  V = U0 + dU / 2
    # so their split-precision error scales with |D - D0| instead of |D|, and
    # the converged operators are FP64-accurate.

    def anchor(self, d: torch.Tensor, c_occ: torch.Tensor, channel: int = 0, with_j: bool = True):
        """FP64 J/K at D0 = 2 C0 C0^T; later increments of ``channel`` are about it.

        Each channel (one per spin of an unrestricted SCF) keeps its own anchor;
        with ``with_j`` False the Coulomb matrix is not formed (returned as None).
        """
        nb, n, x, o = self.nb, self.n, self.x, self.nocc
        with TIMER.stage("anchor_fp64"):
            rho0, u0 = fp64_half(self.b64, c_occ, n, x)  # u0 (nb, N, o, X)
            uf = u0.view(nb, n, o * x)
            k0 = 2.0 * torch.bmm(uf, uf.transpose(1, 2))
            j0 = torch.bmm(self.b64, rho0[:, :, None]).view(nb, n, n) if with_j else None
        self._anc[channel] = {"c0": c_occ.clone(), "rho0": rho0, "j0": j0, "k0": k0, "u0": u0}
        if self.v_hi is None:
            self.v_hi = torch.empty_like(self.u_hi)
            self.v_lo = torch.empty_like(self.u_hi)
        self.nbuild += 1
        return j0, k0, rho0

    def _increment(self, c_occ: torch.Tensor, channel: int):
        """dU = B (C - C0) into u_hi/u_lo; returns rho - rho0."""
        c0 = self._anc[channel]["c0"]
        dc = c_occ - c0
        drho = torch.zeros(self.nb, self.x, dtype=torch.float64, device=c_occ.device)
        self._half(dc, cvec=c0 + 0.5 * dc, rho=drho)  # drho = 2 sum (C0 + dC/2) dU
        return 2.0 * drho

    def build_incremental(self, d: torch.Tensor, c_occ: torch.Tensor, channel: int = 0,
                          with_j: bool = True):
        nb, n, x, o = self.nb, self.n, self.x, self.nocc
        anc = self._anc[channel]
        drho = self._increment(c_occ, channel)
        j = None
        if with_j:
            dj = torch.empty(nb, n, n, dtype=torch.float64, device=d.device)
            with TIMER.stage("J_fp32"):
                self._lib.call("vqc_coulomb_tma", self.b.data_ptr(), drho.data_ptr(), nb, n,
                               self.ld, x, dj.data_ptr(), self.err.data_ptr(), self.st)
            j = anc["j0"] + dj
        COUNTERS["k_flops"] += 2 * nb * x * o * n * (n + 1)  # V dU^T + dU V^T
        with TIMER.stage("K_gram_tc"):
            self._lib.call("vqc_anchor_combine", anc["u0"].data_ptr(), self.u_hi.data_ptr(),
                           self.u_lo.data_ptr(), self.v_hi.data_ptr(), self.v_lo.data_ptr(),
                           nb * n * o, x, self.ldq, 0.5, 0, self.st)
            kh = 0.5 * anc["k0"]
            self._lib.call("vqc_tc_gram_sym2", self.v_hi.data_ptr(), self.v_lo.data_ptr(),
                           self.u_hi.data_ptr(), self.u_lo.data_ptr(), nb, n, o * self.ldq,
                           kh.data_ptr(), self.err.data_ptr(), self.st)
        self.nbuild += 1
        self._check()
        # K = K0 + 2 (V dU^T + dU V^T) = K0 + (kh - K0/2) + (kh - K0/2)^T: the
        # diagonal tiles' FP32 accumulation order leaves a tiny asymmetry
        return j, kh + kh.transpose(1, 2), anc["rho0"] + drho

    def anchored_half(self, c_occ: torch.Tensor, channel: int = 0):
        """(rho, U = U0 + B (C - C0)) at the final orbitals, FP64 (nb, N, o, X).

        Consumes the channel's anchor: U0 is updated in place.
        """
        nb, n, x, o = self.nb, self.n, self.x, self.nocc
        anc = self._anc[channel]
        drho = self._increment(c_occ, channel)
        self._lib.call("vqc_anchor_combine", anc["u0"].data_ptr(), self.u_hi.data_ptr(),
                       self.u_lo.data_ptr(), 0, 0, nb * n * o, x, self.ldq, 1.0, 1, self.st)
        self._check()
        u = anc["u0"]
        anc["u0"] = None
        return anc["rho0"] + drho, u


def make_builder(precision: str, b_packed: torch.Tensor, n: int, x: int, nocc: int):
    if precision == "fp64":
        return FP64Builder(b_packed, n, x, nocc)
    if precision == "mixed":
        return MixedBuilder(b_packed, n, x, nocc)
    raise ValueError(f"unknown precision {precision!r}")

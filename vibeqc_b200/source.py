"""Bounded DF integral source: 3-centre tiles generated on demand from a plan.

The reference keeps a persistent device "integral source" per batch that
generates bounded tiles of raw or transformed (whitened) 3-centre values and
reuses its setup for later geometries of the same topology
(``src/scf/cuda/df_source.cpp:198-389``: ``create_cuda_density_fitting_integral_source``,
``generate_cuda_density_fitting_raw_tile``, ``..._transformed_tile``).  Here the
native plan is that persistent object (shells, pair lists and work tables on
the device, reusable for any coordinates of the same molecules), and
:class:`IntegralSource` hands out row tiles of the packed tensor: all pairs
(mu, nu <= mu) whose larger index mu lies in a range of orbital shells, raw
(``vqc_int3c_rows``) or whitened with a caller's factor W (B = A W).  Tiles
are sized by :meth:`IntegralSource.tiles` to a byte budget, so a consumer can
stream a molecule whose full tensor does not fit in memory.
"""

from __future__ import annotations

import torch

from . import _lib
from . import basis as bas
from .plan import NativePlan


class IntegralSource:
    """Row tiles of the packed 3-centre tensor of each molecule of ``plan``."""

    def __init__(self, plan: NativePlan):
        self.plan = plan
        self._funcs = []  # per molecule: first function of every orbital shell, then N
        for mol in plan.molecules:
            offs, f = [], 0
            for s in mol.orbital_shells:
                offs.append(f)
                f += bas.count_functions([s], plan.spherical)
            offs.append(f)
            self._funcs.append(offs)

    def nshells(self, mol: int) -> int:
        return len(self._funcs[mol]) - 1

    def row_range(self, mol: int, shell_begin: int, shell_end: int) -> tuple[int, int]:
        """First and one-past-last packed row of the tile."""
        f0, f1 = self._funcs[mol][shell_begin], self._funcs[mol][shell_end]
        return f0 * (f0 + 1) // 2, f1 * (f1 + 1) // 2

    def tiles(self, mol: int, max_bytes: int) -> list[tuple[int, int]]:
        """Shell ranges whose FP64 row tiles each stay within ``max_bytes``."""
        naux = self.plan.layout[mol].naux
        out, s0, n = [], 0, self.nshells(mol)
        while s0 < n:
            s1 = s0 + 1
            while s1 < n:
                r0, r1 = self.row_range(mol, s0, s1 + 1)
                if (r1 - r0) * naux * 8 > max_bytes:
                    break
                s1 += 1
            r0, r1 = self.row_range(mol, s0, s1)
            if (r1 - r0) * naux * 8 > max_bytes:
                raise ValueError("max_bytes cannot hold the rows of one orbital shell")
            out.append((s0, s1))
            s0 = s1
        return out

    def raw_tile(self, xyz: torch.Tensor, mol: int, shell_begin: int, shell_end: int,
                 out: torch.Tensor | None = None) -> torch.Tensor:
        """Raw (mu nu|P) rows of the tile, (rows, naux) FP64 on the device."""
        r0, r1 = self.row_range(mol, shell_begin, shell_end)
        naux = self.plan.layout[mol].naux
        if out is None:
            out = torch.empty(r1 - r0, naux, dtype=torch.float64, device=xyz.device)
        if out.shape != (r1 - r0, naux) or out.dtype != torch.float64 or not out.is_contiguous():
            raise ValueError("out must be a contiguous (rows, naux) FP64 tensor")
        _lib.call("vqc_int3c_rows", self.plan.handle, xyz.data_ptr(), mol, shell_begin, shell_end,
                  out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        return out

    def whitened_tile(self, xyz: torch.Tensor, mol: int, shell_begin: int, shell_end: int,
                      w: torch.Tensor) -> torch.Tensor:
        """Rows of B = A W for a whitening factor W (naux, naux) of the molecule."""
        return self.raw_tile(xyz, mol, shell_begin, shell_end) @ w

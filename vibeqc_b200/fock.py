"""Fixed-density DF J/K evaluation with declared Fock coefficients (J/K source for hybrid DFT).

The reference exposes its J/K sources to other methods (hybrid DFT scales the
exchange by a_x) through ``FockPlan`` / ``FockBuildSpec`` / ``FockTerm``
(``python/generativeqc/fock.py:33-100,337-360,383-790``; native semantics
``src/scf/fock_build.cpp:429-495`` and ``src/api/c_api_fock.cpp:180-232``).
This module serves the density-fitted approximation of that interface on the
GPU with the same meanings:

* J = J[D_a + D_b] and K_s = K[D_s] are the raw (unscaled) DF matrices
  (restricted: one total density D and K = K[D]);
* F_s = H + c_J J + c_K K_s;
* E1 = tr(D_t H), E2 = 1/2 c_J tr(D_t J) + 1/2 c_K sum_s tr(D_s K_s);
* ``gradient`` (derivative_order 1) is dE2/dR at the fixed AO density, the
  two-electron geometric response only (no one-electron, nuclear or XC term),
  contracted by the native derivative kernels (vqc_grad3c / vqc_grad2c).

The molecule is given as atoms plus basis names (this engine has no
``NativeAO`` objects).  The plan keeps the raw and whitened 3-centre tensors
and the metric factor resident on the device; every evaluation reuses them.
Only ``approximation="density_fitted"`` and ``operator="full_range"`` are
served; other terms raise ``NotImplementedError`` when the plan is made.
"""

from __future__ import annotations

import math
import threading
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .jk import unpack_index
from .plan import NativePlan, make_molecule
from .timing import TIMER

_OPERATORS = ("full_range", "short_range", "long_range")
_APPROXIMATIONS = ("exact", "density_fitted")
_SPINS = ("restricted", "unrestricted")
Q_BLOCK_BYTES = 1 << 30  # bound on the per-block temporaries of the exchange products


@dataclass(frozen=True)
class FockTerm:
    """One operator/approximation and its signed Fock coefficient."""

    present: bool = True
    coefficient: float = 1.0
    operator: str = "full_range"
    omega: float = 0.0
    approximation: str = "density_fitted"

    def __post_init__(self) -> None:
        if type(self.present) is not bool:
            raise TypeError("Fock presence must be bool")
        if self.operator not in _OPERATORS or self.approximation not in _APPROXIMATIONS:
            raise ValueError("unknown Fock operator/approximation")
        if not math.isfinite(self.coefficient) or not math.isfinite(self.omega) or self.omega < 0:
            raise ValueError("Fock coefficients and nonnegative omega must be finite")


@dataclass(frozen=True)
class FockBuildSpec:
    """Spin, derivative order and the Coulomb/exchange terms (FP64 semantics)."""

    spin: str = "restricted"
    derivative_order: int = 1
    coulomb: FockTerm = field(default_factory=FockTerm)
    exchange: FockTerm = field(default_factory=lambda: FockTerm(coefficient=-0.5))

    def __post_init__(self) -> None:
        if self.spin not in _SPINS or type(self.derivative_order) is not int \
                or self.derivative_order not in (0, 1):
            raise ValueError("unsupported Fock spin/derivative order")
        if not isinstance(self.coulomb, FockTerm) or not isinstance(self.exchange, FockTerm):
            raise TypeError("Fock terms must be FockTerm objects")

    @classmethod
    def hf(cls, spin: str = "restricted", *, coulomb: str = "density_fitted",
           exchange: str = "density_fitted", derivative_order: int = 1) -> "FockBuildSpec":
        """Hartree-Fock coefficients: c_K = -1/2 (restricted) or -1 (unrestricted)."""
        return cls(spin, derivative_order, FockTerm(approximation=coulomb),
                   FockTerm(coefficient=-1.0 if spin == "unrestricted" else -0.5,
                            approximation=exchange))


@dataclass(frozen=True, eq=False)
class FockEvaluation:
    """Fixed-density energies (Hartree), Fock matrices and optional dE2/dR (host arrays)."""

    energy_one_electron: float
    energy_two_electron: float
    nuclear_repulsion: float
    fock: np.ndarray
    coulomb: np.ndarray | None
    exchange: np.ndarray | None
    gradient: np.ndarray | None

    @property
    def energy(self) -> float:
        return self.energy_one_electron + self.energy_two_electron + self.nuclear_repulsion


def _frozen(a: np.ndarray | None) -> np.ndarray | None:
    if a is not None:
        a.setflags(write=False)
    return a


class FockPlan:
    """Resident DF J/K source for one molecule (coordinates in Bohr) on a CUDA device."""

    def __init__(self, atoms, basis, spec: FockBuildSpec | None = None, *, auxiliary_basis,
                 device: str = "cuda", device_id: int = 0, metric_relative_threshold: float = 1e-10,
                 charge: int = 0, multiplicity: int = 1, spherical: bool = True):
        from . import scf as scfm

        spec = FockBuildSpec.hf() if spec is None else spec
        if not isinstance(spec, FockBuildSpec):
            raise TypeError("expected FockBuildSpec")
        for term in (spec.coulomb, spec.exchange):
            if term.present and term.approximation != "density_fitted":
                raise NotImplementedError("this engine serves density-fitted J/K terms only")
            if term.present and term.operator != "full_range":
                raise NotImplementedError("range-separated operators are not served")
        if device != "cuda":
            raise NotImplementedError("FockPlan runs on device='cuda' only")
        if not (0.0 <= metric_relative_threshold < 1.0):
            raise ValueError("metric_relative_threshold must be in [0, 1)")
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device is visible")
        _lib.lib()
        self.spec = spec
        self.device = torch.device("cuda", device_id)
        self.relative_threshold = float(metric_relative_threshold)
        self._lock = threading.Lock()
        self._mol = make_molecule(list(atoms), basis, auxiliary_basis, charge, multiplicity)
        self.natom = len(self._mol.atomic_numbers)
        with torch.cuda.device(self.device):
            self._plan = NativePlan([self._mol], spherical)
            self._xyz = torch.as_tensor(self._mol.coordinates, dtype=torch.float64,
                                        device=self.device).contiguous()
            ints = scfm.compute_integrals(self._plan, self._xyz)
            self.nao, self.naux = ints.s.shape[1], ints.metric.shape[1]
            n, x = self.nao, self.naux
            self._h = ints.h[0].clone()
            self._mf = scfm.factor_metric(ints.metric, self.relative_threshold)
            self._a_raw = ints.a_packed.clone()  # (1, P, X) raw packed, for truncated metrics
            b_packed = ints.a_packed
            scfm.whiten_in_place(b_packed, self._mf)
            self._b = b_packed[0][unpack_index(n, self.device)].contiguous()  # (N*N, X)
            del b_packed, ints
            z = torch.as_tensor(self._mol.atomic_numbers, dtype=torch.float64, device=self.device)
            self._charges = z
            self._enuc = float(scfm.nuclear_repulsion(z, self._xyz)[0])

    # -- helpers ------------------------------------------------------------

    def _exchange(self, d: torch.Tensor) -> torch.Tensor:
        """K[D] = sum_Q B_Q D B_Q over blocks of auxiliary functions."""
        n, x = self.nao, self.naux
        bq = self._b.view(n, n, x)
        k = torch.zeros(n, n, dtype=torch.float64, device=self.device)
        blk = max(1, Q_BLOCK_BYTES // (16 * n * n))
        for q0 in range(0, x, blk):
            b_blk = bq[:, :, q0:q0 + blk].permute(2, 0, 1)  # (blk, N, N)
            k += torch.matmul(torch.matmul(b_blk, d), b_blk).sum(dim=0)
        return k

    def _densities(self, density) -> list[torch.Tensor]:
        n = self.nao
        d = np.array(density, dtype=np.float64, order="C", copy=True)
        separate = self.spec.spin == "unrestricted"
        if np.iscomplexobj(d):
            raise TypeError("Fock densities must be real")
        if d.shape != ((2, n, n) if separate else (n, n)) or not np.isfinite(d).all():
            raise ValueError("Fock density shape/spin/finiteness mismatch")
        t = torch.as_tensor(d, device=self.device)
        return [t[0], t[1]] if separate else [t]

    # -- public --------------------------------------------------------------

    def evaluate(self, density, *, derivative: bool = False) -> FockEvaluation:
        """Raw J/K, the assembled Fock matrices, E1/E2 and optionally dE2/dR.

        ``density`` is (N, N) for restricted spin (the total density) or
        (2, N, N) for unrestricted spin.  J/K accept nonsymmetric densities;
        the gradient requires symmetric ones and fails before any result is
        returned otherwise.
        """
        if type(derivative) is not bool:
            raise TypeError("derivative must be bool")
        if derivative and self.spec.derivative_order != 1:
            raise ValueError("this plan was made without first derivatives")
        ds = self._densities(density)
        if derivative:
            for d in ds:
                if bool((d - d.T).abs().max() > 1e-12 * max(1.0, float(d.abs().max()))):
                    raise ValueError("DF derivatives require symmetric densities")
        cj = self.spec.coulomb.coefficient if self.spec.coulomb.present else 0.0
        ck = self.spec.exchange.coefficient if self.spec.exchange.present else 0.0
        n = self.nao
        with self._lock, torch.cuda.device(self.device), TIMER.stage("fock_evaluate"):
            dt = ds[0] if len(ds) == 1 else ds[0] + ds[1]
            rho_w = self._b.T @ dt.reshape(-1)  # whitened fitted density
            j = (self._b @ rho_w).view(n, n) if self.spec.coulomb.present else None
            ks = [self._exchange(d) for d in ds] if self.spec.exchange.present else None
            fs = []
            for s in range(len(ds)):
                f = self._h.clone()
                if j is not None:
                    f += cj * j
                if ks is not None:
                    f += ck * ks[s]
                fs.append(f)
            e1 = float((dt * self._h).sum())
            e2 = 0.0
            if j is not None:
                e2 += 0.5 * cj * float((dt * j).sum())
            if ks is not None:
                e2 += 0.5 * ck * sum(float((d * k).sum()) for d, k in zip(ds, ks))
            grad = self._gradient(ds, dt, rho_w, cj, ck) if derivative else None
            values = [float(e1), float(e2)]
            if not all(math.isfinite(v) for v in values):
                raise FloatingPointError("nonfinite Fock energy")
            host = lambda t: None if t is None else t.detach().cpu().numpy()  # noqa: E731
            fock = host(torch.stack(fs) if len(fs) == 2 else fs[0])
            exch = None if ks is None else host(torch.stack(ks) if len(ks) == 2 else ks[0])
            return FockEvaluation(e1, e2, self._enuc, _frozen(fock), _frozen(host(j)),
                                  _frozen(exch), _frozen(host(grad)))

    def _gradient(self, ds, dt, rho_w, cj, ck) -> torch.Tensor:
        """dE2/dR at fixed densities: DF reverse weights, then vqc_grad3c / vqc_grad2c.

        Abar  = c_J D_t (x) M+ rho + c_K sum_s D_s At D_s,  At_P = sum_Q M+_PQ A_Q = (B W^T)_P,
        Mbar  = -M+ Mbar+ M+ = -1/2 c_J c c^T - 1/2 c_K sum_s (D_s At D_s) : At  (full rank),
        otherwise the spectral adjoint of Mbar+ = 1/2 c_J rho rho^T + 1/2 c_K sum_s Q(D_s)
        in the raw basis (reference ``src/scf/density_fitting.cpp:464-594``,
        ``density_fitting_metric.cpp:50-99``).
        """
        from .gradient import spectral_metric_adjoint

        n, x = self.nao, self.naux
        mf = self._mf
        w = mf.inv_sqrt[0]
        cvec = w @ rho_w  # M+ rho_raw
        at = (self._b @ w.T).view(n, n, x)
        abar = cj * dt[:, :, None] * cvec[None, None, :]
        mbar = -0.5 * cj * torch.outer(cvec, cvec)
        truncated = mf.rank[0] < x
        for d in ds:
            if ck == 0.0:
                break
            t = torch.matmul(d, at.permute(2, 0, 1))  # (X, N, N): D At_P
            t = torch.matmul(t, d).permute(1, 2, 0)  # (N, N, X): D At_P D
            abar += ck * t
            if not truncated:
                mbar -= 0.5 * ck * (t.reshape(n * n, x).T @ at.reshape(n * n, x))
            del t
        if truncated:
            a_full = self._a_raw[0][unpack_index(n, self.device)].view(n, n, x)
            rho_raw = torch.einsum("mnp,mn->p", a_full, dt)
            mbp = 0.5 * cj * torch.outer(rho_raw, rho_raw)
            for d in ds:
                if ck == 0.0:
                    break
                t = torch.matmul(torch.matmul(d, a_full.permute(2, 0, 1)), d)  # (X, N, N)
                mbp += 0.5 * ck * (t.reshape(x, n * n) @ a_full.permute(2, 0, 1).reshape(x, n * n).T)
            mbar = spectral_metric_adjoint(mf.eigenvalues[0], mf.eigenvectors[0], mf.keep[0], mbp,
                                           self.relative_threshold)
        mu, nu = torch.tril_indices(n, n, device=self.device)
        abar_packed = abar[mu, nu].contiguous()
        grad = torch.zeros(self.natom * 3, dtype=torch.float64, device=self.device)
        st = torch.cuda.current_stream().cuda_stream
        _lib.call("vqc_grad3c", self._plan.handle, self._xyz.data_ptr(), abar_packed.data_ptr(),
                  grad.data_ptr(), st)
        _lib.call("vqc_grad2c", self._plan.handle, self._xyz.data_ptr(),
                  mbar.contiguous().data_ptr(), grad.data_ptr(), st)
        return grad

    def close(self) -> None:
        with self._lock:
            if getattr(self, "_plan", None) is not None:
                self._plan.close()
                self._plan = None
                self._b = self._a_raw = None

    def __enter__(self):
        return self

    def __exit__(self, *_exc):
        self.close()

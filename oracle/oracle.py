"""CPU oracle for the DF-RHF energy and analytic forces.

TEST INFRASTRUCTURE ONLY.  Tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use it as the checker; no product path imports it.

This is a plain restatement of the reference's CPU density-fitting RHF path:

* integrals from ``liboracle.so`` (``df_oracle.c``; McMurchie-Davidson);
* metric factor with the relative eigenvalue cutoff
  (reference ``src/integrals/density_fitting_metric.cpp:101-154``);
* whitened three-centre tensor B = A M^{-1/2}
  (``src/scf/density_fitting.cpp:711-764``);
* RI-J and density-form RI-K (``src/scf/density_fitting.cpp:101-222``);
* the SCF loop: core guess, F = H + J - K/2, Pulay DIIS on FDS - SDF,
  convergence on |dE|, rms(dD) and max|FDS - SDF|
  (``src/scf/solver/mean_field_driver.cpp:233``,
  ``src/scf/cuda/scf_convergence_policy.cuh:28-37``);
* reverse weights Abar and Mbar+ (``src/scf/density_fitting.cpp:464-594``),
  the spectral metric response (``density_fitting_metric.cpp:50-99``) and the
  weighted derivative contractions (``src/integrals/s_integrals.cpp:1073,2187``);
* forces F = -(g_1e + g_DF + dV_nn) (``src/scf/rhf.cpp:856-868``).
"""

from __future__ import annotations

import ctypes
import math
import subprocess
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from vibeqc_b200 import basis as bas

HERE = Path(__file__).resolve().parent
_LIB_PATH = HERE / "liboracle.so"
NSMAX, NCMAX, LMAX = 13, 28, 6


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(_LIB_PATH))
        for name in ("oracle_int3c", "oracle_int2c", "oracle_int1e", "oracle_grad3c",
                     "oracle_grad2c", "oracle_grad1e", "oracle_boys"):
            getattr(_lib, name).restype = None
    return _lib


class _CBasis(ctypes.Structure):
    _fields_ = [
        ("nshell", ctypes.c_int),
        ("l", ctypes.c_void_p),
        ("atom", ctypes.c_void_p),
        ("nprim", ctypes.c_void_p),
        ("prim_off", ctypes.c_void_p),
        ("func_off", ctypes.c_void_p),
        ("exps", ctypes.c_void_p),
        ("coefs", ctypes.c_void_p),
        ("nfunc", ctypes.c_int),
        ("trans", ctypes.c_void_p),
        ("nout", ctypes.c_void_p),
    ]


class OracleBasis:
    """Shell arrays in the layout the C oracle reads; functions in shell order."""

    def __init__(self, shells, spherical: bool = True):
        self.shells = list(shells)
        self.spherical = spherical
        ls, atoms, nprim, poff, foff, exps, coefs = [], [], [], [], [], [], []
        f = p = 0
        for s in self.shells:
            a, c = bas.normalized_coefficients(s)
            ls.append(s.angular_momentum)
            atoms.append(s.atom_index)
            nprim.append(len(a))
            poff.append(p)
            foff.append(f)
            exps.extend(a)
            coefs.extend(c)
            p += len(a)
            f += bas.nfunc(s.angular_momentum, spherical)
        if max(ls) + 1 > LMAX:
            raise ValueError("oracle supports l <= 5")
        self.nfunc = f
        i32 = lambda v: np.ascontiguousarray(v, dtype=np.int32)  # noqa: E731
        self._l, self._atom, self._nprim = i32(ls), i32(atoms), i32(nprim)
        self._poff, self._foff = i32(poff), i32(foff)
        self._exps = np.ascontiguousarray(exps, dtype=np.float64)
        self._coefs = np.ascontiguousarray(coefs, dtype=np.float64)
        trans = np.zeros((LMAX + 1, NSMAX, NCMAX))
        nout = np.zeros(LMAX + 1, dtype=np.int32)
        for l in range(LMAX + 1):
            t = bas.transform_matrix(l, spherical) if 2 * l + 1 <= NSMAX or not spherical else None
            if t is None or t.shape[0] > NSMAX:
                continue
            trans[l, : t.shape[0], : t.shape[1]] = t
            nout[l] = t.shape[0]
        self._trans, self._nout = trans, nout
        self.c = _CBasis(
            len(ls),
            self._l.ctypes.data,
            self._atom.ctypes.data,
            self._nprim.ctypes.data,
            self._poff.ctypes.data,
            self._foff.ctypes.data,
            self._exps.ctypes.data,
            self._coefs.ctypes.data,
            f,
            self._trans.ctypes.data,
            self._nout.ctypes.data,
        )


def _ptr(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.c_void_p)


def boys(mmax: int, t: float) -> np.ndarray:
    out = np.zeros(mmax + 1)
    lib().oracle_boys(ctypes.c_int(mmax), ctypes.c_double(t), _ptr(out))
    return out


def int3c(orb: OracleBasis, aux: OracleBasis, xyz: np.ndarray) -> np.ndarray:
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    out = np.zeros((orb.nfunc, orb.nfunc, aux.nfunc))
    lib().oracle_int3c(ctypes.byref(orb.c), ctypes.byref(aux.c), _ptr(xyz), _ptr(out))
    return out


def int2c(aux: OracleBasis, xyz: np.ndarray) -> np.ndarray:
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    out = np.zeros((aux.nfunc, aux.nfunc))
    lib().oracle_int2c(ctypes.byref(aux.c), _ptr(xyz), _ptr(out))
    return out


def int1e(orb: OracleBasis, xyz: np.ndarray, charges: np.ndarray):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    z = np.ascontiguousarray(charges, dtype=np.float64)
    n = orb.nfunc
    s, t, v = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
    lib().oracle_int1e(ctypes.byref(orb.c), ctypes.c_int(len(z)), _ptr(xyz), _ptr(z),
                       _ptr(s), _ptr(t), _ptr(v))
    return s, t, v


def grad3c(orb, aux, xyz, abar) -> np.ndarray:
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    abar = np.ascontiguousarray(abar, dtype=np.float64)
    g = np.zeros(xyz.size)
    lib().oracle_grad3c(ctypes.byref(orb.c), ctypes.byref(aux.c), ctypes.c_int(len(xyz)),
                        _ptr(xyz), _ptr(abar), _ptr(g))
    return g.reshape(-1, 3)


def grad2c(aux, xyz, mbar) -> np.ndarray:
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    mbar = np.ascontiguousarray(mbar, dtype=np.float64)
    g = np.zeros(xyz.size)
    lib().oracle_grad2c(ctypes.byref(aux.c), ctypes.c_int(len(xyz)), _ptr(xyz), _ptr(mbar),
                        _ptr(g))
    return g.reshape(-1, 3)


def grad1e(orb, xyz, charges, dens, wdens) -> np.ndarray:
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    z = np.ascontiguousarray(charges, dtype=np.float64)
    g = np.zeros(xyz.size)
    lib().oracle_grad1e(ctypes.byref(orb.c), ctypes.c_int(len(z)), _ptr(xyz), _ptr(z),
                        _ptr(np.ascontiguousarray(dens)), _ptr(np.ascontiguousarray(wdens)),
                        _ptr(g))
    return g.reshape(-1, 3)


def nuclear_repulsion(xyz: np.ndarray, charges: np.ndarray) -> tuple[float, np.ndarray]:
    e = 0.0
    g = np.zeros_like(xyz)
    for i in range(len(xyz)):
        for j in range(i):
            d = xyz[i] - xyz[j]
            r = math.sqrt(d @ d)
            e += charges[i] * charges[j] / r
            f = -charges[i] * charges[j] / r**3 * d
            g[i] += f
            g[j] -= f
    return e, g


# --------------------------------------------------------------------------
# metric factor and its spectral response
# --------------------------------------------------------------------------

@dataclass
class MetricFactor:
    eigenvalues: np.ndarray
    eigenvectors: np.ndarray
    keep: np.ndarray
    inv_sqrt: np.ndarray
    pinv: np.ndarray
    rank: int
    condition: float


def factor_metric(m: np.ndarray, relative_threshold: float = 1e-10) -> MetricFactor:
    """Eigen-based M^{-1/2} dropping lambda <= rel * lambda_max.

    Reference: ``src/integrals/density_fitting_metric.cpp:101-154``.
    """
    if not np.all(np.isfinite(m)):
        raise FloatingPointError("non-finite metric")
    lam, v = np.linalg.eigh(0.5 * (m + m.T))
    lmax = lam[-1]
    if not lmax > 0:
        raise FloatingPointError("metric has no positive eigenvalue")
    keep = lam > relative_threshold * lmax
    vk = v[:, keep]
    inv_sqrt = (vk / np.sqrt(lam[keep])) @ vk.T
    pinv = (vk / lam[keep]) @ vk.T
    return MetricFactor(lam, v, keep, inv_sqrt, pinv, int(keep.sum()),
                        float(lmax / lam[keep][0]))


def metric_response(f: MetricFactor, mbar_plus: np.ndarray, relative_threshold=1e-10,
                    power: float = -1.0) -> np.ndarray:
    """Adjoint of M -> f(M) through the thresholded spectral map.

    f(l) = l**power on the retained space and 0 on the discarded one
    (power = -1: the pseudoinverse; -1/2: the inverse square root).  Divided
    differences (f(li) - f(lj)) / (li - lj); f'(l) on retained diagonal
    entries.  Reference ``density_fitting_metric.cpp:50-99`` and
    ``src/tensor/symmetric_matrix_function.cpp:62``.  Eigenvalues within
    128 eps lambda_max of the cutoff are a rank crossing and rejected.
    """
    lam = f.eigenvalues
    lmax = lam[-1]
    cut = relative_threshold * lmax
    if np.any(np.abs(lam - cut) <= 128 * np.finfo(float).eps * lmax):
        raise FloatingPointError("metric eigenvalue at the rank cutoff")
    safe = np.where(f.keep, lam, 1.0)
    fl = np.where(f.keep, safe**power, 0.0)
    dl = lam[:, None] - lam[None, :]
    same = np.abs(dl) <= 1e-14 * lmax
    with np.errstate(divide="ignore", invalid="ignore"):
        gam = (fl[:, None] - fl[None, :]) / np.where(same, 1.0, dl)
    deriv = np.where(f.keep, power * safe ** (power - 1.0), 0.0)
    gam = np.where(same, 0.5 * (deriv[:, None] + deriv[None, :]), gam)
    v = f.eigenvectors
    return v @ ((v.T @ mbar_plus @ v) * gam) @ v.T


# --------------------------------------------------------------------------
# DF-RHF
# --------------------------------------------------------------------------

def molecule_arrays(atoms):
    z = np.array([bas.atomic_number(s) for s, _ in atoms], dtype=np.float64)
    xyz = np.array([p for _, p in atoms], dtype=np.float64)
    return z, xyz


@dataclass
class OracleResult:
    energy: float
    forces: np.ndarray | None
    converged: bool
    iterations: int
    density: np.ndarray
    orbital_energies: np.ndarray
    coefficients: np.ndarray
    nocc: int
    extra: dict


def build_jk(b: np.ndarray, d: np.ndarray):
    """J and density-form K from whitened B (N, N, X)."""
    rho = np.einsum("mnq,mn->q", b, d, optimize=True)
    j = b @ rho
    bq = np.ascontiguousarray(b.transpose(2, 0, 1))
    k = np.einsum("qml,ls,qsn->mn", bq, d, bq, optimize=True)
    return j, k


def df_rhf(atoms, basis="def2-svp", auxiliary_basis="cc-pvdz-jkfit", *, spherical=True,
           charge=0, max_iterations=100, energy_tolerance=1e-10, density_tolerance=1e-8,
           diis_history=8, forces=True, relative_threshold=1e-10) -> OracleResult:
    z, xyz = molecule_arrays(atoms)
    orb_sh = bas.expand_shells(z.astype(int), basis)
    aux_sh = bas.expand_shells(z.astype(int), auxiliary_basis)
    orb, aux = OracleBasis(orb_sh, spherical), OracleBasis(aux_sh, spherical)
    nel = int(z.sum()) - charge
    if nel % 2:
        raise ValueError("RHF needs an even electron count")
    nocc = nel // 2
    s, t, v = int1e(orb, xyz, z)
    h = t + v
    m = int2c(aux, xyz)
    a = int3c(orb, aux, xyz)
    mf = factor_metric(m, relative_threshold)
    b = a @ mf.inv_sqrt
    enuc, gnuc = nuclear_repulsion(xyz, z)
    sl, sv = np.linalg.eigh(s)
    xorth = (sv / np.sqrt(sl)) @ sv.T

    def density_from(f):
        e, cp = np.linalg.eigh(xorth.T @ f @ xorth)
        c = xorth @ cp
        return 2.0 * c[:, :nocc] @ c[:, :nocc].T, e, c

    d, eps, coef = density_from(h)
    e_old = None
    errs, focks = [], []
    converged = False
    it = 0
    energy = 0.0
    for it in range(1, max_iterations + 1):
        j, k = build_jk(b, d)
        f = h + j - 0.5 * k
        energy = 0.5 * np.sum(d * (h + f)) + enuc
        err = f @ d @ s - s @ d @ f
        err_o = xorth.T @ err @ xorth
        d_new, eps, coef = None, None, None
        errs.append(err_o)
        focks.append(f)
        errs, focks = errs[-diis_history:], focks[-diis_history:]
        nh = len(errs)
        if nh > 1:
            bm = -np.ones((nh + 1, nh + 1))
            bm[nh, nh] = 0.0
            for i in range(nh):
                for jj in range(nh):
                    bm[i, jj] = np.sum(errs[i] * errs[jj])
            rhs = np.zeros(nh + 1)
            rhs[nh] = -1.0
            try:
                w = np.linalg.solve(bm, rhs)[:nh]
                f_ext = sum(wi * fi for wi, fi in zip(w, focks))
            except np.linalg.LinAlgError:
                f_ext = f
        else:
            f_ext = f
        d_new, eps, coef = density_from(f_ext)
        de = abs(energy - e_old) if e_old is not None else np.inf
        drms = float(np.sqrt(np.mean((d_new - d) ** 2)))
        comm = float(np.abs(err).max())
        e_old = energy
        # src/scf/cuda/scf_convergence_policy.cuh:28-37 (roundoff guard 16 eps,
        # src/scf/cuda/scf_constants.hpp:16-17)
        guard = 16.0 * 2.220446049250313e-16 * max(1.0, abs(energy), abs(e_old or 0.0))
        if de < energy_tolerance + guard and drms < density_tolerance and comm <= min(1e-8, density_tolerance):
            converged = True
            break
        d = d_new
    # final quantities at the density the energy was evaluated with
    j, k = build_jk(b, d)
    f = h + j - 0.5 * k
    energy = 0.5 * np.sum(d * (h + f)) + enuc
    e_mo, cp = np.linalg.eigh(xorth.T @ f @ xorth)
    coef = xorth @ cp
    result = OracleResult(energy, None, converged, it, d, e_mo, coef, nocc, {})
    if forces:
        result.forces = -df_rhf_gradient(orb, aux, xyz, z, a, mf, d, coef, e_mo, nocc, gnuc,
                                         relative_threshold)
    result.extra.update(nao=orb.nfunc, naux=aux.nfunc, rank=mf.rank, condition=mf.condition)
    return result


def df_rhf_gradient(orb, aux, xyz, z, a, mf, d, coef, e_mo, nocc, gnuc, relative_threshold=1e-10):
    """Positive energy gradient (natom, 3) at the SCF solution."""
    cocc = coef[:, :nocc]
    dmat = 2.0 * cocc @ cocc.T
    wmat = 2.0 * (cocc * e_mo[:nocc]) @ cocc.T
    rho = np.einsum("mnp,mn->p", a, dmat, optimize=True)
    cvec = mf.pinv @ rho
    aq = np.ascontiguousarray(a.transpose(2, 0, 1))  # (X, N, N)
    daq = np.einsum("ml,qls,sn->qmn", dmat, aq, dmat, optimize=True)  # D A_Q D
    abar = dmat[:, :, None] * cvec[None, None, :]
    abar -= 0.5 * np.einsum("pq,qmn->mnp", mf.pinv, daq, optimize=True)
    qmat = np.einsum("pmn,qmn->pq", aq, daq, optimize=True)
    mbar_plus = 0.5 * np.outer(rho, rho) - 0.25 * qmat
    mbar = metric_response(mf, mbar_plus, relative_threshold)
    g = grad1e(orb, xyz, z, dmat, wmat)
    g += grad3c(orb, aux, xyz, abar)
    g += grad2c(aux, xyz, mbar)
    g += gnuc
    return g


# --------------------------------------------------------------------------
# DF-UHF
# --------------------------------------------------------------------------


def build_k(b: np.ndarray, d: np.ndarray) -> np.ndarray:
    """Density-form exchange K[D] = sum_Q B_Q D B_Q from whitened B (N, N, X)."""
    bq = np.ascontiguousarray(b.transpose(2, 0, 1))
    return np.einsum("qml,ls,qsn->mn", bq, d, bq, optimize=True)


def spin_counts(nelectron: int, multiplicity: int) -> tuple[int, int]:
    """(n_alpha, n_beta) for a total electron count and spin multiplicity 2S+1."""
    if multiplicity < 1 or (nelectron + multiplicity - 1) % 2:
        raise ValueError("electron count and multiplicity are inconsistent")
    na = (nelectron + multiplicity - 1) // 2
    nb = nelectron - na
    if nb < 0:
        raise ValueError("multiplicity exceeds the electron count")
    return na, nb


def df_uhf(atoms, basis="def2-svp", auxiliary_basis="cc-pvdz-jkfit", *, spherical=True,
           charge=0, multiplicity=2, max_iterations=100, energy_tolerance=1e-10,
           density_tolerance=1e-8, diis_history=8, forces=True,
           relative_threshold=1e-10) -> OracleResult:
    """Unrestricted DF-HF energy and analytic forces.

    F_s = H + J[D_a + D_b] - K[D_s] (reference ``src/scf/density_fitting.cpp:844``),
    E = 1/2 tr(D_t H) + 1/2 sum_s tr(D_s F_s) + E_nn; Pulay DIIS with one set of
    weights over both spins' residuals F_s D_s S - S D_s F_s (reference
    ``src/scf/cuda/df_scf_diis.cpp:110-185``); convergence on |dE|, the rms of
    both spin-density changes and the larger spin residual
    (``src/scf/cuda/df_scf_kernels.cu:296-340``).
    """
    z, xyz = molecule_arrays(atoms)
    orb_sh = bas.expand_shells(z.astype(int), basis)
    aux_sh = bas.expand_shells(z.astype(int), auxiliary_basis)
    orb, aux = OracleBasis(orb_sh, spherical), OracleBasis(aux_sh, spherical)
    na, nb = spin_counts(int(z.sum()) - charge, multiplicity)
    s, t, v = int1e(orb, xyz, z)
    h = t + v
    m = int2c(aux, xyz)
    a = int3c(orb, aux, xyz)
    mf = factor_metric(m, relative_threshold)
    b = a @ mf.inv_sqrt
    enuc, gnuc = nuclear_repulsion(xyz, z)
    sl, sv = np.linalg.eigh(s)
    xorth = (sv / np.sqrt(sl)) @ sv.T
    occ = (na, nb)

    def densities_from(fs):
        out = []
        for f, n in zip(fs, occ):
            e, cp = np.linalg.eigh(xorth.T @ f @ xorth)
            c = xorth @ cp
            out.append((c[:, :n] @ c[:, :n].T, e, c))
        return out

    ds = [x[0] for x in densities_from((h, h))]
    e_old = None
    errs, focks = [], []
    converged = False
    it = 0
    for it in range(1, max_iterations + 1):
        j = build_jk(b, ds[0] + ds[1])[0]
        fs = [h + j - build_k(b, d) for d in ds]
        energy = (0.5 * np.sum((ds[0] + ds[1]) * h)
                  + 0.5 * sum(np.sum(d * f) for d, f in zip(ds, fs)) + enuc)
        res = [f @ d @ s - s @ d @ f for d, f in zip(ds, fs)]
        errs.append(np.concatenate([xorth.T @ r @ xorth for r in res]))
        focks.append(fs)
        errs, focks = errs[-diis_history:], focks[-diis_history:]
        nh = len(errs)
        f_ext = fs
        if nh > 1:
            bm = -np.ones((nh + 1, nh + 1))
            bm[nh, nh] = 0.0
            for i in range(nh):
                for jj in range(nh):
                    bm[i, jj] = np.sum(errs[i] * errs[jj])
            rhs = np.zeros(nh + 1)
            rhs[nh] = -1.0
            try:
                w = np.linalg.solve(bm, rhs)[:nh]
                f_ext = [sum(wi * fk[sp] for wi, fk in zip(w, focks)) for sp in range(2)]
            except np.linalg.LinAlgError:
                f_ext = fs
        new = [x[0] for x in densities_from(f_ext)]
        de = abs(energy - e_old) if e_old is not None else np.inf
        drms = float(np.sqrt(sum(np.sum((dn - d) ** 2) for dn, d in zip(new, ds))
                             / (2 * ds[0].size)))
        comm = max(float(np.abs(r).max()) for r in res)
        guard = 16.0 * 2.220446049250313e-16 * max(1.0, abs(energy), abs(e_old or 0.0))
        e_old = energy
        if de < energy_tolerance + guard and drms < density_tolerance and comm <= min(1e-8, density_tolerance):
            converged = True
            break
        ds = new
    j = build_jk(b, ds[0] + ds[1])[0]
    fs = [h + j - build_k(b, d) for d in ds]
    energy = (0.5 * np.sum((ds[0] + ds[1]) * h)
              + 0.5 * sum(np.sum(d * f) for d, f in zip(ds, fs)) + enuc)
    result = OracleResult(energy, None, converged, it, ds[0] + ds[1], np.zeros(0),
                          np.zeros((0, 0)), na, {"alpha_density": ds[0], "beta_density": ds[1],
                                                  "nalpha": na, "nbeta": nb})
    if forces:
        result.forces = -df_uhf_gradient(orb, aux, xyz, z, a, mf, ds, fs, gnuc, relative_threshold)
    result.extra.update(nao=orb.nfunc, naux=aux.nfunc, rank=mf.rank, condition=mf.condition)
    return result


def df_uhf_gradient(orb, aux, xyz, z, a, mf, ds, fs, gnuc, relative_threshold=1e-10):
    """Positive energy gradient (natom, 3) of DF-UHF at its SCF solution.

    Reverse weights as the reference's unrestricted weighted gradient
    (``src/scf/density_fitting.cpp:919-944``: Coulomb on D_a + D_b, exchange
    on each spin density with Fock coefficient -1): with rho = A:D_t,
        Abar  = D_t (x) M+ rho - sum_s M+ (D_s A D_s),
        Mbar+ = rho rho^T / 2 - 1/2 sum_s Q(D_s),  Q_PQ = A_P : (D_s A_Q D_s);
    energy-weighted density W = sum_s D_s F_s D_s.
    """
    dt = ds[0] + ds[1]
    wmat = sum(d @ f @ d for d, f in zip(ds, fs))
    rho = np.einsum("mnp,mn->p", a, dt, optimize=True)
    cvec = mf.pinv @ rho
    aq = np.ascontiguousarray(a.transpose(2, 0, 1))
    abar = dt[:, :, None] * cvec[None, None, :]
    mbar_plus = 0.5 * np.outer(rho, rho)
    for d in ds:
        daq = np.einsum("ml,qls,sn->qmn", d, aq, d, optimize=True)
        abar -= np.einsum("pq,qmn->mnp", mf.pinv, daq, optimize=True)
        mbar_plus -= 0.5 * np.einsum("pmn,qmn->pq", aq, daq, optimize=True)
    mbar = metric_response(mf, mbar_plus, relative_threshold)
    g = grad1e(orb, xyz, z, dt, wmat)
    g += grad3c(orb, aux, xyz, abar)
    g += grad2c(aux, xyz, mbar)
    g += gnuc
    return g


# --------------------------------------------------------------------------
# Fixed-density DF J/K with declared Fock coefficients
# --------------------------------------------------------------------------


def fock_evaluate(atoms, basis, auxiliary_basis, densities, coulomb=1.0, exchange=-0.5, *,
                  spherical=True, relative_threshold=1e-10, derivative=True) -> dict:
    """J, K, Fock matrices, energies and dE2/dR at fixed AO densities.

    Reference semantics (``src/scf/fock_build.cpp:429-495``, ``src/api/c_api_fock.cpp:
    180-232``): ``densities`` is [D] (restricted, D the total density) or
    [D_a, D_b] (unrestricted); J = J[D_a + D_b], K_s = K[D_s];
    F_s = H + c_J J + c_K K_s; E1 = tr(D_t H);
    E2 = 1/2 c_J tr(D_t J) + 1/2 c_K sum_s tr(D_s K_s); the gradient is dE2/dR
    at fixed D through the DF reverse weights
        Abar  = c_J D_t (x) M+ rho + c_K sum_s M+ (D_s A D_s),
        Mbar+ = 1/2 c_J rho rho^T + 1/2 c_K sum_s Q(D_s).
    """
    z, xyz = molecule_arrays(atoms)
    orb = OracleBasis(bas.expand_shells(z.astype(int), basis), spherical)
    aux = OracleBasis(bas.expand_shells(z.astype(int), auxiliary_basis), spherical)
    s, t, v = int1e(orb, xyz, z)
    h = t + v
    m = int2c(aux, xyz)
    a = int3c(orb, aux, xyz)
    mf = factor_metric(m, relative_threshold)
    ds = [np.asarray(d, dtype=np.float64) for d in densities]
    dt = sum(ds)
    rho = np.einsum("mnp,mn->p", a, dt, optimize=True)
    cvec = mf.pinv @ rho
    j = a @ cvec
    aq = np.ascontiguousarray(a.transpose(2, 0, 1))
    ks = [np.einsum("pml,ls,qsn,pq->mn", aq, d, aq, mf.pinv, optimize=True) for d in ds]
    fs = [h + coulomb * j + exchange * k for k in ks]
    e1 = float(np.sum(dt * h))
    e2 = 0.5 * coulomb * float(np.sum(dt * j)) + 0.5 * exchange * sum(
        float(np.sum(d * k)) for d, k in zip(ds, ks))
    enuc, _ = nuclear_repulsion(xyz, z)
    out = {"coulomb": j, "exchange": ks, "fock": fs, "energy_one_electron": e1,
           "energy_two_electron": e2, "nuclear_repulsion": enuc, "gradient": None}
    if derivative:
        abar = coulomb * dt[:, :, None] * cvec[None, None, :]
        mbar_plus = 0.5 * coulomb * np.outer(rho, rho)
        for d in ds:
            daq = np.einsum("ml,qls,sn->qmn", d, aq, d, optimize=True)
            abar += exchange * np.einsum("pq,qmn->mnp", mf.pinv, daq, optimize=True)
            mbar_plus += 0.5 * exchange * np.einsum("pmn,qmn->pq", aq, daq, optimize=True)
        mbar = metric_response(mf, mbar_plus, relative_threshold)
        out["gradient"] = grad3c(orb, aux, xyz, abar) + grad2c(aux, xyz, mbar)
    return out

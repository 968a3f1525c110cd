"""Host side of a batch plan: shells -> C-ABI descriptor -> native ``vqc_plan``.

Mirrors what ``generativeqc_batch_prepare`` receives (reference
``include/generativeqc/generativeqc.h:586-599,733-740,1435``): per molecule the
atoms, orbital shells and auxiliary shells.  Auxiliary shells are reordered by
angular momentum inside each molecule (the fitting space is unchanged; only the
internal order of auxiliary functions is).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from . import basis as bas

BOHR_UNITS = "bohr"


@dataclass
class MoleculeSpec:
    """One system of a batch (coordinates in Bohr)."""

    atomic_numbers: np.ndarray
    coordinates: np.ndarray
    orbital_shells: list
    aux_shells: list  # sorted by l
    charge: int = 0
    multiplicity: int = 1

    @property
    def nelectron(self) -> int:
        return int(self.atomic_numbers.sum()) - self.charge

    @property
    def nocc(self) -> int:
        """Doubly occupied orbitals (restricted) or alpha electrons (unrestricted)."""
        if self.multiplicity == 1:
            return self.nelectron // 2
        return self.nalpha

    @property
    def nalpha(self) -> int:
        return (self.nelectron + self.multiplicity - 1) // 2

    @property
    def nbeta(self) -> int:
        return self.nelectron - self.nalpha


def make_molecule(atoms, basis, auxiliary_basis, charge: int = 0, multiplicity: int = 1) -> MoleculeSpec:
    z = np.array([bas.atomic_number(a[0]) for a in atoms], dtype=np.int64)
    xyz = np.array([[float(v) for v in a[1]] for a in atoms], dtype=np.float64).reshape(-1, 3)
    if xyz.shape[0] != len(z) or not np.all(np.isfinite(xyz)):
        raise ValueError("atom coordinates must be finite (natoms, 3) Bohr values")
    orb = bas.expand_shells(z, basis)
    aux = bas.expand_shells(z, auxiliary_basis)
    aux = sorted(aux, key=lambda s: s.angular_momentum)  # stable: atom order kept within l
    for s in orb + aux:
        if s.angular_momentum > 3:
            raise ValueError("shells above f are not supported by the CUDA kernels")
    nel = int(z.sum()) - int(charge)
    if int(multiplicity) < 1 or nel < 1 or (nel + int(multiplicity) - 1) % 2 \
            or int(multiplicity) - 1 > nel:
        raise ValueError("charge and multiplicity are inconsistent with the electron count")
    return MoleculeSpec(z, xyz, orb, aux, int(charge), int(multiplicity))


@dataclass
class MoleculeLayout:
    nao: int
    naux: int
    natom: int
    atom_offset: int
    mat_offset: int
    met_offset: int
    a_offset: int
    nocc: int

    @property
    def npair(self) -> int:
        return self.nao * (self.nao + 1) // 2


def batch_descriptor(molecules: list[MoleculeSpec], spherical: bool = True):
    """``vqc_batch_desc`` for ``molecules`` plus the host arrays it points into.

    The arrays must outlive every native call that reads the descriptor.
    """
    atom_off, sh_off, aux_off = [0], [0], [0]
    charges, sl, sa, sn, sp, pe, pc = [], [], [], [], [], [], []
    al, aa, an, ap, ae, ac = [], [], [], [], [], []
    natom = 0
    for mol in molecules:
        charges.extend(mol.atomic_numbers.astype(np.float64))
        for shells, l_, a_, n_, p_, e_, c_ in (
            (mol.orbital_shells, sl, sa, sn, sp, pe, pc),
            (mol.aux_shells, al, aa, an, ap, ae, ac),
        ):
            for s in shells:
                ex, co = bas.normalized_coefficients(s)
                l_.append(s.angular_momentum)
                a_.append(natom + s.atom_index)
                n_.append(len(ex))
                p_.append(len(e_))
                e_.extend(ex)
                c_.extend(co)
        natom += len(mol.atomic_numbers)
        atom_off.append(natom)
        sh_off.append(len(sl))
        aux_off.append(len(al))
    keep = [
        _lib.i32(atom_off), _lib.i32(sh_off), _lib.i32(aux_off), _lib.f64(charges),
        _lib.i32(sl), _lib.i32(sa), _lib.i32(sn), _lib.i32(sp), _lib.f64(pe), _lib.f64(pc),
        _lib.i32(al), _lib.i32(aa), _lib.i32(an), _lib.i32(ap), _lib.f64(ae), _lib.f64(ac),
    ]
    k = keep
    ptr = lambda a: a.ctypes.data  # noqa: E731
    desc = _lib.BatchDesc(
        ctypes.sizeof(_lib.BatchDesc), _lib.ABI_VERSION, len(molecules), int(spherical),
        ptr(k[0]), ptr(k[1]), ptr(k[2]), ptr(k[3]),
        ptr(k[4]), ptr(k[5]), ptr(k[6]), ptr(k[7]), ptr(k[8]), ptr(k[9]), len(pe),
        ptr(k[10]), ptr(k[11]), ptr(k[12]), ptr(k[13]), ptr(k[14]), ptr(k[15]), len(ae),
    )
    return desc, keep


class NativePlan:
    """Owns a ``vqc_plan`` for a fixed batch topology."""

    def __init__(self, molecules: list[MoleculeSpec], spherical: bool = True):
        self.molecules = molecules
        self.spherical = spherical
        desc, self._keep = batch_descriptor(molecules, spherical)
        handle = ctypes.c_void_p()
        _lib.call("vqc_plan_create", ctypes.byref(desc), ctypes.byref(handle))
        self.handle = handle
        tot = [ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()]
        _lib.call("vqc_plan_totals", handle, *[ctypes.byref(t) for t in tot])
        self.mat_total, self.met_total, self.a_total = (int(t.value) for t in tot[:3])
        self.natom = int(tot[3].value)
        self.layout: list[MoleculeLayout] = []
        for i, mol in enumerate(molecules):
            info = _lib.MoleculeInfo()
            _lib.call("vqc_plan_molecule", handle, i, ctypes.byref(info))
            self.layout.append(
                MoleculeLayout(info.nao, info.naux, info.natom, info.atom_offset,
                               info.mat_offset, info.met_offset, info.a_offset, mol.nocc)
            )

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            _lib.lib().vqc_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def charges(self) -> np.ndarray:
        return np.concatenate([m.atomic_numbers for m in self.molecules]).astype(np.float64)

    def coordinates(self) -> np.ndarray:
        return np.concatenate([m.coordinates for m in self.molecules], axis=0)

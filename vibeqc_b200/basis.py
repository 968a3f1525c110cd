"""Basis sets, shell expansion, normalisation and the Cartesian->spherical map.

Conventions follow the reference's basis records
(``python/generativeqc/basis.py:20-23``): contraction coefficients multiply
*normalised primitives* and each contracted function is then normalised;
Cartesian components are in CCA order (xx, xy, xz, yy, yz, zz, ...); real
spherical functions use the PySCF/libcint order (p: x, y, z; l >= 2:
m = -l..l).  Shells are the reference's ``Shell(atom_index, angular_momentum,
primitives)`` records (``python/generativeqc/_api_types.py:53-63``); general
contractions are split into one shell per coefficient column.
"""

from __future__ import annotations

import json
import math
from dataclasses import dataclass
from functools import lru_cache
from pathlib import Path
from typing import Iterable, Sequence

import numpy as np

SYMBOLS = (
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn "
    "Ga Ge As Se Br Kr"
).split()

_DATA = Path(__file__).with_name("data") / "basis_sets.json"


def atomic_number(element: str | int) -> int:
    if isinstance(element, (int, np.integer)):
        z = int(element)
        if not 1 <= z <= len(SYMBOLS):
            raise ValueError(f"unsupported atomic number {z}")
        return z
    key = str(element).strip().capitalize()
    if key not in SYMBOLS:
        raise ValueError(f"unknown element symbol {element!r}")
    return SYMBOLS.index(key) + 1


@dataclass(frozen=True)
class Primitive:
    exponent: float
    coefficient: float


@dataclass(frozen=True)
class Shell:
    atom_index: int
    angular_momentum: int
    primitives: tuple[Primitive, ...]


@dataclass(frozen=True)
class BasisSet:
    """Per-element shell records: ``{Z: ((l, exponents, coefficient_columns), ...)}``."""

    name: str
    elements: dict

    def shells_for(self, z: int) -> tuple:
        try:
            return self.elements[z]
        except KeyError:
            raise ValueError(f"basis {self.name!r} has no data for Z={z}") from None


@lru_cache(maxsize=None)
def _bundled() -> dict:
    return json.loads(_DATA.read_text())


def bundled_basis_names() -> tuple[str, ...]:
    return tuple(k for k in _bundled() if not k.startswith("_"))


def load_basis(name: str | BasisSet) -> BasisSet:
    if isinstance(name, BasisSet):
        return name
    key = str(name).strip().lower()
    data = _bundled()
    if key not in data or key.startswith("_"):
        raise ValueError(f"unknown basis {name!r}; bundled: {bundled_basis_names()}")
    elements = {}
    for z, rows in data[key].items():
        elements[int(z)] = tuple(
            (
                int(r["l"]),
                tuple(float(e) for e in r["exponents"]),
                tuple(tuple(float(c) for c in col) for col in r["coefficients"]),
            )
            for r in rows
        )
    return BasisSet(key, elements)


def expand_shells(atomic_numbers: Sequence[int], basis: str | BasisSet | Sequence[Shell]) -> list[Shell]:
    """Shells for a molecule, atom by atom; general contractions are split."""
    if not isinstance(basis, (str, BasisSet)):
        shells = list(basis)
        for s in shells:
            if not isinstance(s, Shell):
                raise TypeError("explicit basis must be a sequence of Shell records")
            if not 0 <= s.atom_index < len(atomic_numbers):
                raise ValueError("shell atom_index out of range")
        return shells
    bs = load_basis(basis)
    out: list[Shell] = []
    for atom, z in enumerate(atomic_numbers):
        for l, exps, cols in bs.shells_for(int(z)):
            for col in cols:
                prims = tuple(
                    Primitive(e, c) for e, c in zip(exps, col) if c != 0.0
                )
                out.append(Shell(atom, l, prims))
    return out


# --------------------------------------------------------------------------
# Normalisation
# --------------------------------------------------------------------------

def double_factorial(n: int) -> int:
    return 1 if n <= 0 else n * double_factorial(n - 2)


def primitive_norm(alpha: float, l: int) -> float:
    """Normalisation of x^l exp(-alpha r^2) (the 'axis' Cartesian component)."""
    return (2.0 * alpha / math.pi) ** 0.75 * (4.0 * alpha) ** (l / 2.0) / math.sqrt(
        double_factorial(2 * l - 1)
    )


def normalized_coefficients(shell: Shell) -> tuple[np.ndarray, np.ndarray]:
    """(exponents, coefficients) with primitive and contraction norms folded in.

    The result multiplies x^lx y^ly z^lz exp(-a r^2) for every Cartesian
    component; the axis component x^l of the contracted function has unit norm.
    """
    l = shell.angular_momentum
    a = np.array([p.exponent for p in shell.primitives], dtype=np.float64)
    c = np.array([p.coefficient for p in shell.primitives], dtype=np.float64)
    c = c * np.array([primitive_norm(x, l) for x in a])
    s = a[:, None] + a[None, :]
    overlap = (math.pi / s) ** 1.5 * double_factorial(2 * l - 1) / (2.0 * s) ** l
    norm2 = float(c @ overlap @ c)
    if not norm2 > 0.0:
        raise ValueError("contracted shell has zero norm")
    return a, c / math.sqrt(norm2)


# --------------------------------------------------------------------------
# Cartesian components and the spherical transform
# --------------------------------------------------------------------------

@lru_cache(maxsize=None)
def cartesian_components(l: int) -> tuple[tuple[int, int, int], ...]:
    out = []
    for lx in range(l, -1, -1):
        for ly in range(l - lx, -1, -1):
            out.append((lx, ly, l - lx - ly))
    return tuple(out)


def ncart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def nsph(l: int) -> int:
    return 2 * l + 1


def _cart_gram(l: int) -> np.ndarray:
    """<x^a y^b z^c | x^d y^e z^f> / <x^l|x^l> for one exponent (radial part cancels)."""
    comps = cartesian_components(l)
    g = np.zeros((len(comps), len(comps)))
    for i, p in enumerate(comps):
        for j, q in enumerate(comps):
            s = [p[k] + q[k] for k in range(3)]
            if any(v % 2 for v in s):
                continue
            g[i, j] = (
                double_factorial(s[0] - 1)
                * double_factorial(s[1] - 1)
                * double_factorial(s[2] - 1)
                / double_factorial(2 * l - 1)
            )
    return g


def _solid_harmonic(l: int, m: int) -> dict:
    """Real solid harmonic r^l S_lm as {(lx, ly, lz): coefficient}.

    Closed form of Helgaker, Jorgensen and Olsen, "Molecular Electronic-Structure
    Theory", eqs. 6.4.47-6.4.50 (unnormalised here; normalised numerically).
    """
    am = abs(m)
    vm = 0.0 if m >= 0 else 0.5
    out: dict = {}
    for t in range((l - am) // 2 + 1):
        for u in range(t + 1):
            v = vm
            vmax = math.floor(am / 2.0 - vm) + vm
            while v <= vmax + 1e-9:
                c = (
                    (-1) ** int(round(t + v - vm))
                    * 0.25**t
                    * math.comb(l, t)
                    * math.comb(l - t, am + t)
                    * math.comb(t, u)
                    * math.comb(am, int(round(2 * v)))
                )
                lx = int(round(2 * t + am - 2 * (u + v)))
                ly = int(round(2 * (u + v)))
                lz = l - 2 * t - am
                key = (lx, ly, lz)
                out[key] = out.get(key, 0.0) + c
                v += 1.0
    return out


@lru_cache(maxsize=None)
def cart_to_sph(l: int) -> np.ndarray:
    """(2l+1, ncart) matrix: spherical = T @ cartesian (with common radial norm)."""
    comps = cartesian_components(l)
    index = {c: i for i, c in enumerate(comps)}
    g = _cart_gram(l)
    if l == 0:
        return np.ones((1, 1))
    if l == 1:
        return np.eye(3)  # p: x, y, z
    rows = []
    for m in range(-l, l + 1):
        v = np.zeros(len(comps))
        for key, c in _solid_harmonic(l, m).items():
            v[index[key]] += c
        v /= math.sqrt(v @ g @ v)
        rows.append(v)
    t = np.array(rows)
    t.setflags(write=False)
    return t


@lru_cache(maxsize=None)
def cart_to_cart(l: int) -> np.ndarray:
    """Cartesian representation: each component scaled to unit norm."""
    g = _cart_gram(l)
    return np.diag(1.0 / np.sqrt(np.diag(g)))


def transform_matrix(l: int, spherical: bool) -> np.ndarray:
    return cart_to_sph(l) if spherical else cart_to_cart(l)


def nfunc(l: int, spherical: bool) -> int:
    return nsph(l) if spherical else ncart(l)


def count_functions(shells: Iterable[Shell], spherical: bool = True) -> int:
    return sum(nfunc(s.angular_momentum, spherical) for s in shells)

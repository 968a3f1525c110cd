"""Seeded synthetic geometries for the DF-RHF workloads.

Every generator returns a list of ``(symbol, (x, y, z))`` tuples in Bohr, the
public atom form accepted by ``Calculator.singlepoint`` and
``Calculator.prepare_batch`` (reference ``python/generativeqc/_api_types.py:24-50``).

Workloads (all inputs are synthetic; no public benchmark set is used):

* water clusters: rigid waters (O-H 0.9572 A, H-O-H 104.52 deg) centred on the
  sites of a cubic lattice of 3.1 A spacing, each with a uniformly random
  orientation (unit quaternion from normal draws) and N(0, 0.05 A) jitter on
  every atom;
* all-trans alkanes C_nH_{2n+2}: C-C 1.53 A, C-H 1.09 A, tetrahedral angles,
  N(0, 0.02 A) jitter.
"""

from __future__ import annotations

import math

import numpy as np

BOHR_PER_ANGSTROM = 1.0 / 0.52917721092

WATER_OH = 0.9572
WATER_ANGLE = math.radians(104.52)
LATTICE_SPACING = 3.1


def _quaternion_rotation(q: np.ndarray) -> np.ndarray:
    w, x, y, z = q
    return np.array(
        [
            [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
            [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
            [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)],
        ]
    )


def near_cubic_lattice(n: int) -> tuple[int, int, int]:
    """Smallest (a, b, c) with a >= b >= c >= 1, a - c <= 1 and a*b*c >= n.

    The sequence is 1x1x1, 2x1x1, 2x2x1, 2x2x2, 3x2x2, 3x3x2, 3x3x3, ...
    """
    if n < 1:
        raise ValueError("a cluster needs at least one water")
    dims = [1, 1, 1]
    while dims[0] * dims[1] * dims[2] < n:
        # grow the smallest axis; the order keeps a >= b >= c
        i = dims.index(min(dims))
        dims[i] += 1
        dims.sort(reverse=True)
    return tuple(dims)  # type: ignore[return-value]


def water_cluster(
    n: int,
    seed: int | np.random.Generator = 0,
    lattice: tuple[int, int, int] | None = None,
    jitter: float = 0.05,
) -> list[tuple[str, tuple[float, float, float]]]:
    """(H2O)_n on the first ``n`` sites of a cubic lattice, x slowest, z fastest.

    The random stream is consumed per site: four normals for the orientation,
    then a 3x3 block of jitter normals (O, H, H).
    """
    rng = seed if isinstance(seed, np.random.Generator) else np.random.default_rng(seed)
    if lattice is None:
        lattice = near_cubic_lattice(n)
    base = np.array(
        [
            [0.0, 0.0, 0.0],
            [WATER_OH, 0.0, 0.0],
            [WATER_OH * math.cos(WATER_ANGLE), WATER_OH * math.sin(WATER_ANGLE), 0.0],
        ]
    )
    sites = [
        (ix, iy, iz)
        for ix in range(lattice[0])
        for iy in range(lattice[1])
        for iz in range(lattice[2])
    ][:n]
    if len(sites) < n:
        raise ValueError("lattice too small for the requested cluster")
    atoms = []
    for ix, iy, iz in sites:
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        rot = _quaternion_rotation(q)
        centre = np.array([ix, iy, iz], dtype=np.float64) * LATTICE_SPACING
        xyz = base @ rot.T + centre + rng.normal(0.0, jitter, size=(3, 3))
        for sym, p in zip("OHH", xyz):
            atoms.append((sym, tuple(float(v) for v in p * BOHR_PER_ANGSTROM)))
    return atoms


def water_cluster_batch(
    count: int = 256, n_min: int = 2, n_max: int = 16, seed: int = 0
) -> list[list[tuple[str, tuple[float, float, float]]]]:
    """Ragged batch: sizes n ~ U{n_min..n_max}; cluster i uses stream (seed, i)."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(n_min, n_max + 1, size=count)
    return [
        water_cluster(int(n), np.random.default_rng([seed, i])) for i, n in enumerate(sizes)
    ]


def alkane(
    n: int, seed: int | np.random.Generator = 0, jitter: float = 0.02
) -> list[tuple[str, tuple[float, float, float]]]:
    """All-trans C_nH_{2n+2} zig-zag chain along x, in the xy plane."""
    if n < 1:
        raise ValueError("an alkane needs at least one carbon")
    rng = seed if isinstance(seed, np.random.Generator) else np.random.default_rng(seed)
    cc, ch = 1.53, 1.09
    tet = math.acos(-1.0 / 3.0)
    half = tet / 2.0
    dx = cc * math.sin(half)
    dy = cc * math.cos(half)
    carbons = [np.array([i * dx, (i % 2) * dy, 0.0]) for i in range(n)]
    atoms: list[tuple[str, np.ndarray]] = [("C", c) for c in carbons]
    for i, c in enumerate(carbons):
        # the two in-plane bond directions (to neighbours, real or virtual)
        up = 1.0 if i % 2 == 0 else -1.0  # direction pointing away from the chain
        prev_dir = np.array([-dx, (dy if i % 2 == 0 else -dy), 0.0]) / cc
        next_dir = np.array([dx, (dy if i % 2 == 0 else -dy), 0.0]) / cc
        bisector = -(prev_dir + next_dir)
        bisector /= np.linalg.norm(bisector)
        normal = np.array([0.0, 0.0, 1.0])
        # out-of-plane pair of hydrogens: tetrahedral around the bisector
        for s in (1.0, -1.0):
            d = math.cos(half) * bisector + s * math.sin(half) * normal
            atoms.append(("H", c + ch * d))
        del up
        if i == 0 or i == n - 1:
            # terminal carbon: the missing neighbour direction gets a hydrogen
            d = prev_dir if i == 0 else next_dir
            if n == 1:
                d = prev_dir
            atoms.append(("H", c + ch * d))
            if n == 1:
                atoms.append(("H", c + ch * next_dir))
    out = []
    for sym, p in atoms:
        p = p + rng.normal(0.0, jitter, size=3)
        out.append((sym, tuple(float(v) for v in p * BOHR_PER_ANGSTROM)))
    return out


def alkane_batch(
    count: int = 64, n_min: int = 4, n_max: int = 20, seed: int = 0
) -> list[list[tuple[str, tuple[float, float, float]]]]:
    rng = np.random.default_rng(seed)
    sizes = rng.integers(n_min, n_max + 1, size=count)
    return [alkane(int(n), np.random.default_rng([seed, i])) for i, n in enumerate(sizes)]

"""Generate golden DF-RHF energies and forces from the reference implementation.

This script imports the reference's own Python API (``generativeqc``) over its
CPU density-fitting library and records energies, analytic forces and SCF
iteration counts for small seeded systems.  It needs the reference checkout and
a CPU build of its native library:

    GENERATIVEQC_LIBRARY=/path/to/libgenerativeqc.so \\
    python tests/golden/make_golden.py /path/to/generativeqc [case ...]

The output ``tests/golden/df_rhf_golden.json`` is committed; tests and the
oracle only read that file.  Geometries come from :mod:`vibeqc_b200.geometry`,
so the inputs are reproducible without the reference.
"""

from __future__ import annotations

import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from vibeqc_b200 import geometry  # noqa: E402

OUT = HERE / "df_rhf_golden.json"

# a single-water smoke geometry (Bohr) with a symmetric frame
WATER_SMOKE = [("O", (0.0, 0.0, 0.0)), ("H", (0.0, 1.432, 1.107)), ("H", (0.0, -1.432, 1.107))]


def cases() -> dict:
    return {
        "h2o_def2svp_auxdef2svp": dict(atoms=WATER_SMOKE, basis="def2-svp", aux="def2-svp"),
        "h2o_def2svp_jkfit": dict(
            atoms=geometry.water_cluster(1, 11), basis="def2-svp", aux="cc-pvdz-jkfit"
        ),
        "h2o_ccpvdz_jkfit": dict(
            atoms=geometry.water_cluster(1, 12), basis="cc-pvdz", aux="cc-pvdz-jkfit"
        ),
        "h2o_def2tzvp_jkfit": dict(
            atoms=geometry.water_cluster(1, 13), basis="def2-tzvp", aux="cc-pvdz-jkfit"
        ),
        "h2o2_def2svp_jkfit": dict(
            atoms=geometry.water_cluster(2, np.random.default_rng([0, 7])),
            basis="def2-svp",
            aux="cc-pvdz-jkfit",
        ),
        "h2o3_def2svp_jkfit": dict(
            atoms=geometry.water_cluster(3, np.random.default_rng([0, 3])),
            basis="def2-svp",
            aux="cc-pvdz-jkfit",
        ),
        "ethane_def2svp_auxdef2tzvp": dict(
            atoms=geometry.alkane(2, 5), basis="def2-svp", aux="def2-tzvp"
        ),
        "nh3_ccpvdz_jkfit": dict(
            atoms=[
                ("N", (0.0, 0.0, 0.2)),
                ("H", (1.77, 0.0, -0.5)),
                ("H", (-0.885, 1.533, -0.5)),
                ("H", (-0.885, -1.533, -0.55)),
            ],
            basis="cc-pvdz",
            aux="cc-pvdz-jkfit",
        ),
        "h2o4_ccpvdz_jkfit_seed0": dict(
            atoms=geometry.water_cluster(4, 0, lattice=(2, 2, 1)),
            basis="cc-pvdz",
            aux="cc-pvdz-jkfit",
        ),
    }


def _reference_basis(ref_root: Path, name: str):
    ident = ref_root / "benchmarks/results/issue206-practical-auxiliary/identity"
    if name in ("cc-pvdz", "cc-pvdz-jkfit"):
        from benchmarks._retained_basis import load_retained_basis

        return load_retained_basis(ident / f"{name}.json")
    return name


def main() -> None:
    ref_root = Path(sys.argv[1])
    wanted = set(sys.argv[2:])
    sys.path[:0] = [str(ref_root / "python"), str(ref_root)]
    if "GENERATIVEQC_LIBRARY" not in os.environ:
        raise SystemExit("set GENERATIVEQC_LIBRARY to the reference CPU library")
    from generativeqc import Calculator

    results = json.loads(OUT.read_text()) if OUT.exists() else {}
    for name, case in cases().items():
        if wanted and name not in wanted:
            continue
        calc = Calculator(
            method="rhf",
            basis=_reference_basis(ref_root, case["basis"]),
            auxiliary_basis=_reference_basis(ref_root, case["aux"]),
            density_fitting="cpu",
            basis_representation="spherical",
            energy_tolerance=1e-10,
            density_tolerance=1e-8,
        )
        t0 = time.perf_counter()
        res = calc.singlepoint(case["atoms"], properties=("energy", "forces"))
        dt = time.perf_counter() - t0
        results[name] = {
            "atoms": [[s, list(p)] for s, p in case["atoms"]],
            "basis": case["basis"],
            "auxiliary_basis": case["aux"],
            "energy": float(res.energy),
            "forces": np.asarray(res.forces).tolist(),
            "converged": bool(res.converged),
            "iterations": int(res.iterations),
            "reference_seconds": round(dt, 3),
            "settings": "rhf, density_fitting=cpu, spherical, energy_tolerance=1e-10, "
            "density_tolerance=1e-8, density_fitting_relative_threshold=1e-10",
        }
        print(f"{name}: E={res.energy:.12f} it={res.iterations} t={dt:.1f}s", flush=True)
        OUT.write_text(json.dumps(results, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    main()

"""Energies and forces of workload molecules from the CPU oracle.

The oracle (``oracle/``) is an independent CPU restatement of the reference's
DF-RHF path whose energies and forces agree with the reference's own CPU
library on every case of ``df_rhf_golden.json`` (|dE| ~ 1e-11 Eh, max|dF| ~
1e-8 Eh/Bohr; ``tests/test_oracle.py``).  The molecules here are too large to
run through that scalar-BLAS library in reasonable time, so the pinned oracle
produces their fixtures:

* ``clusters``: from the 256-cluster ragged workload (``water_cluster_batch``
  with seed 0: n ~ U{2..16}), the first molecule of each size n in
  ``CLUSTER_SIZES``; def2-SVP / cc-pVDZ-JKFIT.
* ``alkanes``: from the 64-alkane workload (``alkane_batch`` with seed 0:
  n ~ U{4..20}), the first molecule of each chain length in ``ALKANE_SIZES``;
  def2-SVP standing in for cc-pVDZ (same H/C shell structure) and def2-TZVP as
  the auxiliary basis (no carbon JK-fit set is bundled).

    python tests/golden/make_oracle_fixtures.py [--max-cluster 12]

writes ``tests/golden/oracle_workload_fixtures.json``.  Geometries are stored
in Bohr with the batch index they come from.
"""

from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from oracle import oracle  # noqa: E402
from vibeqc_b200 import geometry  # noqa: E402

OUT = HERE / "oracle_workload_fixtures.json"
CLUSTER_SIZES = tuple(range(2, 17))
ALKANE_SIZES = (4, 5, 6, 8)


def first_of_each(sizes, wanted):
    pick = {}
    for i, n in enumerate(sizes):
        if int(n) in wanted and int(n) not in pick:
            pick[int(n)] = i
    return pick


def run(atoms, basis, aux):
    t0 = time.perf_counter()
    r = oracle.df_rhf(atoms, basis, aux, forces=True)
    assert r.converged
    return {
        "atoms": [[s, [float(v) for v in p]] for s, p in atoms],
        "basis": basis,
        "auxiliary_basis": aux,
        "energy": float(r.energy),
        "forces": np.asarray(r.forces).tolist(),
        "iterations": int(r.iterations),
        "nao": int(r.extra["nao"]),
        "naux": int(r.extra["naux"]),
        "oracle_seconds": round(time.perf_counter() - t0, 2),
    }


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--max-cluster", type=int, default=max(CLUSTER_SIZES))
    args = ap.parse_args()
    out = {"_provenance": "CPU oracle (oracle/oracle.py df_rhf), pinned against the reference's "
                          "own CPU DF-RHF goldens in df_rhf_golden.json",
           "clusters": {}, "alkanes": {}}
    rng = np.random.default_rng(0)
    sizes = rng.integers(2, 17, size=256)
    batch = geometry.water_cluster_batch(256, 2, 16, 0)
    for n, i in sorted(first_of_each(sizes, [c for c in CLUSTER_SIZES if c <= args.max_cluster]).items()):
        rec = run(batch[i], "def2-svp", "cc-pvdz-jkfit")
        rec.update(batch_index=i, n=n, workload="water_cluster_batch(256, 2, 16, seed=0)")
        out["clusters"][f"h2o{n}_idx{i}"] = rec
        print(f"(H2O){n} idx {i}: E={rec['energy']:.10f} ({rec['oracle_seconds']} s)", flush=True)
        OUT.write_text(json.dumps(out, indent=1) + "\n")
    rng = np.random.default_rng(0)
    sizes = rng.integers(4, 21, size=64)
    alk = geometry.alkane_batch(64, 4, 20, 0)
    for n, i in sorted(first_of_each(sizes, ALKANE_SIZES).items()):
        rec = run(alk[i], "def2-svp", "def2-tzvp")
        rec.update(batch_index=i, n=n, workload="alkane_batch(64, 4, 20, seed=0)")
        out["alkanes"][f"c{n}_idx{i}"] = rec
        print(f"C{n} idx {i}: E={rec['energy']:.10f} ({rec['oracle_seconds']} s)", flush=True)
        OUT.write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()

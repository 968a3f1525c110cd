"""Extract the basis-set records this package needs into ``basis_sets.json``.

Run once in a checkout that has the GenerativeQC sources next to it:

    python vibeqc_b200/data/extract_basis.py /path/to/generativeqc

Sources (data only, copied verbatim as decimal values):

* ``python/generativeqc/data/basis_pack.json`` -- def2-SVP, def2-TZVP and
  STO-3G for H-Ar (Basis Set Exchange 0.11).
* ``benchmarks/results/issue206-practical-auxiliary/identity/cc-pvdz.json`` and
  ``cc-pvdz-jkfit.json`` -- cc-pVDZ and cc-pVDZ-JKFIT for H, N, O (PySCF 2.14.0
  packaged basis data, Apache-2.0).

The output keeps every exponent and contraction coefficient as written in the
source; general contractions keep their coefficient columns so that the shell
expansion in :mod:`vibeqc_b200.basis` can split them.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path


def _pack_record(elements: dict) -> dict:
    out = {}
    for z, shells in elements.items():
        rows = []
        for shell in shells:
            coefs = shell["coefficients"]
            if coefs and not isinstance(coefs[0], list):
                coefs = [coefs]
            rows.append(
                {
                    "l": int(shell["angular_momentum"]),
                    "exponents": [str(e) for e in shell["exponents"]],
                    "coefficients": [[str(c) for c in col] for col in coefs],
                }
            )
        out[str(int(z))] = rows
    return out


def main(root: Path) -> None:
    pack = json.loads((root / "python/generativeqc/data/basis_pack.json").read_text())
    result = {"_source": {}}
    for name in ("def2-svp", "def2-tzvp", "sto-3g"):
        result[name] = _pack_record(pack["bases"][name]["elements"])
        result["_source"][name] = pack["source"]
    ident = root / "benchmarks/results/issue206-practical-auxiliary/identity"
    for name in ("cc-pvdz", "cc-pvdz-jkfit"):
        rec = json.loads((ident / f"{name}.json").read_text())
        elements = {el["atomic_number"]: el["shells"] for el in rec["elements"]}
        result[name] = _pack_record(elements)
        prov = rec["provenance"]
        result["_source"][name] = f"{prov['source']} {prov['version']} ({prov['license']})"
    out = Path(__file__).with_name("basis_sets.json")
    out.write_text(json.dumps(result, separators=(",", ":"), sort_keys=True) + "\n")
    print(f"wrote {out} ({out.stat().st_size} bytes)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python extract_basis.py <generativeqc source checkout>")
    main(Path(sys.argv[1]))

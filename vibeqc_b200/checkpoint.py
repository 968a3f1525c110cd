"""Restart files for prepared DF-RHF batches: converged densities as seeds.

Same container idea as the reference's HF checkpoints
(``python/generativeqc/checkpoint.py:1-8``: a fixed header, a checksummed
UTF-8 JSON manifest and contiguous little-endian IEEE-754 binary64 arrays in
C order; only the density and its source coordinates are reusable), with this
package's own schema: the reference's manifests carry its resolved-model
identities, so the two file formats are not interchangeable.

Layout::

    8 bytes  magic b"VQCDFCP1"
    8 bytes  manifest length L (little-endian u64)
    32 bytes SHA-256 of the manifest
    L bytes  manifest (UTF-8 JSON)
    arrays   binary64, at the offsets the manifest lists (relative to the
             end of the manifest), each with its own SHA-256

A checkpoint only proposes seeds: ``load_checkpoint`` checks the file and
its compatibility with the target batch (basis, auxiliary basis,
representation, atomic numbers, charge, multiplicity, function counts) and
places each compatible density as the item's warm start; the next
``execute`` converges the target equations from it.
"""

from __future__ import annotations

import hashlib
import json
import os
import struct
import tempfile
from pathlib import Path

import numpy as np
import torch

MAGIC = b"VQCDFCP1"
HEADER = struct.Struct("<8sQ32s")
SCHEMA = "vibeqc_b200.df_rhf_checkpoint"
ARRAY_FORMAT = "ieee754-binary64-little-endian-c-order"
MAX_MANIFEST = 4 << 20


class CheckpointError(ValueError):
    """A checkpoint is malformed or incompatible; no seed has been applied."""


def _item_identity(batch, i: int) -> dict:
    mol = batch._molecules[i]
    from . import basis as bas

    calc = batch._calc
    return {
        "atomic_numbers": [int(z) for z in mol.atomic_numbers],
        "charge": int(mol.charge),
        "multiplicity": int(mol.multiplicity),
        "nao": int(bas.count_functions(mol.orbital_shells, calc.spherical)),
        "naux": int(bas.count_functions(mol.aux_shells, calc.spherical)),
    }


def _model(batch) -> dict:
    calc = batch._calc
    return {"method": calc.method, "basis": str(calc.basis).lower(),
            "auxiliary_basis": str(calc.auxiliary_basis).lower(),
            "representation": "spherical" if calc.spherical else "cartesian"}


def save_checkpoint(batch, path, *, max_bytes: int = 256 << 20) -> dict:
    """Atomically write the batch's retained densities (items without one keep empty slots)."""
    items, blobs, arrays = [], [], []
    offset = 0
    for i in range(batch.size):
        rec = {"index": i, **_item_identity(batch, i), "seed": batch._warm[i] is not None}
        if rec["seed"]:
            dens = batch._warm[i].detach().to("cpu", torch.float64).numpy()
            xyz = np.asarray(batch._source_coordinates[i], dtype=np.float64)
            for name, arr in (("density", dens), ("coordinates", xyz)):
                raw = np.ascontiguousarray(arr, dtype="<f8").tobytes()
                blobs.append({"name": f"{name}/{i}", "shape": list(arr.shape), "offset": offset,
                              "bytes": len(raw), "sha256": hashlib.sha256(raw).hexdigest()})
                arrays.append(raw)
                offset += len(raw)
        items.append(rec)
    if offset > max_bytes:
        raise CheckpointError(f"checkpoint arrays need {offset} bytes > max_bytes={max_bytes}")
    manifest = json.dumps({"schema": SCHEMA, "schema_version": 1, "array_format": ARRAY_FORMAT,
                           "model": _model(batch), "items": items, "blobs": blobs},
                          sort_keys=True, separators=(",", ":"), allow_nan=False).encode("utf-8")
    header = HEADER.pack(MAGIC, len(manifest), hashlib.sha256(manifest).digest())
    path = Path(path)
    fd, tmp = tempfile.mkstemp(prefix=path.name + ".", dir=str(path.parent or Path(".")))
    try:
        with os.fdopen(fd, "wb") as f:
            f.write(header)
            f.write(manifest)
            for raw in arrays:
                f.write(raw)
        os.replace(tmp, path)
    except BaseException:
        if os.path.exists(tmp):
            os.unlink(tmp)
        raise
    return {"items": len(items), "seeds": sum(1 for r in items if r["seed"]),
            "bytes": HEADER.size + len(manifest) + offset}


def read_checkpoint(path, *, max_bytes: int = 256 << 20) -> tuple[dict, dict]:
    """(manifest, {blob name: array}) after checking every checksum."""
    data = Path(path).read_bytes()
    if len(data) < HEADER.size:
        raise CheckpointError("truncated checkpoint header")
    magic, mlen, digest = HEADER.unpack_from(data, 0)
    if magic != MAGIC:
        raise CheckpointError("not a DF-RHF checkpoint of this package")
    if mlen > MAX_MANIFEST or HEADER.size + mlen > len(data):
        raise CheckpointError("invalid manifest length")
    raw = data[HEADER.size:HEADER.size + mlen]
    if hashlib.sha256(raw).digest() != digest:
        raise CheckpointError("manifest checksum mismatch")
    try:
        doc = json.loads(raw.decode("utf-8"))
    except (UnicodeDecodeError, json.JSONDecodeError) as e:
        raise CheckpointError(f"manifest is not JSON: {e}") from None
    if doc.get("schema") != SCHEMA or doc.get("schema_version") != 1 \
            or doc.get("array_format") != ARRAY_FORMAT:
        raise CheckpointError("unsupported checkpoint schema")
    body = data[HEADER.size + mlen:]
    if len(body) > max_bytes:
        raise CheckpointError("checkpoint arrays exceed max_bytes")
    arrays = {}
    for blob in doc.get("blobs", []):
        off, nbytes, shape = blob["offset"], blob["bytes"], tuple(blob["shape"])
        if off < 0 or off + nbytes > len(body) or int(np.prod(shape)) * 8 != nbytes:
            raise CheckpointError(f"blob {blob['name']} out of range")
        chunk = body[off:off + nbytes]
        if hashlib.sha256(chunk).hexdigest() != blob["sha256"]:
            raise CheckpointError(f"blob {blob['name']} checksum mismatch")
        arrays[blob["name"]] = np.frombuffer(chunk, dtype="<f8").reshape(shape).astype(np.float64)
    return doc, arrays


def load_checkpoint(batch, path, *, allow_warm: bool = False, strict: bool = True,
                    max_bytes: int = 256 << 20) -> dict:
    """Place the file's densities as warm starts of ``batch``.

    ``allow_warm=False`` (exact restart) also requires the item's prepared
    coordinates to equal the checkpoint's source coordinates.  With
    ``strict=True`` any incompatible item rejects the whole file (nothing is
    applied); with ``strict=False`` incompatible items keep their state.
    Returns a report with the seeded and skipped indices.
    """
    doc, arrays = read_checkpoint(path, max_bytes=max_bytes)
    if doc["model"] != _model(batch):
        raise CheckpointError(f"checkpoint model {doc['model']} differs from {_model(batch)}")
    items = doc["items"]
    if len(items) != batch.size:
        raise CheckpointError("checkpoint item count differs from the batch size")
    seeds, skipped = {}, {}
    for i, rec in enumerate(items):
        if rec.get("index") != i:
            raise CheckpointError("checkpoint items are out of order")
        if not rec.get("seed"):
            continue
        want = _item_identity(batch, i)
        got = {k: rec.get(k) for k in want}
        reason = None
        if got != want:
            reason = "system identity differs"
        else:
            dens = arrays.get(f"density/{i}")
            xyz = arrays.get(f"coordinates/{i}")
            n = want["nao"]
            shape = (2, n, n) if batch._calc.method == "uhf" else (n, n)
            if dens is None or xyz is None or dens.shape != shape or not np.isfinite(dens).all():
                reason = "missing or invalid density"
            elif not allow_warm and not np.array_equal(xyz, batch._molecules[i].coordinates):
                reason = "coordinates differ (pass allow_warm=True for a changed geometry)"
        if reason is not None:
            if strict:
                raise CheckpointError(f"item {i}: {reason}")
            skipped[i] = reason
            continue
        seeds[i] = (dens, xyz)
    dev = batch._calc.device
    for i, (dens, xyz) in seeds.items():
        batch._warm[i] = torch.as_tensor(dens, dtype=torch.float64).to(dev)
        batch._warm_origin[i] = "checkpoint"
        batch._source_coordinates[i] = xyz.copy()
    return {"seeded": sorted(seeds), "skipped": skipped}

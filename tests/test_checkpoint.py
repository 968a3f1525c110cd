"""Checkpoint files (host logic): round trip, checksums and compatibility rules.

A stand-in batch object carries what the checkpoint module reads from a
PreparedBatch (molecules, calculator model, retained densities and their
source coordinates); no device is needed.
"""

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from vibeqc_b200 import checkpoint as ck
from vibeqc_b200 import geometry
from vibeqc_b200.plan import make_molecule


def _batch(n=2, seed=0):
    mols = [make_molecule(geometry.water_cluster(k + 1, seed + k), "def2-svp", "cc-pvdz-jkfit")
            for k in range(n)]
    calc = SimpleNamespace(method="rhf", basis="def2-svp", auxiliary_basis="cc-pvdz-jkfit",
                           spherical=True, device=torch.device("cpu"))
    b = SimpleNamespace(_molecules=mols, _calc=calc, size=n, _warm=[None] * n,
                        _warm_origin=[None] * n, _source_coordinates=[None] * n)
    return b


def _seed(b, i, value):
    nao = 24 * (i + 1)
    d = np.full((nao, nao), value)
    b._warm[i] = torch.tensor(d)
    b._source_coordinates[i] = b._molecules[i].coordinates.copy()


def test_round_trip_and_exact_restart(tmp_path):
    src = _batch()
    _seed(src, 0, 0.25)
    _seed(src, 1, -1.5)
    info = ck.save_checkpoint(src, tmp_path / "a.ckpt")
    assert info["seeds"] == 2
    dst = _batch()
    rep = ck.load_checkpoint(dst, tmp_path / "a.ckpt")
    assert rep["seeded"] == [0, 1] and not rep["skipped"]
    assert torch.equal(dst._warm[1], src._warm[1])
    assert dst._warm_origin[0] == "checkpoint"


def test_items_without_a_seed_keep_empty_slots(tmp_path):
    src = _batch()
    _seed(src, 1, 0.5)
    ck.save_checkpoint(src, tmp_path / "b.ckpt")
    dst = _batch()
    rep = ck.load_checkpoint(dst, tmp_path / "b.ckpt")
    assert rep["seeded"] == [1] and dst._warm[0] is None


def test_changed_geometry_needs_allow_warm(tmp_path):
    src = _batch()
    _seed(src, 0, 0.25)
    src._source_coordinates[0] = src._source_coordinates[0] + 0.01
    ck.save_checkpoint(src, tmp_path / "c.ckpt")
    with pytest.raises(ck.CheckpointError, match="coordinates differ"):
        ck.load_checkpoint(_batch(), tmp_path / "c.ckpt")
    dst = _batch()
    rep = ck.load_checkpoint(dst, tmp_path / "c.ckpt", strict=False)
    assert rep["seeded"] == [] and 0 in rep["skipped"] and dst._warm[0] is None
    rep = ck.load_checkpoint(dst, tmp_path / "c.ckpt", allow_warm=True)
    assert rep["seeded"] == [0]


def test_corruption_and_model_mismatch_reject_the_file(tmp_path):
    src = _batch()
    _seed(src, 0, 0.25)
    p = tmp_path / "d.ckpt"
    ck.save_checkpoint(src, p)
    raw = bytearray(p.read_bytes())
    raw[-3] ^= 0x40  # flip a bit inside the last array
    bad = tmp_path / "e.ckpt"
    bad.write_bytes(bytes(raw))
    with pytest.raises(ck.CheckpointError, match="checksum"):
        ck.load_checkpoint(_batch(), bad)
    raw = bytearray(p.read_bytes())
    raw[60] ^= 0x01  # inside the manifest
    bad.write_bytes(bytes(raw))
    with pytest.raises(ck.CheckpointError, match="checksum"):
        ck.load_checkpoint(_batch(), bad)
    other = _batch()
    other._calc.auxiliary_basis = "def2-tzvp"
    with pytest.raises(ck.CheckpointError, match="model"):
        ck.load_checkpoint(other, p)
    with pytest.raises(ck.CheckpointError, match="item count"):
        ck.load_checkpoint(_batch(n=3), p)
    bad.write_bytes(b"NOTACKPT" + bytes(64))
    with pytest.raises(ck.CheckpointError, match="not a DF-RHF checkpoint"):
        ck.load_checkpoint(_batch(), bad)

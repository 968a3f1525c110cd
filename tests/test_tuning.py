"""Autotuning table (host logic) and the library's tuning knobs (no device work)."""

import ctypes

import pytest

from vibeqc_b200 import _lib, tuning


def test_schedule_validation():
    with pytest.raises(ValueError):
        tuning.Schedule(whiten="bf16")
    with pytest.raises(ValueError):
        tuning.Schedule(sp2_steps=5)
    with pytest.raises(ValueError):
        tuning.Schedule(gram_waves=0)


def test_table_round_trip_and_nearest_lookup(tmp_path):
    t = tuning.TuningTable(meta={"device": "test"})
    t.entries[tuning.shape_key(96, 464, 20)] = tuning.Schedule("fp64", 4, 4)
    t.entries[tuning.shape_key(384, 1856, 80)] = tuning.Schedule("int8", 1, 16)
    t.timings[tuning.shape_key(96, 464, 20)] = {"whiten": {"int8": 2.0, "fp64": 1.0}}
    p = tmp_path / "t.json"
    t.save(p)
    u = tuning.TuningTable.load(p)
    assert u.lookup(96, 464, 20) == tuning.Schedule("fp64", 4, 4)
    assert u.lookup(360, 1740, 75) == tuning.Schedule("int8", 1, 16)  # nearest N
    assert u.lookup(100, 480, 21).whiten == "fp64"
    assert u.timings[tuning.shape_key(96, 464, 20)]["whiten"]["fp64"] == 1.0
    assert tuning.TuningTable.load(tmp_path / "missing.json").lookup(10, 20, 3) == tuning.DEFAULT
    (tmp_path / "bad.json").write_text('{"schema": "other"}')
    with pytest.raises(ValueError):
        tuning.TuningTable.load(tmp_path / "bad.json")


def test_committed_table_is_valid_when_present():
    t = tuning.TuningTable.load()
    for key, sched in t.entries.items():
        assert len(key.split("/")) == 3 and isinstance(sched, tuning.Schedule)


def test_library_knobs_are_range_checked():
    lib = _lib.lib()
    v = ctypes.c_int32()
    assert lib.vqc_tune_get(_lib.TUNE_GRAM_WAVES, ctypes.byref(v)) == 0
    old = v.value
    assert lib.vqc_tune_set(_lib.TUNE_GRAM_WAVES, 4) == 0
    assert lib.vqc_tune_get(_lib.TUNE_GRAM_WAVES, ctypes.byref(v)) == 0 and v.value == 4
    assert lib.vqc_tune_set(_lib.TUNE_GRAM_WAVES, 0) == 1
    assert lib.vqc_tune_set(99, 1) == 1
    assert lib.vqc_tune_get(99, ctypes.byref(v)) == 1
    assert lib.vqc_tune_set(_lib.TUNE_GRAM_WAVES, old) == 0

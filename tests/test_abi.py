"""The C-ABI library loads on a CPU-only host and exports every declared symbol."""

import ctypes
import re
from pathlib import Path

from vibeqc_b200 import _lib

INCLUDE = Path(__file__).resolve().parent.parent / "include"


def declared_symbols():
    names = set()
    for h in INCLUDE.glob("*.h"):
        text = h.read_text()
        names.update(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(vqc_\w+)\s*\(", text, re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "vqc_plan_create" in names and "vqc_int3c" in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_symbols()) <= set(_lib.exported_symbols())


def test_abi_version_and_error_path():
    lib = _lib.lib()
    assert lib.vqc_abi_version() == _lib.ABI_VERSION
    # invalid descriptor is rejected without touching a device
    desc = _lib.BatchDesc()
    desc.struct_size = 4
    handle = ctypes.c_void_p()
    status = lib.vqc_plan_create(ctypes.byref(desc), ctypes.byref(handle))
    assert status == 2  # GENERATIVEQC_STATUS_ABI_MISMATCH
    assert b"struct_size" in lib.vqc_last_error()


def test_df_gradient_rejects_mismatched_descriptors_before_any_device_work():
    lib = _lib.lib()
    desc = _lib.BatchDesc()
    desc.struct_size = 4  # not a vqc_batch_desc
    grad = (ctypes.c_double * 3)(7.0, 7.0, 7.0)
    res = _lib.DfGradientResources()
    status = lib.vqc_df_gradient(ctypes.byref(desc), grad, None, 0, None, 0, 0, 1 << 20, 0, grad, 3,
                                 ctypes.byref(res))
    assert status == 2 and b"struct_size" in lib.vqc_last_error()
    desc.struct_size = ctypes.sizeof(_lib.BatchDesc)
    desc.abi_version = _lib.ABI_VERSION
    res.struct_size = 8  # resources record of another ABI
    status = lib.vqc_df_gradient(ctypes.byref(desc), grad, None, 0, None, 0, 0, 1 << 20, 0, grad, 3,
                                 ctypes.byref(res))
    assert status == 2
    status = lib.vqc_df_gradient(ctypes.byref(desc), grad, None, 0, None, 0, 2, 1 << 20, 0, grad, 3,
                                 None)
    assert status == 1  # schedule must be 0 or 1
    assert list(grad) == [7.0, 7.0, 7.0]

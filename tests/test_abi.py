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
    assert status == 1
    assert b"struct_size" in lib.vqc_last_error()

"""ctypes binding of ``libvqc_b200.so`` (the C ABI declared in include/vqc_df.h).

The product path has no fallback: if the library is missing or fails to load,
every entry point raises.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().with_name("libvqc_b200.so")
ABI_VERSION = 1
TUNE_GRAM_WAVES = 1

STATUS = {
    0: "success",
    1: "invalid argument",
    2: "ABI mismatch",
    4: "not converged",
    5: "numerical failure",
    6: "CUDA error",
    7: "out of memory",
}


class VqcError(RuntimeError):
    def __init__(self, status: int, detail: str):
        super().__init__(f"{STATUS.get(status, status)}: {detail}")
        self.status = status
        self.detail = detail


class BatchDesc(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("abi_version", ctypes.c_uint32),
        ("nmol", ctypes.c_int32),
        ("spherical", ctypes.c_int32),
        ("mol_atom_offset", ctypes.c_void_p),
        ("mol_shell_offset", ctypes.c_void_p),
        ("mol_aux_offset", ctypes.c_void_p),
        ("atom_charge", ctypes.c_void_p),
        ("shell_l", ctypes.c_void_p),
        ("shell_atom", ctypes.c_void_p),
        ("shell_nprim", ctypes.c_void_p),
        ("shell_prim_off", ctypes.c_void_p),
        ("prim_exp", ctypes.c_void_p),
        ("prim_coef", ctypes.c_void_p),
        ("nprim", ctypes.c_int32),
        ("aux_l", ctypes.c_void_p),
        ("aux_atom", ctypes.c_void_p),
        ("aux_nprim", ctypes.c_void_p),
        ("aux_prim_off", ctypes.c_void_p),
        ("aux_exp", ctypes.c_void_p),
        ("aux_coef", ctypes.c_void_p),
        ("naux_prim", ctypes.c_int32),
    ]


class MoleculeInfo(ctypes.Structure):
    _fields_ = [
        ("nao", ctypes.c_int32),
        ("naux", ctypes.c_int32),
        ("natom", ctypes.c_int32),
        ("atom_offset", ctypes.c_int32),
        ("mat_offset", ctypes.c_int64),
        ("met_offset", ctypes.c_int64),
        ("a_offset", ctypes.c_int64),
    ]


class DfGradientResources(ctypes.Structure):
    """``vqc_df_gradient_resources`` (reference ``generativeqc_df_gradient_resources``)."""

    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("abi_version", ctypes.c_uint32),
        ("host_bytes", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64),
        ("host_to_device_bytes", ctypes.c_uint64),
        ("device_to_host_bytes", ctypes.c_uint64),
        ("weight_tile_elements", ctypes.c_uint64),
        ("tiles", ctypes.c_uint64),
        ("uploads", ctypes.c_uint64),
        ("stream_synchronizations", ctypes.c_uint64),
    ]


# name -> argtypes (every function returns int status unless listed below)
_P = ctypes.c_void_p
_SIGNATURES = {
    "vqc_last_error": ([], ctypes.c_char_p),
    "vqc_abi_version": ([], ctypes.c_uint32),
    "vqc_launch_count": ([], ctypes.c_uint64),
    "vqc_tune_set": ([ctypes.c_int32, ctypes.c_int32], ctypes.c_int),
    "vqc_tune_get": ([ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "vqc_plan_create": ([ctypes.POINTER(BatchDesc), ctypes.POINTER(_P)], ctypes.c_int),
    "vqc_plan_destroy": ([_P], ctypes.c_int),
    "vqc_plan_totals": ([_P, _P, _P, _P, _P], ctypes.c_int),
    "vqc_plan_molecule": ([_P, ctypes.c_int32, ctypes.POINTER(MoleculeInfo)], ctypes.c_int),
    "vqc_int1e": ([_P, _P, _P, _P, _P, _P], ctypes.c_int),
    "vqc_int2c": ([_P, _P, _P, _P], ctypes.c_int),
    "vqc_int3c": ([_P, _P, _P, _P], ctypes.c_int),
    "vqc_int3c_rows": ([_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P],
                       ctypes.c_int),
    "vqc_grad3c": ([_P, _P, _P, _P, _P], ctypes.c_int),
    "vqc_grad2c": ([_P, _P, _P, _P, _P], ctypes.c_int),
    "vqc_grad1e": ([_P, _P, _P, _P, _P, _P], ctypes.c_int),
    "vqc_df_gradient": ([ctypes.POINTER(BatchDesc), _P, _P, ctypes.c_size_t, _P, ctypes.c_size_t,
                         ctypes.c_uint32, ctypes.c_size_t, ctypes.c_size_t, _P, ctypes.c_size_t,
                         ctypes.POINTER(DfGradientResources)], ctypes.c_int),
    "vqc_ozaki_slice_rows": ([_P, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, ctypes.c_int64,
                              ctypes.c_int64, _P, ctypes.c_int32, _P, ctypes.c_int32, _P, _P],
                             ctypes.c_int),
    "vqc_ozaki_gemm": ([_P, _P, ctypes.c_int64, _P, _P, ctypes.c_int32, ctypes.c_int32,
                        ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P,
                        ctypes.c_int64, ctypes.c_int64, _P, _P], ctypes.c_int),
    "vqc_sp2_update": ([_P, _P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                        ctypes.c_double, _P, _P], ctypes.c_int),
    "vqc_unpack_aux_major": ([_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                              ctypes.c_int32, _P, _P], ctypes.c_int),
    "vqc_split_tf32": ([_P, _P, _P, ctypes.c_int64, _P], ctypes.c_int),
    "vqc_wait_selftest": ([ctypes.c_int32, _P, _P], ctypes.c_int),
    "vqc_tc_half_transform": ([_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                               ctypes.c_int32, _P, _P, _P, ctypes.c_int32, ctypes.c_int32,
                               ctypes.c_int32, _P, _P, _P, _P, _P, _P, _P], ctypes.c_int),
    "vqc_tc_gram": ([_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P, _P],
                    ctypes.c_int),
    "vqc_tc_gram_sym2": ([_P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P,
                          _P, _P], ctypes.c_int),
    "vqc_fitted_density_fp32_noalloc": ([_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                         ctypes.c_int32, _P, _P], ctypes.c_int),
    "vqc_anchor_combine": ([_P, _P, _P, _P, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                            ctypes.c_double, ctypes.c_int32, _P], ctypes.c_int),
    "vqc_fitted_density_fp32": ([_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                 ctypes.c_int32, _P, _P, _P], ctypes.c_int),
    "vqc_coulomb_fp32": ([_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                          ctypes.c_int32, _P, _P], ctypes.c_int),
    "vqc_coulomb_tma": ([_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                         ctypes.c_int32, _P, _P, _P], ctypes.c_int),
}

_lib = None


def exported_symbols() -> tuple[str, ...]:
    return tuple(_SIGNATURES)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m vibeqc_b200.build`"
            )
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.argtypes = args
            fn.restype = res
        if handle.vqc_abi_version() != ABI_VERSION:
            raise ImportError("libvqc_b200.so ABI version mismatch")
        _lib = handle
    return _lib


def check(status: int) -> None:
    if status != 0:
        raise VqcError(status, lib().vqc_last_error().decode(errors="replace"))


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def i32(values) -> np.ndarray:
    return np.ascontiguousarray(values, dtype=np.int32)


def f64(values) -> np.ndarray:
    return np.ascontiguousarray(values, dtype=np.float64)

"""Loads the CPU oracles (test infrastructure).

- ``port()``: oracle/_build/libsci_oracle.so, this repository's restatement of libsci's CPU
  arithmetic (oracle/sci_oracle.cpp); built with ``make -C oracle port`` when missing.
- ``reference()``: oracle/_ref/libsci_ref.so, libsci's own CPU path compiled from the reference
  sources (oracle/Makefile); None when it was never built.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

from libsci_b200.chunk import ChunkStruct

ROOT = Path(__file__).resolve().parent.parent
PORT = ROOT / "oracle" / "_build" / "libsci_oracle.so"
REF = ROOT / "oracle" / "_ref" / "libsci_ref.so"
P = ctypes.POINTER
_cache: dict[str, ctypes.CDLL | None] = {}


def port() -> ctypes.CDLL:
    if "port" in _cache:
        return _cache["port"]
    if not PORT.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "port"], check=True, capture_output=True)
    lib = ctypes.CDLL(str(PORT))
    lib.sci_oracle_execute.argtypes = [P(ChunkStruct), ctypes.c_void_p, ctypes.c_uint64]
    lib.sci_oracle_reduce.argtypes = [P(ChunkStruct), ctypes.c_uint32, ctypes.c_uint64, P(ctypes.c_double)]
    lib.sci_oracle_apply_f32.restype = ctypes.c_float
    lib.sci_oracle_apply_f32.argtypes = [ctypes.c_uint32, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int]
    lib.sci_oracle_apply_f64.restype = ctypes.c_double
    lib.sci_oracle_apply_f64.argtypes = [ctypes.c_uint32, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
    lib.sci_oracle_factor_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
    lib.sci_oracle_factor_f64.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
    lib.sci_oracle_substitute_f64.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_uint64, ctypes.c_uint64]
    lib.sci_oracle_product_rows.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_uint64] * 5
    lib.sci_oracle_tail_width.restype = ctypes.c_uint64
    lib.sci_oracle_execute_elements.argtypes = [ctypes.c_uint32, P(ChunkStruct), ctypes.c_void_p, ctypes.c_uint64]
    lib.sci_oracle_reduce_elements.argtypes = [ctypes.c_uint32, P(ChunkStruct), ctypes.c_uint32, ctypes.c_uint64,
                                               ctypes.c_void_p]
    _cache["port"] = lib
    return lib


def reference() -> ctypes.CDLL | None:
    if "ref" in _cache:
        return _cache["ref"]
    if not REF.exists():
        _cache["ref"] = None
        return None
    lib = ctypes.CDLL(str(REF))
    lib.sci_ref_execute.argtypes = [P(ChunkStruct), ctypes.c_void_p, ctypes.c_uint64]
    lib.sci_ref_reduce.restype = ctypes.c_double
    lib.sci_ref_reduce.argtypes = [P(ChunkStruct), ctypes.c_uint32, ctypes.c_uint64]
    lib.sci_ref_product.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]
    lib.sci_ref_factor_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
    lib.sci_ref_factor_f64.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
    lib.sci_ref_solve_f64.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_uint64] * 2
    lib.sci_ref_solve_f32.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_uint64] * 2
    lib.sci_ref_threads.restype = ctypes.c_uint64
    lib.sci_ref_record.argtypes = [ctypes.c_int, ctypes.c_int, P(ChunkStruct)]
    lib.sci_ref_workload_create.restype = ctypes.c_void_p
    lib.sci_ref_workload_create.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_uint64]
    lib.sci_ref_workload_step.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    lib.sci_ref_workload_output.restype = ctypes.c_void_p
    lib.sci_ref_workload_output.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.sci_ref_workload_destroy.argtypes = [ctypes.c_void_p]
    lib.sci_ref_plain_create.restype = ctypes.c_void_p
    lib.sci_ref_plain_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
    lib.sci_ref_plain_step.restype = ctypes.c_double
    lib.sci_ref_plain_step.argtypes = [ctypes.c_void_p]
    lib.sci_ref_plain_output.restype = ctypes.c_void_p
    lib.sci_ref_plain_output.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.sci_ref_plain_destroy.argtypes = [ctypes.c_void_p]
    lib.sci_ref_elements.argtypes = [ctypes.c_int, ctypes.c_uint32] + [ctypes.c_void_p] * 3 + [ctypes.c_uint64,
                                                                                            ctypes.c_void_p]
    _cache["ref"] = lib
    return lib


def on_host(chunk, mapping: dict) -> ChunkStruct:
    """A copy of `chunk` whose device input pointers are replaced by host arrays.

    `mapping` maps each device pointer to the numpy array holding the same values on the host;
    the oracle dereferences inputs on the CPU, so it must never see a device pointer."""
    copy = ChunkStruct.from_buffer_copy(bytes(chunk))
    for index in range(copy.arguments):
        host = mapping[chunk.inputs[index]]
        copy.inputs[index] = host.ctypes.data
    return copy


def execute(lib, chunk, count: int, dtype) -> np.ndarray:
    out = np.empty(count, dtype)
    fn = lib.sci_oracle_execute if hasattr(lib, "sci_oracle_execute") else lib.sci_ref_execute
    rc = fn(ctypes.byref(chunk), out.ctypes.data if count else None, count)
    assert rc == 0
    return out


def reduce(lib, chunk, fold: int, count: int) -> float:
    if hasattr(lib, "sci_oracle_reduce"):
        result = ctypes.c_double()
        assert lib.sci_oracle_reduce(ctypes.byref(chunk), fold, count, ctypes.byref(result)) == 0
        return result.value
    return lib.sci_ref_reduce(ctypes.byref(chunk), fold, count)


def bits(a: np.ndarray) -> np.ndarray:
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)


def mismatches(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Indices where two arrays differ in bits, counting any two NaNs as equal."""
    both_nan = np.isnan(a) & np.isnan(b)
    return np.nonzero((bits(a) != bits(b)) & ~both_nan)[0]


def ulp_distance(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Distance in units in the last place between two float arrays (NaN pairs count 0,
    a NaN against a number counts as a huge distance)."""
    def ordered(x):
        if x.dtype == np.float32:
            i = x.view(np.int32).astype(np.int64)
            return np.where(i < 0, -(i & 0x7FFFFFFF), i)
        i = x.view(np.int64)
        return np.where(i < 0, -(i & 0x7FFFFFFFFFFFFFFF), i)

    d = np.abs(ordered(a) - ordered(b))
    nan_a, nan_b = np.isnan(a), np.isnan(b)
    d[nan_a & nan_b] = 0
    d[nan_a ^ nan_b] = np.iinfo(np.int64).max
    return d

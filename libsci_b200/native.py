"""ctypes binding of libsci_cuda.so (include/sci_cuda.h).

The library is built in-tree by ``python -m libsci_b200.build`` (or ``__graft_entry__.build()``).
There is no fallback: if the shared library is missing or fails to load, importing this module
raises, so nothing can silently run on the CPU instead of the B200 kernels.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

from .chunk import ChunkStruct

LIBRARY = Path(__file__).resolve().parent / "libsci_cuda.so"

OK, INVALID, MEMORY, LAUNCH, UNSUPPORTED, DEVICE, TIMEOUT, COMPILE = range(8)
STATUS = {
    OK: "ok", INVALID: "invalid argument", MEMORY: "out of device memory", LAUNCH: "CUDA launch error",
    UNSUPPORTED: "unsupported", DEVICE: "no usable sm_100 device", TIMEOUT: "device wait timed out",
    COMPILE: "NVRTC compile failed",
}
MEMORY_DEVICE, MEMORY_MANAGED = 0, 1


class SciCudaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class SolveReport(ctypes.Structure):
    """sci_solve_report (include/sci_cuda.h)."""

    _fields_ = [("backward_error", ctypes.c_double), ("iterations", ctypes.c_int)]


class BatchItems(ctypes.Structure):
    """sci_batch_items (include/sci_cuda.h)."""

    _fields_ = [("items", ctypes.c_uint32), ("inputs", ctypes.c_void_p), ("outputs", ctypes.c_void_p),
                ("counts", ctypes.c_void_p), ("results", ctypes.c_void_p)]


class SolveItems(ctypes.Structure):
    """sci_solve_items (include/sci_cuda.h)."""

    _fields_ = [("systems", ctypes.c_uint32), ("orders", ctypes.c_void_p), ("matrices", ctypes.c_void_p),
                ("rights", ctypes.c_void_p), ("solutions", ctypes.c_void_p), ("errors", ctypes.c_void_p),
                ("iterations", ctypes.c_void_p)]


def _load() -> ctypes.CDLL:
    if not LIBRARY.exists():
        raise ImportError(f"{LIBRARY} is not built; run `python -m libsci_b200.build` (needs nvcc)")
    lib = ctypes.CDLL(str(LIBRARY))
    c_ctx = ctypes.c_void_p
    P = ctypes.POINTER
    sig = {
        "sci_cuda_open": (ctypes.c_int, [ctypes.c_uint32, P(c_ctx)]),
        "sci_cuda_close": (ctypes.c_int, [c_ctx]),
        "sci_cuda_name": (ctypes.c_char_p, [c_ctx]),
        "sci_cuda_synchronize": (ctypes.c_int, [c_ctx]),
        "sci_cuda_last_error": (ctypes.c_int, [c_ctx, ctypes.c_char_p, ctypes.c_size_t]),
        "sci_cuda_stream": (ctypes.c_void_p, [c_ctx]),
        "sci_cuda_allocate": (ctypes.c_int, [c_ctx, ctypes.c_uint64, ctypes.c_uint32, P(ctypes.c_void_p)]),
        "sci_cuda_dispose": (ctypes.c_int, [c_ctx, ctypes.c_void_p]),
        "sci_cuda_upload": (ctypes.c_int, [c_ctx, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]),
        "sci_cuda_download": (ctypes.c_int, [c_ctx, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]),
        "sci_cuda_execute": (ctypes.c_int, [c_ctx, P(ChunkStruct), ctypes.c_void_p, ctypes.c_uint64]),
        "sci_cuda_reduce": (ctypes.c_int, [c_ctx, P(ChunkStruct), ctypes.c_uint32, ctypes.c_uint64, P(ctypes.c_double)]),
        "sci_cuda_reduce_async": (ctypes.c_int, [c_ctx, P(ChunkStruct), ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p]),
        "sci_cuda_jit_wait": (ctypes.c_int, [c_ctx]),
        "sci_cuda_product": (ctypes.c_int, [c_ctx, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
    }
    sig["sci_cuda_gradient"] = (ctypes.c_int, [c_ctx, P(ChunkStruct), ctypes.c_uint64, ctypes.c_double,
                                               P(ctypes.c_void_p), P(ctypes.c_double), ctypes.c_uint32])
    sig["sci_cuda_product_gradient"] = (ctypes.c_int, [c_ctx, ctypes.c_uint32, ctypes.c_uint32] + [ctypes.c_void_p] * 5 +
                                        [ctypes.c_uint64] * 3)
    sig["sci_cuda_solve_gradient"] = (ctypes.c_int, [c_ctx, ctypes.c_uint32, ctypes.c_uint32] + [ctypes.c_void_p] * 6 +
                                      [ctypes.c_uint64, ctypes.c_uint64, P(SolveReport)])
    sig["sci_cuda_batch_create"] = (ctypes.c_int, [c_ctx, P(ChunkStruct), ctypes.c_uint32, P(BatchItems),
                                                   P(ctypes.c_void_p)])
    sig["sci_cuda_batch_launch"] = (ctypes.c_int, [ctypes.c_void_p])
    sig["sci_cuda_batch_spans"] = (ctypes.c_int, [ctypes.c_void_p, P(ctypes.c_uint32), P(ctypes.c_int32)])
    sig["sci_cuda_batch_destroy"] = (ctypes.c_int, [ctypes.c_void_p])
    sig["sci_cuda_solve_batch_create"] = (ctypes.c_int, [c_ctx, P(SolveItems), P(ctypes.c_void_p)])
    sig["sci_cuda_solve_batch_launch"] = (ctypes.c_int, [ctypes.c_void_p])
    sig["sci_cuda_solve_batch_shapes"] = (ctypes.c_int, [ctypes.c_void_p, P(ctypes.c_uint32)])
    sig["sci_cuda_solve_batch_destroy"] = (ctypes.c_int, [ctypes.c_void_p])
    U64, F64, U32, VP = ctypes.c_uint64, ctypes.c_double, ctypes.c_uint32, ctypes.c_void_p
    sig["sci_cuda_fill"] = (ctypes.c_int, [c_ctx, U32, VP, U64, F64])
    sig["sci_cuda_linspace"] = (ctypes.c_int, [c_ctx, U32, VP, U64, F64, F64])
    sig["sci_cuda_range_count"] = (U64, [U32, F64, F64, F64])
    sig["sci_cuda_range"] = (ctypes.c_int, [c_ctx, U32, VP, U64, F64, F64])
    sig["sci_cuda_eye"] = (ctypes.c_int, [c_ctx, U32, VP, U64, U64])
    sig["sci_cuda_grid"] = (ctypes.c_int, [c_ctx, U32, VP, U64, VP, U64, VP, VP])
    sig["sci_cuda_decompose"] = (ctypes.c_int, [c_ctx, U32, U32, VP, VP, VP, VP, U64])
    sig["sci_cuda_transpose"] = (ctypes.c_int, [c_ctx, U32, VP, U32, P(U64), VP])
    sig["sci_cuda_upload_lane"] = (ctypes.c_int, [c_ctx, VP, VP, U64])
    sig["sci_cuda_download_lane"] = (ctypes.c_int, [c_ctx, VP, VP, U64])
    sig["sci_cuda_join"] = (ctypes.c_int, [c_ctx])
    sig["sci_cuda_broadcast"] = (ctypes.c_int, [c_ctx, U32, U32, U32, P(U64), U32, P(VP), P(U64), VP])
    sig["sci_cuda_reduce_axis"] = (ctypes.c_int, [c_ctx, U32, U32, VP, U32, P(U64), U32, VP])
    sig["sci_cuda_element_size"] = (U64, [U32])
    sig["sci_cuda_execute_elements"] = (ctypes.c_int, [c_ctx, U32, P(ChunkStruct), VP, U64])
    sig["sci_cuda_reduce_elements"] = (ctypes.c_int, [c_ctx, U32, P(ChunkStruct), U32, U64, VP])
    optional = {}
    sig["sci_cuda_factor"] = (ctypes.c_int, [c_ctx, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_uint64])
    sig["sci_cuda_solve"] = (ctypes.c_int, [c_ctx, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, P(SolveReport)])
    for name, (res, args) in list(sig.items()):
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    for name, (res, args) in optional.items():
        if hasattr(lib, name):
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
    return lib


lib = _load()


def check(status: int, context=None) -> None:
    if status == OK:
        return
    message = ""
    if context:
        buffer = ctypes.create_string_buffer(512)
        lib.sci_cuda_last_error(context, buffer, 512)
        message = buffer.value.decode(errors="replace")
    raise SciCudaError(status, message)

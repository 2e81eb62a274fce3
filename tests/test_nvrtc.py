"""The specialised chunk kernels compile under NVRTC for sm_100a (no GPU needed).

libsci_cuda.so bakes a repeated chunk into the kernel source with NVRTC at run time
(csrc/specialize.cu, program_of), and falls back to the interpreter when that compile fails, so a
source change that NVRTC rejects would only show up as a slower run. This test builds the same
program text for representative chunks (the stored chunk of the large fused workload, its
reductions, a batch and a gradient), compiles it with NVRTC and the library's options, and checks
that it succeeds. NVRTC is a host library: it runs without a GPU.
"""
import ctypes
import ctypes.util
from pathlib import Path

import numpy as np
import pytest

from libsci_b200 import chunk as C

CSRC = Path(__file__).resolve().parent.parent / "libsci_b200" / "csrc"
HEADERS = ["sci_math.cuh", "chunk_kernel.cuh", "gradient_kernel.cuh", "batch_kernel.cuh"]
OPTIONS = [b"-default-device", b"-arch=sm_100a", b"-std=c++17", b"-lineinfo", b"--extra-device-vectorization",
           b"--fmad=false"]
K_DOT, K_GRAD = 2, 8  # chunk_kernel.cuh's kDot, gradient_kernel.cuh's kGradRecompute


def nvrtc():
    for name in ("/usr/local/cuda/lib64/libnvrtc.so.12", ctypes.util.find_library("nvrtc")):
        if name:
            try:
                return ctypes.CDLL(name)
            except OSError:
                continue
    pytest.skip("libnvrtc is not available")


def program(chunk, mode, kind="chunk"):
    """The text csrc/specialize.cu's program_of writes for a chunk (same structure)."""
    contract = mode == K_DOT
    length = chunk.length - 1 if contract else chunk.length
    left = right = 0xFF
    if contract:
        left = chunk.instructions[chunk.length - 1].sources[0]
        right = chunk.instructions[chunk.length - 1].sources[1]
    header = {"chunk": "chunk_kernel.cuh", "batch": "batch_kernel.cuh", "gradient": "gradient_kernel.cuh"}[kind]
    steps = ", ".join("{%d, %d, %d, %d, %d}" % (ins.code, ins.target, *ins.sources)
                      for ins in list(chunk.instructions)[:length]) or "{0, 255, 255, 255, 255}"
    source = (f'#include "{header}"\nstruct SciBaked {{\n'
              f"  static constexpr int length = {length}, arguments = {chunk.arguments}, "
              f"temporaries = {chunk.temporaries}, result = {chunk.result}, dot_left = {left}, dot_right = {right};\n"
              f"  static constexpr sci_cuda::Step steps[] = {{{steps}}};\n}};\n")
    element = "double" if chunk.precision == C.WIDE else "float"
    if kind == "batch":
        name = f"&sci_cuda::batch_stream<{element}, sci_cuda::Baked<SciBaked>>"
    else:
        stream = "gradient_stream" if kind == "gradient" else "chunk_stream"
        name = f"&sci_cuda::{stream}<{element}, sci_cuda::Baked<SciBaked>, {mode}>"
    return source, name


def compile_source(lib, source, name):
    headers = (ctypes.c_char_p * len(HEADERS))(*[(CSRC / h).read_bytes() for h in HEADERS])
    names = (ctypes.c_char_p * len(HEADERS))(*[h.encode() for h in HEADERS])
    prog = ctypes.c_void_p()
    assert lib.nvrtcCreateProgram(ctypes.byref(prog), source.encode(), b"sci_specialized.cu", len(HEADERS), headers,
                                  names) == 0
    assert lib.nvrtcAddNameExpression(prog, name.encode()) == 0
    options = (ctypes.c_char_p * len(OPTIONS))(*OPTIONS)
    status = lib.nvrtcCompileProgram(prog, len(OPTIONS), options)
    size = ctypes.c_size_t()
    lib.nvrtcGetProgramLogSize(prog, ctypes.byref(size))
    log = ctypes.create_string_buffer(size.value + 1)
    lib.nvrtcGetProgramLog(prog, log)
    lib.nvrtcDestroyProgram(ctypes.byref(prog))
    return status, log.value.decode(errors="replace")


def references():
    return [C.Reference(0x1000 * (i + 1), 1 << 20, np.float32) for i in range(3)]


def cases():
    x, y, z = (r for r in references())
    stored = C.record_output(C.unary("root", C.unary("absolute", x)) * C.unary("logarithm", y) + C.unary("tanh", z))
    yield "stored", stored, 0, "chunk"
    yield "mean", C.record_reduce(C.unary("exponential", -x * x)), 1, "chunk"
    yield "peak", C.record_reduce(C.unary("sin", x) * C.unary("cos", z)), 1, "chunk"
    yield "dot", C.record_reduce(x * z), K_DOT, "chunk"
    yield "tanh_sum", C.record_reduce(C.unary("tanh", x * y + z)), 1, "batch"
    yield "gradient", C.record_reduce(C.unary("exponential", -x * x) * C.unary("sin", y)
                                      + C.unary("logarithm", 1 + z * z)), K_GRAD, "gradient"


@pytest.mark.parametrize("label,chunk,mode,kind", list(cases()), ids=[c[0] for c in cases()])
def test_specialised_source_compiles(label, chunk, mode, kind):
    lib = nvrtc()
    source, name = program(chunk, mode, kind)
    status, log = compile_source(lib, source, name)
    assert status == 0, f"{label}: NVRTC status {status}\n{log}"


def test_a_broken_source_is_reported():
    lib = nvrtc()
    source, name = program(next(cases())[1], 0)
    status, log = compile_source(lib, source + "\nthis is not C++;\n", name)
    assert status != 0 and "error" in log

"""sci_cuda_reduce_noalloc: the chunk reduction that allocates no device memory.

It serves callers that may not create device memory themselves (a framework that owns the GPU heap
through its own pool, a plugin inside one, a latency-critical thread where an allocation would
synchronize the device). Its scratch is a fixed array compiled into libsci_cuda.so, shared by
every call on a device. These tests call it through the C ABI, twice in a row on the same data,
and hold it to the same bar as sci_cuda_reduce, the entry point that allocates its scratch per
context: minimum and maximum identical, sums within 1e-9 relative. The file is named to be
collected last, so a run that stops at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

from libsci_b200 import chunk as C

pytestmark = pytest.mark.gpu


def bind():
    from libsci_b200.native import lib

    fn = lib.sci_cuda_reduce_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(C.ChunkStruct), ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_uint32, ctypes.c_char_p, ctypes.c_size_t]
    return fn


def test_no_alloc_reduction_matches_the_allocating_one(device):
    fn = bind()
    rng = np.random.default_rng(42)
    n = (1 << 21) + 11
    x = rng.standard_normal(n).astype(np.float32)
    z = rng.uniform(-1, 1, n).astype(np.float32)
    dx, dz = device.array(x), device.array(z)
    result = device.empty(1, np.float64)
    a, c = dx.expression(), dz.expression()
    cases = [
        (C.record_reduce(C.unary("exponential", -a * a)), C.SUM),   # mean(exp(-x*x)) numerator
        (C.record_reduce(C.unary("sin", a) * C.unary("cos", c)), C.MAXIMUM),
        (C.record_reduce(C.unary("sin", a) * C.unary("cos", c)), C.MINIMUM),
        (C.record_reduce(a * c), C.SUM),                             # contracted dot
    ]
    message = ctypes.create_string_buffer(256)
    for chunk, fold in cases:
        want = device.reduce_chunk(chunk, fold, n)
        for _ in range(2):  # two calls in a row share (and reuse) the fixed scratch
            status = fn(ctypes.byref(chunk), fold, n, result.pointer, device.stream, 0, message, 256)
            assert status == 0, message.value
            device.synchronize()
            got = float(result.numpy()[0])
            if fold == C.SUM:
                assert abs(got - want) <= 1e-9 * max(1.0, abs(want))
            else:
                assert got == want


def test_no_alloc_reduction_limits(device):
    fn = bind()
    x = device.array(np.arange(1000, dtype=np.float32))
    result = device.empty(1, np.float64)
    chunk = C.record_reduce(x.expression())
    message = ctypes.create_string_buffer(256)
    assert fn(ctypes.byref(chunk), C.SUM, 1000, result.pointer, device.stream, 4097, message, 256) != 0
    assert b"4096" in message.value
    # an explicit launch width within the limit, then the empty cases
    assert fn(ctypes.byref(chunk), C.MAXIMUM, 1000, result.pointer, device.stream, 3, message, 256) == 0
    device.synchronize()
    assert float(result.numpy()[0]) == 999.0
    assert fn(ctypes.byref(chunk), C.SUM, 0, result.pointer, device.stream, 0, message, 256) == 0
    device.synchronize()
    assert float(result.numpy()[0]) == 0.0
    assert fn(ctypes.byref(chunk), C.MINIMUM, 0, result.pointer, device.stream, 0, message, 256) == 0
    device.synchronize()
    assert np.isnan(result.numpy()[0])


FRESH_PROCESS = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from libsci_b200 import chunk as C
from libsci_b200.device import Device
from libsci_b200.native import lib

fn = lib.sci_cuda_reduce_noalloc
fn.restype = ctypes.c_int
fn.argtypes = [ctypes.POINTER(C.ChunkStruct), ctypes.c_uint32, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
               ctypes.c_uint32, ctypes.c_char_p, ctypes.c_size_t]
device = Device(0)
n = (1 << 22) + 5
x = device.array(np.random.default_rng(3).uniform(2.0, 3.0, n).astype(np.float32))
result = device.empty(1, np.float64)
a = x.expression()
# one input and two temporaries, arithmetic only: 16 KiB of temporaries and four 8 KiB ring stages
# at 256 threads, exactly 48 KiB of dynamic shared memory, which needs the kernel's opt-in
chunk = C.record_reduce((a - 1.0) / (a + 1.0))
assert chunk.arguments == 1 and chunk.temporaries == 2
message = ctypes.create_string_buffer(256)
got = []
for _ in range(2):
    status = fn(ctypes.byref(chunk), C.SUM, n, result.pointer, device.stream, 0, message, 256)
    assert status == 0, message.value
    device.synchronize()
    got.append(float(result.numpy()[0]))
want = device.reduce_chunk(chunk, C.SUM, n)
assert all(abs(g - want) <= 1e-9 * abs(want) for g in got), (got, want)
print("fresh", got[0], want)
"""


def test_no_alloc_first_call_in_a_fresh_process():
    """The first call of a process, with no earlier launch that could have raised the kernel's
    shared-memory limit, on a chunk that needs exactly 48 KiB of dynamic shared memory."""
    import subprocess
    import sys
    from pathlib import Path

    root = str(Path(__file__).resolve().parent.parent)
    run = subprocess.run([sys.executable, "-c", FRESH_PROCESS, root], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "fresh" in run.stdout

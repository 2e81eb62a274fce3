"""The fast forms of exp, log, the sin/cos family and float tanh (sci_math.cuh) against the full
forms they shortcut: every one of the 2^32 float inputs and 2^31 sampled doubles must give the same
bits. The full forms are the ones the oracle parity tests pin (test_chunk_gpu.py).

Two routes: a compiled checker calling both forms side by side, and the library itself, where the
specialised (NVRTC) kernels run the fast forms and the interpreter (specialisation off) the full
forms, over every float bit pattern."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SOURCE = os.path.join(ROOT, "tests", "fast_forms_check.cu")
BINARY = os.path.join(ROOT, "tests", "_build", "fast_forms_check")
HEADERS = [os.path.join(ROOT, "libsci_b200", "csrc", name) for name in ("sci_math.cuh", "chunk_kernel.cuh")]


def build_checker() -> str:
    """Compiles the checker for sm_100a when it is missing or older than its sources."""
    newest = max(os.path.getmtime(p) for p in [SOURCE, *HEADERS])
    if not os.path.exists(BINARY) or os.path.getmtime(BINARY) < newest:
        os.makedirs(os.path.dirname(BINARY), exist_ok=True)
        # contraction off, as the specialised kernels are compiled (specialize.cu)
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-fmad=false",
                        "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "libsci_b200", "csrc"),
                        "-o", BINARY, SOURCE], check=True)
    return BINARY


@pytest.mark.gpu
def test_fast_forms_match_full_forms():
    run = subprocess.run([build_checker()], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stdout + run.stderr
    lines = [line.split() for line in run.stdout.splitlines() if line.strip()]
    assert len(lines) == 20, run.stdout
    for name, precision, checked, bad, first in lines:
        assert int(checked) == (1 << 32 if precision == "float" else 1 << 31)
        assert int(bad) == 0, f"{name} ({precision}): {bad} inputs differ, first {first}"


FAST_CODES = ["exponential", "logarithm", "sin", "cos", "tan", "csc", "sec", "cot", "tanh", "coth"]


def open_device(jit: str):
    from libsci_b200.device import Device

    saved = os.environ.get("SCI_CUDA_JIT")
    os.environ["SCI_CUDA_JIT"] = jit
    try:
        return Device(0)
    finally:
        if saved is None:
            del os.environ["SCI_CUDA_JIT"]
        else:
            os.environ["SCI_CUDA_JIT"] = saved


@pytest.mark.gpu
def test_specialised_kernels_match_the_interpreter_on_every_float():
    import torch

    from libsci_b200 import chunk as C

    interpreter, specialised = open_device("0"), open_device("sync")
    span = 1 << 28
    try:
        patterns = torch.empty(span, dtype=torch.int32, device="cuda")
        first, second = torch.empty_like(patterns), torch.empty_like(patterns)
        for code in FAST_CODES:
            chunk = C.record_output(C.unary(code, C.Reference(patterns.data_ptr(), span, np.float32)))
            for start in range(0, 1 << 32, span):
                # the bit patterns start .. start + span - 1 as int32: shift into the int32 range,
                # then flip the top bit back
                shifted = torch.arange(start - (1 << 31), start - (1 << 31) + span, dtype=torch.int64, device="cuda")
                patterns.copy_(shifted.to(torch.int32) ^ (-(1 << 31)))
                torch.cuda.synchronize()
                interpreter.execute(chunk, first.data_ptr(), span)
                specialised.execute(chunk, second.data_ptr(), span)
                interpreter.synchronize()
                specialised.synchronize()
                differ = int((first != second).sum())
                assert differ == 0, f"{code}: {differ} of the patterns {start:#x}.. differ"
    finally:
        interpreter.close()
        specialised.close()


COMPOSITES = {
    "exp(x) + y": lambda x, y, z: C_unary("exponential", x) + y,
    "log(y) * x + z": lambda x, y, z: C_unary("logarithm", y) * x + z,
    "sin(x) * cos(z) + y": lambda x, y, z: C_unary("sin", x) * C_unary("cos", z) + y,
    "sqrt|x| * log(y) + tanh(z)": lambda x, y, z: C_unary("root", C_unary("absolute", x)) * C_unary("logarithm", y)
    + C_unary("tanh", z),
    "exp(-x * x) * y - z": lambda x, y, z: C_unary("exponential", -x * x) * y - z,
    "tan(x) - cot(z) * y": lambda x, y, z: C_unary("tan", x) - C_unary("cot", z) * y,
    "coth(z) / sec(x)": lambda x, y, z: C_unary("coth", z) / C_unary("sec", x),
}


def C_unary(code, item):
    from libsci_b200 import chunk as C

    return C.unary(code, item)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(COMPOSITES))
def test_composite_chunks_match_the_interpreter(name):
    """Fast forms inside longer chunks: packed or fused arithmetic must not leak across codes."""
    import torch

    from libsci_b200 import chunk as C

    count = 1 << 26
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randn(count, device="cuda", generator=g) * 3
    x[: count // 4] = (torch.rand(count // 4, device="cuda", generator=g) - 0.5) * 200
    y = torch.rand(count, device="cuda", generator=g) * 9.9 + 0.1
    z = torch.rand(count, device="cuda", generator=g) * 2 - 1
    specials = torch.tensor([0.0, -0.0, float("inf"), -float("inf"), float("nan"), 1e-45, -1e-45, 1e-38, 88.7,
                             -103.9, 2e6, -3e7, 1e30, 1.5707964, 0.5, -1.0], device="cuda")
    for t in (x, y, z):
        t[1000:1000 + len(specials)] = specials
        t[5000:5000 + len(specials)] = specials.flip(0)
    y[::997] = -y[::997]
    interpreter, specialised = open_device("0"), open_device("sync")
    try:
        refs = [C.Reference(t.data_ptr(), count, np.float32) for t in (x, y, z)]
        expression = COMPOSITES[name](*refs)
        first, second = torch.empty_like(x), torch.empty_like(x)
        chunk = C.record_output(expression)
        torch.cuda.synchronize()
        interpreter.execute(chunk, first.data_ptr(), count)
        specialised.execute(chunk, second.data_ptr(), count)
        interpreter.synchronize()
        specialised.synchronize()
        differ = int((first.view(torch.int32) != second.view(torch.int32)).sum())
        assert differ == 0, f"{name}: {differ} elements differ"
        for fold in (C.MINIMUM, C.MAXIMUM):
            reduced = C.record_reduce(expression)
            a, b = interpreter.reduce_chunk(reduced, fold, count), specialised.reduce_chunk(reduced, fold, count)
            assert (np.isnan(a) and np.isnan(b)) or a == b, (name, fold, a, b)
    finally:
        interpreter.close()
        specialised.close()


REACH = 1048576.0  # 2^20: the circular functions' own reduction reaches this far
CIRCULAR = {"sin": 2, "cos": 2, "tan": 4, "csc": 4, "sec": 4, "cot": 4}  # ulp allowed beyond REACH


@pytest.mark.gpu
def test_exact_codes_match_the_oracle_across_the_float_range(oracle):
    """The exact codes (every code but the C-library functions) through the interpreter and through
    the specialised kernels, against the oracle (itself pinned to libsci's CPU path over the same
    inputs in test_oracle.py): every 257th float bit pattern and 2^22 hashed doubles, bit for bit,
    except the circular functions beyond |x| = 2^20, which both sides take from a double-precision
    library and which stay within 2 ulp (4 for the quotients)."""
    from libsci_b200 import chunk as C
    from tests import _oracle
    from tests.test_oracle import EXACT_UNARY, hashed_doubles, spread_floats

    devices = [open_device("0"), open_device("sync")]
    try:
        for x in (spread_floats(), hashed_doubles(1 << 22)):
            n = x.size
            expected = {}
            for device in devices:
                dx = device.array(x)
                out = device.empty(n, x.dtype)
                for code in EXACT_UNARY:
                    chunk = C.record_output(C.Node(code, [dx.expression()]))
                    if code not in expected:
                        expected[code] = _oracle.execute(oracle, _oracle.on_host(chunk, {dx.pointer: x}), n, x.dtype)
                    device.execute(chunk, out.pointer, n)
                    device.synchronize()
                    got = out.numpy()
                    near = ~(np.abs(x) > REACH) if code in CIRCULAR else np.ones(n, bool)
                    bad = _oracle.mismatches(got[near], expected[code][near])
                    assert bad.size == 0, f"{code} ({x.dtype}): {bad.size} differ, first input {x[near][bad[0]]!r}"
                    if code in CIRCULAR:
                        # beyond the reduction's reach both sides round a double-precision library
                        # result, CUDA's here and glibc's in the reference
                        far = ~near
                        worst = int(_oracle.ulp_distance(got[far], expected[code][far]).max(initial=0))
                        assert worst <= CIRCULAR[code], f"{code} ({x.dtype}) beyond 2^20: {worst} ulp"
                dx.free()
                out.free()
    finally:
        for device in devices:
            device.close()

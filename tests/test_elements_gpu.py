"""Integer-element chunks on the device (sci_cuda_execute_elements / sci_cuda_reduce_elements)
against the oracle, which test_elements.py pins to the reference's own host loop.

Bit for bit: the arithmetic codes, all eight integer types, aligned (128-bit) and unaligned
(element-wise) operands, ragged counts, the 128-thread path a chunk with many temporaries takes,
wrapping sums over 2^26 elements, and the cases C++ leaves undefined, with the definitions the
backend documents (wrap, zero divisor -> 0, MIN / -1 -> MIN, NaN -> 0, saturation). The 27 real
functions go through the GPU's double functions and the oracle's glibc ones: the integer results
agree except where the double value lies within a few ulps of an integer boundary.
"""
import ctypes

import numpy as np
import pytest

from libsci_b200 import chunk as C
from libsci_b200.native import lib
from tests import _oracle
from tests.test_elements import EVALUATIONS, INTEGERS, REDUCTIONS, named, operands, oracle_elements

pytestmark = pytest.mark.gpu


def on_device(device, arrays):
    return [device.array(a) for a in arrays]


def device_elements(device, which, arrays):
    x, y, z = (a.expression() for a in arrays)
    expression = named(which, x, y, z)
    if which in REDUCTIONS:
        return np.array([device.reduce(expression, REDUCTIONS[which])], arrays[0].dtype)
    return device.evaluate(expression).numpy()


@pytest.mark.parametrize("dtype", INTEGERS)
@pytest.mark.parametrize("count", [1, 4099, (1 << 20) + 3])
def test_named_expressions_match_oracle(device, oracle, dtype, count):
    host = operands(dtype, count, seed=count)
    arrays = on_device(device, host)
    for which in EVALUATIONS + list(REDUCTIONS):
        got = device_elements(device, which, arrays)
        want = oracle_elements(oracle, which, host, dtype)
        bad = np.flatnonzero(got != want)
        assert bad.size == 0, (np.dtype(dtype).name, count, which, bad[:5], got[bad[:5]], want[bad[:5]])


@pytest.mark.parametrize("dtype", [np.int8, np.int32, np.uint64])
def test_unaligned_operands_take_the_element_path(device, oracle, dtype):
    count = 10007
    host = operands(dtype, count + 3, seed=3)
    arrays = on_device(device, host)
    shifted = [a.offset(1, count) for a in arrays]  # 1 element past a 256-byte boundary
    shifted_host = [h[1:count + 1].copy() for h in host]
    for which in (0, 3, 10, 12):
        got = device_elements(device, which, shifted)
        want = oracle_elements(oracle, which, shifted_host, dtype)
        assert np.array_equal(got, want), (np.dtype(dtype).name, which)


def test_undefined_cases_follow_the_documented_definitions(device, oracle):
    for dtype in (np.int8, np.int32, np.int64, np.uint16):
        info = np.iinfo(dtype)
        edge = np.array([info.min, info.max, 0, 1, -1 if info.min < 0 else 2, info.min, 7, info.max], dtype)
        divisor = np.array([-1 if info.min < 0 else 1, 0, 0, 0, 1, 2, -1 if info.min < 0 else 3, info.max], dtype)
        x, y = device.array(edge), device.array(divisor)
        for expression in (
                x.expression() / y.expression(),                      # zero divisor, MIN / -1
                x.expression() * y.expression() + x.expression(),     # signed overflow wraps
                -x.expression(),
                C.unary("absolute", x.expression()),
                C.unary("root", x.expression() - 3),                  # sqrt of a negative: NaN -> 0
                C.unary("exponential", x.expression()),               # overflow saturates
                C.unary("logarithm", x.expression()),                 # log(0) = -inf saturates
        ):
            chunk = C.record_output(expression)
            got = device.evaluate(expression).numpy()
            mapping = {x.pointer: edge, y.pointer: divisor}
            host_chunk = _oracle.on_host(chunk, mapping)
            want = np.empty(edge.size, dtype)
            assert oracle.sci_oracle_execute_elements(C.ELEMENT[np.dtype(dtype)], ctypes.byref(host_chunk),
                                                      want.ctypes.data, edge.size) == 0
            assert np.array_equal(got, want), (np.dtype(dtype).name, chunk.listing(), got, want)


REAL = ["root", "exponential", "logarithm", "sin", "cos", "tan", "asin", "acos", "atan", "csc", "sec", "cot",
        "acsc", "asec", "acot", "sinh", "cosh", "tanh", "asinh", "acosh", "atanh", "csch", "sech", "coth",
        "acsch", "asech", "acoth"]
NUMPY = {
    "root": np.sqrt, "exponential": np.exp, "logarithm": np.log, "sin": np.sin, "cos": np.cos, "tan": np.tan,
    "asin": np.arcsin, "acos": np.arccos, "atan": np.arctan, "csc": lambda v: 1 / np.sin(v),
    "sec": lambda v: 1 / np.cos(v), "cot": lambda v: 1 / np.tan(v), "acsc": lambda v: np.arcsin(1 / v),
    "asec": lambda v: np.arccos(1 / v), "acot": lambda v: np.arctan(1 / v), "sinh": np.sinh, "cosh": np.cosh,
    "tanh": np.tanh, "asinh": np.arcsinh, "acosh": np.arccosh, "atanh": np.arctanh,
    "csch": lambda v: 1 / np.sinh(v), "sech": lambda v: 1 / np.cosh(v), "coth": lambda v: 1 / np.tanh(v),
    "acsch": lambda v: np.arcsinh(1 / v), "asech": lambda v: np.arccosh(1 / v), "acoth": lambda v: np.arctanh(1 / v),
}


@pytest.mark.parametrize("dtype", [np.int16, np.int64])
def test_real_functions_every_int16_and_sampled_int64(device, oracle, dtype):
    if dtype == np.int16:
        values = np.arange(-32768, 32768, dtype=np.int16)
    else:
        rng = np.random.default_rng(5)
        values = np.concatenate([rng.integers(-(1 << 40), 1 << 40, 1 << 16), np.arange(-300, 300)]).astype(np.int64)
    x = device.array(values)
    info = np.iinfo(dtype)
    with np.errstate(all="ignore"):
        for name in REAL:
            expression = C.unary(name, x.expression())
            got = device.evaluate(expression).numpy()
            host_chunk = _oracle.on_host(C.record_output(expression), {x.pointer: values})
            want = np.empty(values.size, dtype)
            assert oracle.sci_oracle_execute_elements(C.ELEMENT[np.dtype(dtype)], ctypes.byref(host_chunk),
                                                      want.ctypes.data, values.size) == 0
            bad = np.flatnonzero(got != want)
            if bad.size:
                # a GPU double and a glibc double may differ by an ulp or two; after truncation that
                # shows only where the value sits that close to an integer (or to the saturation
                # bound) -- anything else is a real mismatch
                exact = NUMPY[name](values[bad].astype(np.float64))
                near = np.abs(exact - np.round(exact)) <= 4 * np.spacing(np.abs(exact))
                near |= np.abs(exact) >= float(info.max) * (1 - 1e-15)
                apart = np.abs(got[bad].astype(np.float64) - want[bad].astype(np.float64))
                assert near.all() and np.all(apart <= 4 * np.spacing(np.abs(exact)) + 1), \
                    (name, values[bad][~near][:5], got[bad][~near][:5], want[bad][~near][:5])


def test_many_temporaries_take_the_narrow_block(device, oracle):
    # (x*y) + ((x*y) + (... + z)): every level holds its product in a temporary while the right side
    # records, so the chunk needs 20 temporaries (> 48 KB of slot file at 256 threads)
    dtype = np.int16
    host = operands(dtype, 70001, seed=11)
    arrays = on_device(device, host)
    x, y, z = (a.expression() for a in arrays)
    expression = z
    for _ in range(20):
        expression = C.binary("add", C.binary("multiply", x, y), expression)
    chunk = C.record_output(expression)
    assert chunk.valid() and chunk.temporaries >= 13, chunk.temporaries
    got = device.evaluate(expression).numpy()
    mapping = {a.pointer: h for a, h in zip(arrays, host)}
    want = np.empty(host[0].size, dtype)
    assert oracle.sci_oracle_execute_elements(C.ELEMENT[np.dtype(dtype)], ctypes.byref(_oracle.on_host(chunk, mapping)),
                                              want.ctypes.data, want.size) == 0
    assert np.array_equal(got, want)


def test_wrapping_reductions_at_size(device):
    # size-independent check at 2^26 int32: the wrapped sum equals numpy's int64 sum taken mod 2^32;
    # minimum and maximum are exact; an empty reduction is element{} = 0
    count = 1 << 26
    rng = np.random.default_rng(13)
    a = rng.integers(-(1 << 31), (1 << 31) - 1, count, dtype=np.int32)
    b = rng.integers(-(1 << 31), (1 << 31) - 1, count, dtype=np.int32)
    x, y = device.array(a), device.array(b)
    product = (a.astype(np.int64) * b.astype(np.int64)).astype(np.int32)  # wraps per element
    total = np.int64(product.astype(np.int64).sum()).astype(np.int32)      # wraps once more
    assert device.reduce(x.expression() * y.expression(), C.SUM) == total
    assert device.reduce(x.expression() - y.expression(), C.MINIMUM) == (a - b).min()
    assert device.reduce(x.expression() - y.expression(), C.MAXIMUM) == (a - b).max()
    empty = device.empty(0, np.int32)
    assert device.reduce(empty.expression() * 2, C.MINIMUM) == 0


def test_float_elements_forward_to_the_native_path(device):
    values = np.linspace(-3, 3, 1001, dtype=np.float32)
    x = device.array(values)
    chunk = C.record_output(C.unary("tanh", x.expression()) * 2)
    native = device.empty(values.size, np.float32)
    device.execute(chunk, native.pointer, values.size)
    forwarded = device.empty(values.size, np.float32)
    device.execute_elements(np.float32, chunk, forwarded.pointer, values.size)
    assert np.array_equal(native.numpy().view(np.uint32), forwarded.numpy().view(np.uint32))
    assert lib.sci_cuda_element_size(C.ELEMENT[np.dtype(np.uint16)]) == 2

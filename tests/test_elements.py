"""Integer-element expressions: the oracle's restatement against the reference's own host loop.

libsci evaluates expressions over non-native element types (anything but float and double)
element by element with array::calculate (include/array/calculate.hpp:17-93) inside assign() and
reduce() (include/array/expression.hpp:178-184,203-220). oracle/_ref's sci_ref_elements runs
named expressions through exactly that code for the eight integer types; here the same
expressions, recorded into bytecode by libsci_b200.chunk, run through the oracle's restatement
(sci_oracle_execute_elements / reduce_elements) and must agree bit for bit. Inputs stay inside
the ranges where C++ defines every step (no signed overflow, no zero divisor, no NaN or
out-of-range real result), since outside them the reference has no defined answer.
"""
import ctypes

import numpy as np
import pytest

from libsci_b200 import chunk as C

INTEGERS = [np.int8, np.int16, np.int32, np.int64, np.uint8, np.uint16, np.uint32, np.uint64]
EVALUATIONS = [0, 1, 2, 3, 4, 5, 6]
REDUCTIONS = {10: C.SUM, 11: C.MINIMUM, 12: C.MAXIMUM}


def defined_range(dtype):
    """Operand bounds under which every named expression stays defined in C++ (products and
    sums of int32 / int64 do not overflow; uint16 products stay below INT_MAX after promotion;
    |x| + 1 and -x stay representable)."""
    info = np.iinfo(dtype)
    if dtype == np.int32:
        return -(1 << 12), 1 << 12
    if dtype == np.int64:
        return -(1 << 20), 1 << 20
    if dtype == np.uint16:
        return 0, (1 << 15) - 1
    return int(info.min) + 1, int(info.max) - 1


def operands(dtype, count, seed=7):
    rng = np.random.default_rng(seed)
    lo, hi = defined_range(dtype)
    x, y, z = (rng.integers(lo, hi, count, dtype=dtype, endpoint=True) for _ in range(3))
    y[y == 0] = 1  # the divisor of expression 3
    return x, y, z


def named(which, x, y, z):
    """The expressions of sci_ref_elements, in the same order, over any three operands."""
    u, b = C.unary, C.binary
    if which == 0:
        return x * y + z
    if which == 1:
        return -x + y * 3
    if which == 2:
        return u("absolute", x) - b("minimum", y, z)
    if which == 3:
        return b("maximum", x, z) / y
    if which == 4:
        return u("root", u("absolute", x)) + y
    if which == 5:
        return u("atan", x) * y + u("cos", z)
    if which == 6:
        return u("logarithm", u("absolute", x) + 1) * 2 - u("tanh", y)
    if which == 10:
        return x * y
    if which == 11:
        return x - z
    if which == 12:
        return u("absolute", y) + x
    raise ValueError(which)


def leaves(arrays, dtype):
    return [C.Reference(a.ctypes.data, a.size, dtype) for a in arrays]


def oracle_elements(oracle, which, arrays, dtype):
    """The oracle's value of named expression `which` over host arrays."""
    dtype = np.dtype(dtype)
    count = arrays[0].size
    expression = named(which, *leaves(arrays, dtype))
    element = C.ELEMENT[dtype]
    if which in REDUCTIONS:
        chunk = C.record_reduce(expression)
        out = np.zeros(1, dtype)
        assert oracle.sci_oracle_reduce_elements(element, ctypes.byref(chunk), REDUCTIONS[which], count,
                                                 out.ctypes.data) == 0
        return out
    chunk = C.record_output(expression)
    out = np.empty(count, dtype)
    assert oracle.sci_oracle_execute_elements(element, ctypes.byref(chunk), out.ctypes.data, count) == 0
    return out


def reference_elements(reference, which, arrays, dtype):
    dtype = np.dtype(dtype)
    count = arrays[0].size
    out = np.zeros(1 if which in REDUCTIONS or which == 13 else count, dtype)
    x, y, z = arrays
    assert reference.sci_ref_elements(which, C.ELEMENT[dtype], x.ctypes.data, y.ctypes.data, z.ctypes.data, count,
                                      out.ctypes.data) == 0
    return out


@pytest.mark.parametrize("dtype", INTEGERS)
def test_oracle_matches_reference_host_loop(oracle, reference, dtype):
    arrays = operands(dtype, 4099)
    for which in EVALUATIONS + list(REDUCTIONS):
        got = oracle_elements(oracle, which, arrays, dtype)
        want = reference_elements(reference, which, arrays, dtype)
        bad = np.flatnonzero(got != want)
        assert bad.size == 0, (np.dtype(dtype).name, which, bad[:5], got[bad[:5]], want[bad[:5]])


@pytest.mark.parametrize("dtype", [np.int8, np.uint32, np.int64])
def test_oracle_single_element_and_wrapping_sums(oracle, reference, dtype):
    # one element (the reduction starts from item.at(0)), and sums that wrap in the element's width
    # where C++ defines the wrap (unsigned types, and int8 through promotion)
    for count in (1, 2, 65537):
        arrays = operands(dtype, count, seed=count)
        if dtype != np.int64:
            info = np.iinfo(dtype)
            arrays = tuple(np.random.default_rng(count).integers(int(info.min) + 1, int(info.max), count, dtype=dtype,
                                                                 endpoint=True) for _ in range(3))
        for which in REDUCTIONS:
            got = oracle_elements(oracle, which, arrays, dtype)
            want = reference_elements(reference, which, arrays, dtype)
            assert got[0] == want[0], (np.dtype(dtype).name, count, which, got, want)


def test_elements_recorder_uses_float_bytecode_layout():
    # the recorder writes the same bytecode whatever the element type: literals as doubles, the
    # multiply-add contracted into fuse (chunk.hpp:119-168)
    a = C.Reference(16, 4, np.int32)
    b = C.Reference(32, 4, np.int32)
    chunk = C.record_output(a * b + 3)
    assert [step[0] for step in chunk.listing()] == ["fuse"]
    assert chunk.literals == 1 and chunk.constants[0] == 3.0


@pytest.mark.parametrize("dtype", [np.int8, np.int16, np.int32, np.uint8, np.uint32])
def test_integer_mean_matches_reference(oracle, reference, dtype):
    # sci::mean (reduce.hpp:24-28) over int arrays: the wrapped sum divided by the count converted to
    # the element type; the host side of libsci_b200.device.mean does that division on the device's
    # sum (here the oracle's)
    from libsci_b200.device import integer_mean

    for count in (1, 7, 100, 4099):
        arrays = operands(dtype, count, seed=count)
        total = oracle_elements(oracle, 10, arrays, dtype)[0]  # sum(x * y)
        want = reference_elements(reference, 13, arrays, dtype)[0]  # mean(x * y)
        assert integer_mean(total, count, dtype) == want, (np.dtype(dtype).name, count, total, want)


def test_golden_elements(oracle):
    """The reference's host-loop results committed by tests/golden/make_golden.py (elements.npz):
    the oracle matches them without oracle/_ref present, and its integer mean with the host-side
    division matches sci::mean."""
    from pathlib import Path

    from libsci_b200.device import integer_mean

    data = np.load(Path(__file__).resolve().parent / "golden" / "elements.npz")
    for dtype in INTEGERS:
        name = np.dtype(dtype).name
        arrays = tuple(np.ascontiguousarray(data[f"{v}_{name}"]) for v in "xyz")
        for which in EVALUATIONS + list(REDUCTIONS):
            got = oracle_elements(oracle, which, arrays, dtype)
            assert np.array_equal(got, data[f"{which}_{name}"]), (name, which)
        total = oracle_elements(oracle, 10, arrays, dtype)[0]
        assert integer_mean(total, arrays[0].size, dtype) == data[f"13_{name}"][0], name


def test_oracle_defines_the_undefined_cases(oracle):
    """Where C++ leaves the host loop undefined, the backend defines the result (and the device is
    held to the oracle there): division by zero gives 0, MIN / -1 wraps to MIN, signed overflow
    wraps, a NaN real result converts to 0 and out-of-range real results saturate."""
    def run(expression, arrays, dtype):
        chunk = C.record_output(expression)
        out = np.empty(arrays[0].size, dtype)
        assert oracle.sci_oracle_execute_elements(C.ELEMENT[np.dtype(dtype)], ctypes.byref(chunk), out.ctypes.data,
                                                  out.size) == 0
        return out

    for dtype in (np.int8, np.int32, np.int64):
        info = np.iinfo(dtype)
        x = np.array([7, info.min, info.max, -9, 0], dtype)
        y = np.array([0, -1, 2, 0, 0], dtype)
        a, b = leaves((x, y), dtype)
        assert run(a / b, (x, y), dtype).tolist() == [0, info.min, info.max // 2, 0, 0]
        wrapped = (x.astype(object) * 2 + 0)
        want = [((int(v) - int(info.min)) % (1 << (8 * np.dtype(dtype).itemsize))) + int(info.min) for v in wrapped]
        assert run(a * 2, (x, y), dtype).tolist() == want
        assert run(C.unary("root", a), (x, y), dtype).tolist()[1] == 0            # sqrt(MIN) is NaN -> 0
        assert run(C.unary("exponential", a), (x, y), dtype).tolist()[2] == info.max  # saturates
        assert run(C.unary("logarithm", a), (x, y), dtype).tolist()[4] == info.min    # log(0) = -inf

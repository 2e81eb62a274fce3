"""The oracle, pinned (CPU only).

oracle/sci_oracle.cpp restates libsci's CPU arithmetic; here it is checked bit for bit against
libsci's own CPU path compiled from the reference sources (oracle/_ref/libsci_ref.so) and against
the committed golden vectors, which tests/golden/make_golden.py produced from that same library.
The reference's own pins (tests/operations/test_binary.cpp, test_unary.cpp, test_reduce.cpp,
tests/linear/test_decompose.cpp, test_solve.cpp) are restated against the oracle as well.
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from libsci_b200 import chunk as C
from tests import _oracle

GOLDEN = Path(__file__).resolve().parent / "golden"


def host_inputs(dtype, count, seed):
    rng = np.random.default_rng(seed)
    x = np.concatenate([rng.standard_normal(count // 2) * 3, rng.uniform(-100, 100, count - count // 2)]).astype(dtype)
    y = rng.uniform(0, 10, count).astype(dtype)
    specials = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45, 1e-38, 3e-39, 88.7, 89.5, -103.9,
                         -104.5, 1e6, 2e6, -3e7, 1e30, 710.0, -746.0], dtype)
    x[: specials.size] = specials
    y[::97] = -0.0
    y[::101] = np.nan
    return x, y


def expression(code, a, b):
    if code < C.CODE["add"]:
        return C.Node(C.CODES[code], [a])
    if code == C.CODE["fuse"]:
        return a * b + b
    return C.Node(C.CODES[code], [a, b])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_oracle_matches_the_reference_bit_for_bit(oracle, reference, dtype):
    n = 20011  # crosses 1024-element blocks, leaves a ragged tail
    x, y = host_inputs(dtype, n, seed=3)
    a, b = C.Reference(x.ctypes.data, n, dtype), C.Reference(y.ctypes.data, n, dtype)
    for code in range(C.CODE["fuse"] + 1):
        chunk = C.record_output(expression(code, a, b))
        mine = _oracle.execute(oracle, chunk, n, dtype)
        theirs = _oracle.execute(reference, chunk, n, dtype)
        bad = _oracle.mismatches(mine, theirs)
        assert bad.size == 0, f"{C.CODES[code]}: {bad.size} differ"


def test_oracle_reductions_against_the_reference(oracle, reference):
    n = 300_007
    x, y = host_inputs(np.float32, n, seed=4)
    x = np.nan_to_num(x, nan=1.0, posinf=2.0, neginf=-2.0)
    y = np.nan_to_num(y, nan=0.5)
    a, b = C.Reference(x.ctypes.data, n, np.float32), C.Reference(y.ctypes.data, n, np.float32)
    for expr in (C.unary("sin", a) * C.unary("cos", b), C.unary("exponential", -a * a), a * b):
        chunk = C.record_reduce(expr)
        for fold in (C.SUM, C.MINIMUM, C.MAXIMUM):
            mine = _oracle.reduce(oracle, chunk, fold, n)
            theirs = _oracle.reduce(reference, chunk, fold, n)
            if fold == C.SUM:
                # the reference folds float partials per 1024-block (dispatch.cpp:121-150)
                assert abs(mine - theirs) <= 1e-4 * np.abs(x).sum()
            else:
                assert mine == theirs


def test_golden_vectors(oracle):
    """Per-code outputs of libsci's CPU path, committed by tests/golden/make_golden.py."""
    data = np.load(GOLDEN / "codes.npz")
    for dtype, suffix in ((np.float32, "f32"), (np.float64, "f64")):
        x, y = data[f"x_{suffix}"], data[f"y_{suffix}"]
        n = x.size
        a, b = C.Reference(x.ctypes.data, n, dtype), C.Reference(y.ctypes.data, n, dtype)
        for code in range(C.CODE["fuse"] + 1):
            chunk = C.record_output(expression(code, a, b))
            mine = _oracle.execute(oracle, chunk, n, dtype)
            want = data[f"{C.CODES[code]}_{suffix}"]
            assert _oracle.mismatches(mine, want).size == 0, C.CODES[code]


def test_golden_workloads(oracle):
    """The plain fused workload (t, e, s) at 4099 elements, from libsci's CPU path."""
    data = np.load(GOLDEN / "workloads.npz")
    a, b, c = data["a"], data["b"], data["c"]
    n = a.size
    ra, rb, rc = (C.Reference(v.ctypes.data, n, np.float32) for v in (a, b, c))
    t = _oracle.execute(oracle, C.record_output(ra * rb + rc * 2.0), n, np.float32)
    assert _oracle.mismatches(t, data["t"]).size == 0
    rt = C.Reference(t.ctypes.data, n, np.float32)
    e = _oracle.execute(oracle, C.record_output(C.unary("exponential", rt) * 0.5), n, np.float32)
    assert _oracle.mismatches(e, data["e"]).size == 0
    s = _oracle.reduce(oracle, C.record_reduce(C.unary("sin", rt)), C.SUM, n)
    assert abs(s - float(data["s"])) <= 1e-5 * abs(float(data["s"]))
    rows = np.zeros(64, np.uint64)
    m = data["lu_input"].copy()
    oracle.sci_oracle_factor_f32(m.ctypes.data, rows.ctypes.data, 64)
    assert np.array_equal(rows, data["lu_rows"])
    assert _oracle.mismatches(m.ravel(), data["lu_factors"].ravel()).size == 0


def test_reference_pins_restated(oracle):
    """tests/operations/test_binary.cpp:26-50 and test_unary.cpp:76-102 against the oracle."""
    n = 300_000
    first = (np.float64(-3.0) + np.arange(n) * (8.0 / (n - 1.0))).astype(np.float32)
    second = (np.float64(2.0) + np.arange(n) * (5.0 / (n - 1.0))).astype(np.float32)
    a, b = C.Reference(first.ctypes.data, n, np.float32), C.Reference(second.ctypes.data, n, np.float32)
    run = lambda e: _oracle.execute(oracle, C.record_output(e), n, np.float32)
    assert np.array_equal(run(a + b), first + second)
    assert np.array_equal(run(a / b), first / second)
    assert np.array_equal(run(C.binary("minimum", a, b)), np.minimum(first, second))
    assert np.array_equal(run(a + 2.0), first + np.float32(2.0))
    chunk = C.record_output(a * b + a)
    assert C.CODES[chunk.instructions[0].code] == "fuse" and chunk.length == 1
    wide = (np.float64(-4.0) + np.arange(100_000) * (8.0 / 99_999.0)).astype(np.float32)
    w = C.Reference(wide.ctypes.data, wide.size, np.float32)
    for name, fn in (("exponential", np.exp), ("sin", np.sin), ("cos", np.cos), ("tanh", np.tanh), ("atan", np.arctan)):
        got = _oracle.execute(oracle, C.record_output(C.unary(name, w)), wide.size, np.float32).astype(np.float64)
        want = fn(wide.astype(np.float64))
        assert np.all(np.abs(got - want) <= 1e-5 * np.maximum(1.0, np.abs(want))), name


def test_factor_restates_the_reference(oracle, reference):
    """LU pivot order and factors: decompose.hpp:29-72 (zero first pivot: test_decompose.cpp:21-36)."""
    a = np.array([[0, 2, 1], [4, 1, 3], [2, 5, 7]], np.float64)
    for lib, fn in ((oracle, "sci_oracle_factor_f64"), (reference, "sci_ref_factor_f64")):
        m = a.copy()
        rows = np.zeros(3, np.uint64)
        getattr(lib, fn)(m.ctypes.data, rows.ctypes.data, 3)
        lower = np.tril(m, -1) + np.eye(3)
        upper = np.triu(m)
        assert np.allclose(a[rows.astype(int)], lower @ upper, atol=1e-12)
        assert list(rows) == [1, 2, 0]
    rng = np.random.default_rng(9)
    g = rng.standard_normal((128, 128)).astype(np.float32)
    m1, m2 = g.copy(), g.copy()
    r1, r2 = np.zeros(128, np.uint64), np.zeros(128, np.uint64)
    oracle.sci_oracle_factor_f32(m1.ctypes.data, r1.ctypes.data, 128)
    reference.sci_ref_factor_f32(m2.ctypes.data, r2.ctypes.data, 128)
    assert np.array_equal(r1, r2)
    assert _oracle.mismatches(m1.ravel(), m2.ravel()).size == 0


# The codes whose results are exact sequences of rounded operations (not the C library's): every one
# must match libsci's CPU path bit for bit on any input.
EXACT_UNARY = ["copy", "negate", "absolute", "root", "exponential", "logarithm", "sin", "cos", "tan", "csc",
               "sec", "cot"]


def spread_floats(stride: int = 257) -> np.ndarray:
    """Every stride-th float bit pattern, 2^32 / stride values spanning every exponent and sign."""
    return (np.arange(0, 1 << 32, stride, dtype=np.uint64).astype(np.uint32)).view(np.float32)


def hashed_doubles(count: int, seed: int = 11) -> np.ndarray:
    """Doubles from hashed 64-bit patterns, half of them any pattern, half in each code's ordinary range."""
    rng = np.random.default_rng(seed)
    out = rng.integers(0, 1 << 63, count, dtype=np.int64).view(np.float64).copy()
    out[1::4] = rng.uniform(-750, 750, out[1::4].size)
    out[2::4] = rng.uniform(0, 1e6, out[2::4].size)
    out[3::4] = rng.uniform(-2.2e6, 2.2e6, out[3::4].size)
    return out


@pytest.mark.parametrize("code", EXACT_UNARY)
def test_oracle_matches_the_reference_across_the_float_range(oracle, reference, code):
    """The exact codes on every 257th float bit pattern (16.7 M values: all exponents, both signs,
    subnormals, infinities and NaNs) and on 2^22 hashed doubles."""
    for x in (spread_floats(), hashed_doubles(1 << 22)):
        n = x.size
        chunk = C.record_output(C.Node(code, [C.Reference(x.ctypes.data, n, x.dtype)]))
        mine = _oracle.execute(oracle, chunk, n, x.dtype)
        theirs = _oracle.execute(reference, chunk, n, x.dtype)
        bad = _oracle.mismatches(mine, theirs)
        assert bad.size == 0, f"{code} ({x.dtype}): {bad.size} of {n} differ, first input {x[bad[0]]!r}"


# ---- creation (include/operations/creation.hpp) -------------------------------------------------
def creation_functions(lib, prefix):
    """ctypes signatures of the creation functions of the oracle or of the reference bridge."""
    U32, U64, F64, VP = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_double, ctypes.c_void_p
    table = {"fill": [U32, VP, U64, F64], "full": [U32, VP, U64, F64], "linspace": [U32, VP, U64, F64, F64],
             "range_count": [U32, F64, F64, F64], "range": [U32, VP, U64, F64, F64], "eye": [U32, VP, U64, U64],
             "grid": [U32, VP, U64, VP, U64, VP, VP]}
    out = {}
    for name, args in table.items():
        fn = getattr(lib, f"{prefix}_{name}", None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = U64 if name == "range_count" else None
        out[name] = fn
    if prefix == "sci_ref":
        out["range"].argtypes = [U32, VP, U64, F64, F64, F64]
        out["range"].restype = U64
    return out


LINSPACES = [(0.0, 1.0, 5), (-3.7, 11.2, 1001), (1e-30, 1e30, 257), (5.0, 5.0, 10), (-0.0, 3.0, 1), (2.5, -7.25, 100003),
             (0.1, 0.7, 2), (0.0, 1.0, 0), (-1.0, 1.0, (1 << 20) + 3)]
RANGES = [(0.0, 10.0, 1.0), (-5.5, 17.25, 0.37), (10.0, 0.0, -0.3), (0.0, 3e7, 1.0), (1.0, 1.0, 1.0), (0.0, 1.0, 3.0),
          (0.1, 100.1, 0.01)]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_creation_oracle_matches_the_reference(oracle, reference, dtype):
    mine, theirs = creation_functions(oracle, "sci_oracle"), creation_functions(reference, "sci_ref")
    precision = 1 if dtype == np.float64 else 0
    for value in (0.0, 1.0, 2.5, -0.0, float("inf"), float("nan"), 1e40):
        a, b = np.empty(1003, dtype), np.empty(1003, dtype)
        mine["fill"](precision, a.ctypes.data, a.size, value)
        theirs["full"](precision, b.ctypes.data, b.size, value)
        assert _oracle.mismatches(a, b).size == 0, value
    for start, stop, count in LINSPACES:
        a, b = np.empty(max(count, 1), dtype), np.empty(max(count, 1), dtype)
        mine["linspace"](precision, a.ctypes.data, count, start, stop)
        theirs["linspace"](precision, b.ctypes.data, count, start, stop)
        assert _oracle.mismatches(a[:count], b[:count]).size == 0, (start, stop, count)
    for start, stop, step in RANGES:
        count = mine["range_count"](precision, start, stop, step)
        a, b = np.empty(max(count, 1), dtype), np.empty(max(count, 1), dtype)
        mine["range"](precision, a.ctypes.data, count, start, step)
        assert theirs["range"](precision, b.ctypes.data, b.size, start, stop, step) == count, (start, stop, step)
        assert _oracle.mismatches(a[:count], b[:count]).size == 0, (start, stop, step)
    for rows, columns in ((3, 3), (4, 7), (7, 4), (1, 1), (1000, 999)):
        a, b = np.empty(rows * columns, dtype), np.empty(rows * columns, dtype)
        mine["eye"](precision, a.ctypes.data, rows, columns)
        theirs["eye"](precision, b.ctypes.data, rows, columns)
        assert _oracle.mismatches(a, b).size == 0, (rows, columns)
    x, y = np.arange(7, dtype=dtype) * 0.5, np.arange(5, dtype=dtype) - 2
    xx, yy = np.empty(35, dtype), np.empty(35, dtype)
    mine["grid"](precision, x.ctypes.data, 7, y.ctypes.data, 5, xx.ctypes.data, yy.ctypes.data)
    gx, gy = np.meshgrid(x, y)  # numpy.meshgrid, which grid is named after
    assert np.array_equal(xx.reshape(5, 7), gx) and np.array_equal(yy.reshape(5, 7), gy)


def test_plain_workload_through_the_reference_api(oracle, reference):
    """The plain fused workload as bench.py's CPU arm runs it through libsci's public API
    (sci_ref_plain_*: a = linspace(0, 1, n), t = a*b + c*2, e = exp(t)*0.5, s = sum(sin t)) equals the
    oracle's chunks bit for bit, with s within the reference's float-block fold."""
    n = (1 << 16) + 5
    b = np.random.default_rng(0).uniform(-1, 1, n).astype(np.float32)
    c = np.ones(n, np.float32)
    handle = reference.sci_ref_plain_create(b.ctypes.data, c.ctypes.data, n)
    s = reference.sci_ref_plain_step(handle)

    def output(which):
        pointer = ctypes.cast(reference.sci_ref_plain_output(handle, which), ctypes.POINTER(ctypes.c_float))
        return np.ctypeslib.as_array(pointer, shape=(n,)).copy()

    t, e, a = output(0), output(1), output(2)
    reference.sci_ref_plain_destroy(handle)
    refs = [C.Reference(v.ctypes.data, n, np.float32) for v in (a, b, c)]
    t_want = _oracle.execute(oracle, C.record_output(refs[0] * refs[1] + refs[2] * 2.0), n, np.float32)
    assert _oracle.mismatches(t, t_want).size == 0
    tr = C.Reference(t_want.ctypes.data, n, np.float32)
    e_want = _oracle.execute(oracle, C.record_output(C.unary("exponential", tr) * 0.5), n, np.float32)
    assert _oracle.mismatches(e, e_want).size == 0
    s_want = _oracle.reduce(oracle, C.record_reduce(C.unary("sin", tr)), C.SUM, n)
    assert abs(s - s_want) <= 1e-6 * abs(s_want)

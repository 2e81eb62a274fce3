"""sci::gradient on the device (new; the reference has no differentiation, so no reference pins).

Oracles, as planned for this path: FP64 central differences evaluated on libsci's own CPU path
(oracle/_ref, the same expression recorded as a Precision::wide chunk), and closed-form FP64
gradients computed here with numpy.

Tolerance: |g - g64| <= 1e-6 * max(|g64|, 1e-3 * max|g64|), i.e. 1e-6 relative per coordinate with a
floor at a thousandth of the array's largest gradient (near a zero crossing relative error means
nothing). A float32 gradient carries the float rounding of the forward values it uses (a few ulps,
about 3e-7) and one final rounding; adjoints accumulate in double.
"""
import ctypes

import numpy as np
import pytest

from libsci_b200 import chunk as C
from tests import _oracle

pytestmark = pytest.mark.gpu

TOL = 1e-6


def close(got, want, tol=TOL):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    floor = 1e-3 * np.max(np.abs(want)) if want.size else 0.0
    scale = np.maximum(np.abs(want), floor)
    bad = np.abs(got - want) > tol * scale
    return not bad.any(), (np.abs(got - want) / np.where(scale > 0, scale, 1)).max() if want.size else 0.0


def c4(a, b, c):
    """L = sum(exponential(-a*a) * sin(b) + logarithm(1 + c*c)) (the differentiation workload)."""
    return C.unary("exponential", -a * a) * C.unary("sin", b) + C.unary("logarithm", 1 + c * c)


def fd_gradient(reference, build, hosts, index, coords, step=1e-5):
    """Central differences of f = build(*arguments) with respect to argument `index` at `coords`,
    evaluated in double on libsci's CPU path (a Precision::wide chunk through oracle/_ref)."""
    base = [np.ascontiguousarray(h[coords].astype(np.float64)) for h in hosts]
    h = step * np.maximum(1.0, np.abs(base[index]))

    def run(arrays):
        refs = [C.Reference(x.ctypes.data, len(coords), np.float64) for x in arrays]
        chunk = C.record_output(C._operand(build(*refs), None))
        return _oracle.execute(reference, chunk, len(coords), np.float64)

    plus = [x.copy() for x in base]
    minus = [x.copy() for x in base]
    plus[index] = base[index] + h
    minus[index] = base[index] - h
    return (run(plus) - run(minus)) / (plus[index] - minus[index])


def run_gradient(device, build, hosts, stored=False, seed=1.0):
    arrays = [device.array(h) for h in hosts]
    value, grads = device.gradient(build(*[x.expression() for x in arrays]), arrays, seed=seed, stored=stored)
    out = [g.numpy() for g in grads]
    for x in arrays + grads:
        x.free()
    return value, out


def c4_inputs(n, seed=0):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(n).astype(np.float32) for _ in range(3)]


def c4_analytic(a, b, c):
    a, b, c = (x.astype(np.float64) for x in (a, b, c))
    e = np.exp(-a * a)
    return [-2.0 * a * e * np.sin(b), e * np.cos(b), 2.0 * c / (1.0 + c * c)], float(np.sum(e * np.sin(b) + np.log1p(c * c)))


@pytest.mark.parametrize("stored", [False, True], ids=["recompute", "stored"])
def test_c4_gradient_against_fp64(device, stored):
    n = (1 << 20) + 3  # ragged: the last group of a thread is partial
    hosts = c4_inputs(n, seed=1)
    value, grads = run_gradient(device, c4, hosts, stored=stored)
    want, want_value = c4_analytic(*hosts)
    for g, w in zip(grads, want):
        ok, worst = close(g, w)
        assert ok, worst
    assert abs(value - want_value) <= 1e-6 * abs(want_value) + 1e-3


def test_c4_gradient_against_central_differences(device, reference):
    if reference is None:
        pytest.skip("oracle/_ref not built")
    n = 1 << 16
    hosts = c4_inputs(n, seed=2)
    _, grads = run_gradient(device, c4, hosts)
    coords = np.sort(np.random.default_rng(3).choice(n, 256, replace=False))
    for index in range(3):
        fd = fd_gradient(reference, c4, hosts, index, coords)
        ok, worst = close(grads[index][coords], fd)
        assert ok, (index, worst)


def test_forms_and_specialisation_agree(device):
    """The interpreter (first call) and the NVRTC-baked kernel (after jit_wait), recomputing and
    stored: the same forward values and the same double adjoints, so gradients agree to one ulp."""
    hosts = c4_inputs(100_003, seed=4)
    first = run_gradient(device, c4, hosts)
    device.jit_wait()
    baked = run_gradient(device, c4, hosts)
    stored = run_gradient(device, c4, hosts, stored=True)
    for other in (baked, stored):
        for g0, g1 in zip(first[1], other[1]):
            assert _oracle.ulp_distance(g0, g1).max() <= 1
        assert abs(first[0] - other[0]) <= 1e-9 * abs(first[0])


def test_value_matches_the_reduction(device, oracle):
    hosts = c4_inputs(4096, seed=5)
    value, _ = run_gradient(device, c4, hosts)
    arrays = [device.array(h) for h in hosts]
    want = device.reduce(c4(*[x.expression() for x in arrays]), C.SUM)
    assert abs(value - want) <= 1e-5 * abs(want)


def test_seed_scales_and_argument_used_twice(device):
    x = np.random.default_rng(6).standard_normal(1000).astype(np.float32)
    value, (g,) = run_gradient(device, lambda a: a * a, [x], seed=0.5)
    np.testing.assert_allclose(g, x.astype(np.float64), rtol=1e-7)  # d(0.5 * a^2)/da = a
    assert abs(value - float(np.sum(x.astype(np.float64) ** 2))) <= 1e-5 * value


# Unary codes with a domain each where they are smooth, and the closed-form derivative.
UNARY = {
    "copy": ((-2, 2), lambda x: np.ones_like(x)),
    "negate": ((-2, 2), lambda x: -np.ones_like(x)),
    "absolute": ((0.1, 2), lambda x: np.sign(x)),
    "root": ((0.1, 4), lambda x: 0.5 / np.sqrt(x)),
    "exponential": ((-3, 3), np.exp),
    "logarithm": ((0.1, 10), lambda x: 1 / x),
    "sin": ((-1.3, 1.3), np.cos),
    "cos": ((-1.3, 1.3), lambda x: -np.sin(x)),
    "tan": ((-1.2, 1.2), lambda x: 1 / np.cos(x) ** 2),
    "asin": ((-0.9, 0.9), lambda x: 1 / np.sqrt(1 - x * x)),
    "acos": ((-0.9, 0.9), lambda x: -1 / np.sqrt(1 - x * x)),
    "atan": ((-3, 3), lambda x: 1 / (1 + x * x)),
    "csc": ((0.2, 1.4), lambda x: -np.cos(x) / np.sin(x) ** 2),
    "sec": ((-1.2, 1.2), lambda x: np.sin(x) / np.cos(x) ** 2),
    "cot": ((0.2, 1.4), lambda x: -1 / np.sin(x) ** 2),
    "acsc": ((1.2, 5), lambda x: -1 / (np.abs(x) * np.sqrt(x * x - 1))),
    "asec": ((1.2, 5), lambda x: 1 / (np.abs(x) * np.sqrt(x * x - 1))),
    "acot": ((0.2, 3), lambda x: -1 / (1 + x * x)),
    "sinh": ((-3, 3), np.cosh),
    "cosh": ((-3, 3), np.sinh),
    "tanh": ((-3, 3), lambda x: 1 / np.cosh(x) ** 2),
    "asinh": ((-3, 3), lambda x: 1 / np.sqrt(x * x + 1)),
    "acosh": ((1.2, 5), lambda x: 1 / np.sqrt(x * x - 1)),
    "atanh": ((-0.9, 0.9), lambda x: 1 / (1 - x * x)),
    "csch": ((0.2, 3), lambda x: -np.cosh(x) / np.sinh(x) ** 2),
    "sech": ((-3, 3), lambda x: -np.sinh(x) / np.cosh(x) ** 2),
    "coth": ((0.2, 3), lambda x: -1 / np.sinh(x) ** 2),
    "acsch": ((0.2, 5), lambda x: -1 / (np.abs(x) * np.sqrt(x * x + 1))),
    "asech": ((0.1, 0.9), lambda x: -1 / (np.abs(x) * np.sqrt(1 - x * x))),
    "acoth": ((1.2, 5), lambda x: 1 / (1 - x * x)),
}


@pytest.mark.parametrize("code", list(UNARY))
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_unary_codes(device, reference, code, dtype):
    (lo, hi), derivative = UNARY[code]
    n = 4099
    x = np.random.default_rng(C.CODE[code]).uniform(lo, hi, n).astype(dtype)
    build = lambda a: C.unary(code, a)
    _, (g,) = run_gradient(device, build, [x])
    tol = TOL if dtype == np.float32 else 1e-12
    ok, worst = close(g, derivative(x.astype(np.float64)), tol)
    assert ok, worst
    if reference is not None:
        coords = np.arange(0, n, 64)
        fd = fd_gradient(reference, build, [x], 0, coords)
        ok, worst = close(g[coords], fd, max(tol, 1e-8))
        assert ok, worst


@pytest.mark.parametrize("code", ["add", "subtract", "multiply", "divide", "minimum", "maximum", "fuse"])
def test_binary_codes(device, reference, code):
    n = 4099
    rng = np.random.default_rng(40 + len(code))
    x = rng.uniform(0.5, 2, n).astype(np.float32)
    y = rng.uniform(0.5, 2, n).astype(np.float32)
    z = rng.uniform(-1, 1, n).astype(np.float32)
    if code == "fuse":
        build = lambda a, b, c: a * b + c
        hosts = [x, y, z]
    else:
        build = lambda a, b: C.binary(code, a, b)
        hosts = [x, y]
    _, grads = run_gradient(device, build, hosts)
    x64, y64 = x.astype(np.float64), y.astype(np.float64)
    want = {
        "add": [np.ones(n), np.ones(n)],
        "subtract": [np.ones(n), -np.ones(n)],
        "multiply": [y64, x64],
        "divide": [1 / y64, -x64 / y64 ** 2],
        "minimum": [(x64 < y64) * 1.0, (x64 >= y64) * 1.0],
        "maximum": [(x64 > y64) * 1.0, (x64 <= y64) * 1.0],
        "fuse": [y64, x64, np.ones(n)],
    }[code]
    for g, w in zip(grads, want):
        ok, worst = close(g, w)
        assert ok, worst
    if reference is not None and code not in ("minimum", "maximum"):
        coords = np.arange(0, n, 97)
        for index in range(len(hosts)):
            ok, worst = close(grads[index][coords], fd_gradient(reference, build, hosts, index, coords))
            assert ok, worst


def test_minimum_maximum_conventions(device):
    """Ties and NaNs: the adjoint goes to the operand the forward form returned. Elements from
    tail_start = n - n % 16 on take the loop-tail (Scalar) forms, as in the forward pass."""
    nan = np.nan
    # body (first 16) and tail (last 4): a tie, a NaN left, a NaN right, an ordinary pair
    x = np.array([1, nan, 2, 0.5] * 4 + [1, nan, 2, 0.5], np.float32)
    y = np.array([1, 3, nan, 0.25] * 4 + [1, 3, nan, 0.25], np.float32)
    _, (gx, gy) = run_gradient(device, lambda a, b: C.binary("minimum", a, b), [x, y])
    # body vmin: tie -> right; NaN left -> left; NaN right -> right (l < NaN is false); 0.25 < 0.5 -> right
    assert list(gx[:4]) == [0, 1, 0, 0] and list(gy[:4]) == [1, 0, 1, 1]
    # tail smin: tie -> left; any NaN -> l + r, both; 0.25 < 0.5 -> right
    assert list(gx[16:]) == [1, 1, 1, 0] and list(gy[16:]) == [0, 1, 1, 1]


def test_empty_and_skipped_gradients(device):
    from libsci_b200.native import lib

    x = device.array(np.ones(8, np.float32))
    y = device.array(np.ones(8, np.float32))
    chunk = C.record_reduce(x.expression() * y.expression())
    value = ctypes.c_double(7.0)
    slots = (ctypes.c_void_p * 2)()
    assert lib.sci_cuda_gradient(device.handle, ctypes.byref(chunk), 0, 1.0, slots, ctypes.byref(value), 0) == 0
    assert value.value == 0.0
    g = device.empty(8, np.float32)
    slots[0] = g.pointer  # only d/dx
    assert lib.sci_cuda_gradient(device.handle, ctypes.byref(chunk), 8, 1.0, slots, ctypes.byref(value), 0) == 0
    assert value.value == 8.0 and np.array_equal(g.numpy(), np.ones(8, np.float32))
    assert lib.sci_cuda_gradient(device.handle, ctypes.byref(chunk), 8, 1.0, None, None, 5) != 0  # unknown form

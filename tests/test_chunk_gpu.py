"""Parity of the CUDA chunk interpreter with libsci's CPU path (through the C ABI).

Bar (what the reference's own tests pin, tightened):
- every code except the nine C-library functions is bit-identical to the AVX-512 kernel table,
  NaN placement included (tests/operations/test_binary.cpp:29-42 pins exact `==` and the fused
  multiply-add; test_unary.cpp pins 1e-5 relative, far looser than bits);
- the C-library functions (asin ... atanh) and their reciprocal forms stay within 2 ulp (3 for
  1/f(x)) of glibc's float result, and within 1 ulp of the FP64 value;
- reductions: minimum / maximum exact; sum, mean and dot within 1e-9 relative of the FP64 fold;
  NaN anywhere gives NaN; empty sums 0 and empty extremes NaN (dispatch.cpp:109-111).
"""
import numpy as np
import pytest

from libsci_b200 import chunk as C
from tests import _oracle

pytestmark = pytest.mark.gpu

LIBRARY = {"asin", "acos", "atan", "sinh", "cosh", "tanh", "asinh", "acosh", "atanh",
           "acsc", "asec", "acot", "acsch", "asech", "acoth"}
RECIPROCAL_OF_LIBRARY = {"csch", "sech", "coth"}
SPECIALS = [0.0, -0.0, np.inf, -np.inf, np.nan, 1e-45, -1e-45, 1e-38, 3e-39, 88.7, 89.5, -103.9, -104.5,
            1e6, 2e6, -3e7, 1e30, 1.5707964, 710.0, -746.0, 0.5, -0.5, 1.0, -1.0, 2.0]


def inputs(dtype, count, seed=0):
    rng = np.random.default_rng(seed)
    x = np.concatenate([rng.standard_normal(count // 2) * 3, rng.uniform(-100, 100, count - count // 2)]).astype(dtype)
    y = rng.uniform(0, 10, count).astype(dtype)
    z = rng.uniform(-1, 1, count).astype(dtype)
    k = min(len(SPECIALS), count)
    x[:k] = np.array(SPECIALS[:k], dtype)
    if count > 200:
        y[::97] = -0.0
        y[::101] = np.nan
        x[count - 3:] = np.array([-0.0, 0.0, np.nan], dtype)[: 3]
        z[count - 3:] = np.array([0.0, -0.0, 1.0], dtype)[: 3]
    return x, y, z


class Mirror:
    """Device arrays with the host copies the oracle reads in their place."""

    def __init__(self, device):
        self.device, self.hosts = device, {}

    def put(self, host):
        arr = self.device.array(host)
        self.hosts[arr.pointer] = np.ascontiguousarray(host)
        return arr

    def view(self, arr, host):
        self.hosts[arr.pointer] = np.ascontiguousarray(host)
        return arr

    def execute(self, oracle, chunk, count, dtype):
        return _oracle.execute(oracle, _oracle.on_host(chunk, self.hosts), count, dtype)

    def reduce(self, oracle, chunk, fold, count):
        return _oracle.reduce(oracle, _oracle.on_host(chunk, self.hosts), fold, count)


def expression_for(code, a, b, c):
    if code < C.CODE["add"]:
        return C.Node(C.CODES[code], [a])
    if code == C.CODE["fuse"]:
        return a * b + c
    return C.Node(C.CODES[code], [a, b])


CIRCULAR = {"sin", "cos", "tan", "csc", "sec", "cot"}
REACH = 1048576.0  # beyond it sin/cos take the C library path (trigonometry.hpp:189-205)


def check_against_oracle(name, got, want, x=None):
    if name in CIRCULAR and x is not None:
        far = ~(np.abs(x) <= REACH)  # |x| > 2^20, inf and NaN go to the library on the CPU
        bad = _oracle.mismatches(got[~far], want[~far])
        assert bad.size == 0, f"{name}: {bad.size} in-range elements differ"
        bound = 2 if name in ("sin", "cos") else 4
        d = _oracle.ulp_distance(got[far], want[far])
        assert d.size == 0 or d.max() <= bound, f"{name}: far-range elements beyond {bound} ulp"
        return
    if name in LIBRARY or name in RECIPROCAL_OF_LIBRARY:
        # float: CUDA's double function rounded once vs glibc's float function (each within ~1 ulp
        # of the true value). double: two double libraries, each within ~2 ulp.
        wide = got.dtype == np.float64
        bound = (5 if wide else 3) if name in RECIPROCAL_OF_LIBRARY else (4 if wide else 2)
        d = _oracle.ulp_distance(got, want)
        assert d.max() <= bound, f"{name}: {int((d > bound).sum())} elements beyond {bound} ulp"
    else:
        bad = _oracle.mismatches(got, want)
        assert bad.size == 0, f"{name}: {bad.size} elements differ, first at {bad[:5]}: {got[bad[:5]]} vs {want[bad[:5]]}"


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("code", range(C.CODE["fuse"] + 1), ids=C.CODES)
def test_every_code_matches_the_cpu_path(device, oracle, code, dtype):
    n = 65536 + 13
    x, y, z = inputs(dtype, n, seed=code)
    m = Mirror(device)
    dx, dy, dz = m.put(x), m.put(y), m.put(z)
    expr = expression_for(code, dx.expression(), dy.expression(), dz.expression())
    got = device.evaluate(expr).numpy()
    want = m.execute(oracle, C.record_output(expr), n, dtype)
    check_against_oracle(C.CODES[code], got, want, x)


@pytest.mark.parametrize("count", [1, 2, 15, 16, 17, 31, 1023, 1024, 1025, 4099, (1 << 20) + 7])
def test_sizes_and_loop_tails(device, oracle, count):
    """Ragged sizes: the last count % 16 elements take the Scalar min/max forms, as on the CPU."""
    x, y, z = inputs(np.float32, count, seed=count)
    x[~(np.abs(x) <= REACH / 2)] = 0.75  # keep sin on its polynomial path: this test pins bits
    if count >= 4:
        x[-2:] = [0.0, -0.0]
        z[-2:] = [-0.0, 0.0]
        x[:2] = [0.0, -0.0]
        z[:2] = [-0.0, 0.0]
    m = Mirror(device)
    dx, dy, dz = m.put(x), m.put(y), m.put(z)
    a, b, c = dx.expression(), dy.expression(), dz.expression()
    for expr in (a * b + c * 2.0, C.binary("minimum", a, c), C.binary("maximum", c, a),
                 C.unary("exponential", a * b + c) * 0.5, C.unary("logarithm", b) - C.unary("sin", a)):
        got = device.evaluate(expr).numpy()
        want = m.execute(oracle, C.record_output(expr), count, np.float32)
        check_against_oracle("mixed", got, want)


def test_unaligned_operands_take_the_direct_path(device, oracle):
    n = 10007
    x, y, z = inputs(np.float32, n + 3, seed=7)
    m = Mirror(device)
    dx, dy = device.array(x), device.array(y)
    a = m.view(dx.offset(1, n), x[1:1 + n])
    b = m.view(dy.offset(3, n), y[3:3 + n])
    out = device.empty(n + 1, np.float32).offset(1, n)
    expr = C.unary("cos", a.expression()) * b.expression() + 1.5
    device.evaluate(expr, out)
    want = m.execute(oracle, C.record_output(expr), n, np.float32)
    check_against_oracle("unaligned", out.numpy(), want)


def test_plain_fused_expression_workload(device, oracle):
    """t = a*b + c*2, e = exp(t)*0.5, s = sum(sin(t)) at n = 2^20 (the plain fused workload)."""
    n = 1 << 20
    step = (1.0 - 0.0) / (n - 1.0)
    a = (0.0 + np.arange(n, dtype=np.float64) * step).astype(np.float32)  # linspace (creation.hpp:65-84)
    b = np.random.default_rng(0).uniform(-1, 1, n).astype(np.float32)
    c = np.ones(n, np.float32)
    m = Mirror(device)
    da, db, dc = m.put(a), m.put(b), m.put(c)
    t_expr = da * db + dc * 2.0
    t = device.evaluate(t_expr)
    t_host = t.numpy()
    assert _oracle.mismatches(t_host, m.execute(oracle, C.record_output(t_expr), n, np.float32)).size == 0
    m.view(t, t_host)
    e_expr = C.unary("exponential", t.expression()) * 0.5
    e = device.evaluate(e_expr)
    assert _oracle.mismatches(e.numpy(), m.execute(oracle, C.record_output(e_expr), n, np.float32)).size == 0
    s_chunk = C.record_reduce(C.unary("sin", t.expression()))
    s = device.reduce_chunk(s_chunk, C.SUM, n)
    s_want = m.reduce(oracle, s_chunk, C.SUM, n)
    assert abs(s - s_want) <= 1e-9 * abs(s_want)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_large_fused_chunks_with_nan(device, oracle, dtype):
    """The large fused chunks at a reduced n, NaN injected into z at rate 1e-6 (plus one sure NaN)."""
    n = (1 << 22) + 5
    rng = np.random.default_rng(1)
    x = rng.standard_normal(n).astype(dtype)
    y = rng.uniform(0.1, 10, n).astype(dtype)
    z = rng.uniform(-1, 1, n).astype(dtype)
    z[rng.choice(n, max(1, int(n * 1e-6)), replace=False)] = np.nan
    z[12345] = np.nan
    m = Mirror(device)
    dx, dy, dz = m.put(x), m.put(y), m.put(z)
    a, b, c = dx.expression(), dy.expression(), dz.expression()
    stored = C.unary("root", C.unary("absolute", a)) * C.unary("logarithm", b) + C.unary("tanh", c)
    got = device.evaluate(stored).numpy()
    want = m.execute(oracle, C.record_output(stored), n, dtype)
    # Everything but tanh is bit-exact, so the two results differ by tanh's library difference
    # (<= 2 ulp of tanh(z) for float, 4 for double) carried through the final add, plus that add's
    # rounding: an absolute bound, since the add can cancel.
    tanh_z = np.tanh(z.astype(np.float64)).astype(dtype)
    library_ulps = 4 if dtype == np.float64 else 2
    bound = library_ulps * np.spacing(np.abs(tanh_z)) + np.spacing(np.abs(want))
    finite = ~np.isnan(want)
    assert np.all(np.abs(got[finite].astype(np.float64) - want[finite]) <= bound[finite])
    assert np.array_equal(np.isnan(got), np.isnan(want))
    assert np.array_equal(np.isnan(got), np.isnan(z))
    for expr in (C.binary("minimum", a, c), C.binary("maximum", a, c)):
        out = device.evaluate(expr).numpy()
        assert _oracle.mismatches(out, m.execute(oracle, C.record_output(expr), n, dtype)).size == 0
    # reductions
    mean_chunk = C.record_reduce(C.unary("exponential", -a * a))
    total = device.reduce_chunk(mean_chunk, C.SUM, n)
    total_want = m.reduce(oracle, mean_chunk, C.SUM, n)
    assert abs(total - total_want) <= 1e-9 * abs(total_want)
    peak = C.record_reduce(C.unary("sin", a) * C.unary("cos", c))
    assert np.isnan(device.reduce_chunk(peak, C.MAXIMUM, n))
    assert np.isnan(device.reduce_chunk(C.record_reduce(a * c), C.SUM, n))
    # the same without NaN: exact extremes, dot contracted
    clean = np.nan_to_num(z, nan=0.25)
    dz.upload(clean)
    m.view(dz, clean)
    assert device.reduce_chunk(peak, C.MAXIMUM, n) == m.reduce(oracle, peak, C.MAXIMUM, n)
    assert device.reduce_chunk(peak, C.MINIMUM, n) == m.reduce(oracle, peak, C.MINIMUM, n)
    dot_chunk = C.record_reduce(a * c)
    assert dot_chunk.contracted(C.SUM)
    got_dot = device.reduce_chunk(dot_chunk, C.SUM, n)
    want_dot = m.reduce(oracle, dot_chunk, C.SUM, n)
    scale = float(np.sum(np.abs(x.astype(np.float64) * clean.astype(np.float64))))
    assert abs(got_dot - want_dot) <= 1e-9 * scale


def test_reduction_edges(device):
    empty = device.empty(0, np.float32)
    ref = empty.expression()
    assert device.reduce_chunk(C.record_reduce(ref), C.SUM, 0) == 0.0
    assert np.isnan(device.reduce_chunk(C.record_reduce(ref), C.MINIMUM, 0))
    assert np.isnan(device.reduce_chunk(C.record_reduce(ref), C.MAXIMUM, 0))
    one = device.array(np.array([3.5], np.float32))
    for fold in (C.SUM, C.MINIMUM, C.MAXIMUM):
        assert device.reduce_chunk(C.record_reduce(one.expression()), fold, 1) == 3.5
    infs = device.array(np.array([np.inf, -np.inf, 1.0] * 1000, np.float32))
    assert np.isnan(device.reduce_chunk(C.record_reduce(infs.expression()), C.SUM, 3000))
    assert device.reduce_chunk(C.record_reduce(infs.expression()), C.MINIMUM, 3000) == -np.inf
    assert device.reduce_chunk(C.record_reduce(infs.expression()), C.MAXIMUM, 3000) == np.inf


def test_reference_pins_on_the_device(device, oracle):
    """tests/operations/test_binary.cpp and test_reduce.cpp, restated on the device."""
    n = 300_000
    first = (np.float64(-3.0) + np.arange(n) * ((5.0 - -3.0) / (n - 1.0))).astype(np.float32)
    second = (np.float64(2.0) + np.arange(n) * ((7.0 - 2.0) / (n - 1.0))).astype(np.float32)
    f, s = device.array(first), device.array(second)
    a, b = f.expression(), s.expression()
    assert np.array_equal(device.evaluate(a + b).numpy(), first + second)
    assert np.array_equal(device.evaluate(a - b).numpy(), first - second)
    assert np.array_equal(device.evaluate(a * b).numpy(), first * second)
    assert np.array_equal(device.evaluate(a / b).numpy(), first / second)
    assert np.array_equal(device.evaluate(C.binary("minimum", a, b)).numpy(), np.minimum(first, second))
    assert np.array_equal(device.evaluate(C.binary("maximum", a, b)).numpy(), np.maximum(first, second))
    fused = device.evaluate(a * b + a).numpy()
    want = np.array([oracle.sci_oracle_apply_f32(C.CODE["fuse"], p, q, p, 0) for p, q in zip(first[:5000], second[:5000])],
                    np.float32)
    assert np.array_equal(fused[:5000], want)  # std::fma(a, b, a): one rounding
    nan = device.array(np.full(4, np.nan, np.float32))
    ones = device.array(np.ones(4, np.float32))
    assert np.isnan(device.evaluate(C.binary("minimum", nan.expression(), ones.expression())).numpy()).all()
    assert np.isnan(device.evaluate(C.binary("maximum", ones.expression(), nan.expression())).numpy()).all()
    ramp = (np.float64(-1.0) + np.arange(1_000_000) * (3.0 / 999_999.0)).astype(np.float32)
    r = device.array(ramp)
    total = ramp.astype(np.float64).sum()
    assert abs(device.reduce_chunk(C.record_reduce(r.expression()), C.SUM, ramp.size) - total) < 1e-3 * ramp.size
    assert device.reduce_chunk(C.record_reduce(r.expression()), C.MINIMUM, ramp.size) == ramp.min()
    assert device.reduce_chunk(C.record_reduce(r.expression()), C.MAXIMUM, ramp.size) == ramp.max()


def test_invalid_chunks_are_rejected(device):
    from libsci_b200.native import SciCudaError

    x = device.array(np.ones(16, np.float32))
    out = device.empty(16)
    bad = C.record_output(x.expression() * 2.0)
    bad.instructions[0].code = 99
    with pytest.raises(SciCudaError):
        device.execute(bad, out.pointer, 16)
    bad = C.record_output(x.expression() * 2.0)
    bad.instructions[0].sources[1] = C.LITERAL | 5
    with pytest.raises(SciCudaError):
        device.execute(bad, out.pointer, 16)
    host = np.ones(16, np.float32)
    foreign = C.record_output(C.Reference(host.ctypes.data, 16, np.float32) * 2.0)
    with pytest.raises(SciCudaError):
        device.execute(foreign, out.pointer, 16)
    # the context still works afterwards
    device.evaluate(x.expression() * 2.0, out)
    assert np.array_equal(out.numpy(), np.full(16, 2.0, np.float32))


@pytest.mark.parametrize("name,function,low,high", [
    ("asin", np.arcsin, -1, 1), ("acos", np.arccos, -1, 1), ("atan", np.arctan, -20, 20),
    ("sinh", np.sinh, -20, 20), ("cosh", np.cosh, -20, 20), ("tanh", np.tanh, -5, 5),
    ("asinh", np.arcsinh, -50, 50), ("acosh", np.arccosh, 1, 50), ("atanh", np.arctanh, -1, 1)])
def test_library_functions_against_fp64(device, name, function, low, high):
    """The nine C-library codes are computed in double and rounded once: within 1 ulp of the
    correctly rounded float (the FP64 value rounded to float)."""
    x = np.random.default_rng(5).uniform(low, high, 200_003).astype(np.float32)
    got = device.evaluate(C.unary(name, device.array(x).expression())).numpy()
    with np.errstate(all="ignore"):
        truth = function(x.astype(np.float64)).astype(np.float32)
    assert _oracle.ulp_distance(got, truth).max() <= 1

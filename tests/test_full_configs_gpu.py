"""Parity at the workloads' full sizes (the other GPU tests run reduced sizes).

Each test runs one workload at the size the benchmark measures and checks it against the CPU
oracles with the same bars as the reduced tests:

- large fused chunks, float32, 2^28 per array, NaN in z at rate 1e-6: every stored element of the
  three elementwise chunks against the oracle's restatement of libsci's CPU path (bit for bit for
  minimum / maximum, within tanh's library bound for the stored chunk), the three reductions
  against FP64 folds of the oracle's per-element values (1e-9 relative; extremes exact) and against
  libsci's own reduce (1e-6: it folds 1024-element blocks in float);
- product, M = N = K = 8192, every mode: 64 seeded rows against the oracle's FP64 rows, within the
  per-mode bounds of tests/test_product_gpu.py;
- solve, n = 8192 with 16 right-hand sides, A = G + nI and A = G: normwise backward error <= 1e-14
  for FP32 LU + FP64 refinement and for plain FP64 LU; the tensor-core FP32 factor's pivot sequence
  equal to libsci's factor<float> (include/linear/decompose.hpp:29-72) on a tie-free input;
- gradients: sum(exp(-a*a)*sin(b) + log(1+c*c)) at 2^26 per array, every coordinate against the
  closed form in FP64 (1e-6 relative, floor at 1e-3 of the largest) and 256 seeded coordinates
  per argument against central differences on libsci's CPU path; the adjoint of sum(G * solve(A, B))
  at 4096 x 64 against FP64 (1e-10 normwise) and central differences through libsci's solve<double>;
- batches: all 8192 expression items (t bit for bit against libsci's CPU path item by item, the
  reduced value within 1e-6 of the sum of magnitudes) and all 4096 small solves (backward error
  <= 1e-14, the solution within 1e-10 of libsci's solve<double>).

Reference pins these follow: tests/operations/test_binary.cpp:29-42 (exact elementwise results),
tests/linear/test_decompose.cpp:21-36 (pivot order), tests/linear/test_solve.cpp:8-25 (solutions).
"""
import ctypes
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from libsci_b200 import chunk as C
from tests import _oracle

pytestmark = pytest.mark.gpu

THREADS = 16
BLOCK = 1 << 24  # oracle work is cut into blocks of this many elements (a multiple of 16: no loop tail)


def blockwise(count, work):
    """Runs work(begin, end) over [0, count) in BLOCK pieces on a thread pool (the oracle's ctypes
    calls release the GIL) and returns the results in order."""
    spans = [(o, min(count, o + BLOCK)) for o in range(0, count, BLOCK)]
    with ThreadPoolExecutor(THREADS) as pool:
        return list(pool.map(lambda span: work(*span), spans))


def oracle_values(oracle, build, hosts, begin, end):
    """The oracle's per-element float values of build(*inputs) over [begin, end)."""
    n = end - begin
    views = [np.ascontiguousarray(h[begin:end]) for h in hosts]
    refs = [C.Reference(v.ctypes.data, n, v.dtype) for v in views]
    return _oracle.execute(oracle, C.record_output(C._operand(build(*refs), None)), n, views[0].dtype)


# ---- large fused chunks, 2^28 floats ---------------------------------------------------------------
def test_large_fused_chunks_at_full_size(device, oracle):
    import bench

    n = 1 << 28
    x, y, z = bench.generate(n, seed=0)
    nan_at = np.flatnonzero(np.isnan(z))
    assert nan_at.size == 268
    dx, dy, dz = device.array(x), device.array(y), device.array(z)
    a, b, c = dx.expression(), dy.expression(), dz.expression()

    def stored_of(p, q, r):
        return C.unary("root", C.unary("absolute", p)) * C.unary("logarithm", q) + C.unary("tanh", r)

    out = device.empty(n)
    device.execute(C.record_output(stored_of(a, b, c)), out.pointer, n)
    got = out.numpy()

    def check_stored(begin, end):
        want = oracle_values(oracle, stored_of, (x, y, z), begin, end)
        g = got[begin:end]
        # everything but tanh is bit-exact: the results differ by tanh's library difference (<= 2 ulp
        # of tanh(z)) carried through the final add, plus that add's rounding
        tanh_z = np.tanh(z[begin:end].astype(np.float64)).astype(np.float32)
        bound = 2 * np.spacing(np.abs(tanh_z)).astype(np.float64) + np.spacing(np.abs(want)).astype(np.float64)
        finite = ~np.isnan(want)
        within = bool(np.all(np.abs(g[finite].astype(np.float64) - want[finite]) <= bound[finite]))
        return within, bool(np.array_equal(np.isnan(g), np.isnan(want)))

    results = blockwise(n, check_stored)
    assert all(r[0] for r in results), "stored chunk outside tanh's library bound"
    assert all(r[1] for r in results), "NaN placement of the stored chunk"
    assert np.array_equal(np.flatnonzero(np.isnan(got)), nan_at)

    for name in ("minimum", "maximum"):
        device.execute(C.record_output(C.binary(name, a, c)), out.pointer, n)
        got = out.numpy()
        counts = blockwise(n, lambda s, e: _oracle.mismatches(
            got[s:e], oracle_values(oracle, lambda p, r: C.binary(name, p, r), (x, z), s, e)).size)
        assert sum(counts) == 0, (name, sum(counts))
    out.free()

    # reductions: FP64 folds of the oracle's per-element float values
    mean_chunk = C.record_reduce(C.unary("exponential", -a * a))
    total = device.reduce_chunk(mean_chunk, C.SUM, n)
    parts = blockwise(n, lambda s, e: float(np.sum(oracle_values(
        oracle, lambda p: C.unary("exponential", -p * p), (x,), s, e).astype(np.float64))))
    want_total = float(np.sum(parts))
    assert abs(total - want_total) <= 1e-9 * abs(want_total)

    peak_chunk = C.record_reduce(C.unary("sin", a) * C.unary("cos", c))
    dot_chunk = C.record_reduce(a * c)
    assert dot_chunk.contracted(C.SUM)
    assert np.isnan(device.reduce_chunk(peak_chunk, C.MAXIMUM, n))  # the NaN in z wins
    assert np.isnan(device.reduce_chunk(dot_chunk, C.SUM, n))

    reference = _oracle.reference()
    if reference is not None:  # libsci's own reduce folds float blocks: 1e-6
        on_host = _oracle.on_host(mean_chunk, {dx.pointer: x})
        assert abs(total - reference.sci_ref_reduce(ctypes.byref(on_host), C.SUM, n)) <= 1e-6 * abs(want_total)

    # the same without NaN: exact extremes, the dot against exact FP64 products
    clean = np.where(np.isnan(z), np.float32(0.25), z)
    dz.upload(clean)
    sin_cos = lambda p, r: C.unary("sin", p) * C.unary("cos", r)  # noqa: E731
    values = blockwise(n, lambda s, e: (lambda v: (float(v.max()), float(v.min())))(
        oracle_values(oracle, sin_cos, (x, clean), s, e)))
    assert device.reduce_chunk(peak_chunk, C.MAXIMUM, n) == max(v[0] for v in values)
    assert device.reduce_chunk(peak_chunk, C.MINIMUM, n) == min(v[1] for v in values)
    got_dot = device.reduce_chunk(dot_chunk, C.SUM, n)
    parts = blockwise(n, lambda s, e: (float(np.dot(x[s:e].astype(np.float64), clean[s:e].astype(np.float64))),
                                       float(np.sum(np.abs(x[s:e].astype(np.float64) * clean[s:e])))))
    want_dot, scale = sum(p[0] for p in parts), sum(p[1] for p in parts)
    assert abs(got_dot - want_dot) <= 1e-9 * scale
    for arr in (dx, dy, dz):
        arr.free()


# ---- product, 8192^3 -------------------------------------------------------------------------------
BF16, SPLIT, FP32, SPLIT3 = 0, 1, 2, 3


def product_bound(mode, k, s):
    return {FP32: k * 2.0 ** -23, BF16: 2.0 ** -7 + k * 2.0 ** -22, SPLIT: 2.0 ** -14 + k * 2.0 ** -22,
            SPLIT3: 2.0 ** -21 + k * 2.0 ** -22}[mode] * s + 1e-30


def test_product_at_full_size(device, oracle):
    size = 8192
    rng = np.random.default_rng(0)
    a = rng.uniform(-1, 1, (size, size)).astype(np.float32)
    b = rng.uniform(-1, 1, (size, size)).astype(np.float32)
    rows = np.sort(rng.choice(size, 64, replace=False))
    want = np.zeros((len(rows), size))

    def oracle_row(i):
        oracle.sci_oracle_product_rows(a.ctypes.data, b.ctypes.data, want[i].ctypes.data, size, size, size,
                                       int(rows[i]), int(rows[i]) + 1)

    with ThreadPoolExecutor(THREADS) as pool:
        list(pool.map(oracle_row, range(len(rows))))
    s = np.abs(a[rows].astype(np.float64)) @ np.abs(b.astype(np.float64))
    da, db, dc = device.array(a.ravel()), device.array(b.ravel()), device.empty(size * size)
    errors = {}
    for mode in (BF16, SPLIT, SPLIT3, FP32):
        device.product(da, db, size, size, size, mode=mode, out=dc)
        got = dc.numpy().reshape(size, size)[rows]
        assert np.all(np.abs(got - want) <= product_bound(mode, size, s)), mode
        errors[mode] = np.linalg.norm(got - want) / np.linalg.norm(want)
    # split3 at FP32's accuracy (measured 1.9e-6 against plain FP32's 1.6e-6), split about 16 bits,
    # bf16 about 8
    assert errors[FP32] <= 4e-6 and errors[SPLIT3] <= 4e-6
    assert errors[SPLIT] <= 2e-5 and errors[BF16] <= 4e-3
    for arr in (da, db, dc):
        arr.free()


# ---- solve and factor, n = 8192 ----------------------------------------------------------------------
def backward_errors(a, b, x):
    r = np.abs(b - a @ x).max(axis=0)
    return r / (np.abs(a).sum(axis=1).max() * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))


@pytest.mark.parametrize("shift", [True, False], ids=["G+nI", "G"])
def test_solve_at_full_size(device, shift):
    n, width = 8192, 16
    rng = np.random.default_rng(17 + int(shift))
    a = rng.standard_normal((n, n)) + (n * np.eye(n) if shift else 0.0)
    b = rng.standard_normal((n, width))
    da, db = device.array(a.ravel()), device.array(b.ravel())
    solutions = {}
    for refine in (True, False):
        x, berr, iterations = device.solve(da, db, n, width, refine=refine)
        solutions[refine] = x.numpy().reshape(n, width)
        x.free()
        assert berr <= 1e-14, (refine, berr)
        # recomputed here in FP64 (numpy's own summation adds its rounding to the residual)
        assert backward_errors(a, b, solutions[refine]).max() <= 4e-14
        if refine:
            assert 1 <= iterations <= 30
    scale = np.abs(solutions[False]).max() * (1 if shift else 1e3)
    assert np.abs(solutions[True] - solutions[False]).max() <= 1e-9 * scale
    da.free()
    db.free()


def test_tensor_core_factor_pivots_at_full_size(device, reference):
    """libsci's factor<float> (about 20 s on the host) against the tensor-core and plain FP32
    factors on a tie-free input: a row-shuffled diagonally dominant matrix, whose every column has
    one entry far above the rest, so rounding cannot reorder the candidates. On a plain Gaussian
    matrix P A = L U is checked on 64 seeded rows."""
    n = 8192
    rng = np.random.default_rng(8192)
    shuffled = (rng.standard_normal((n, n)) + 4 * n * np.eye(n))[rng.permutation(n)].astype(np.float32)
    want_rows = np.zeros(n, np.uint64)
    host = shuffled.copy()
    reference.sci_ref_factor_f32(host.ctypes.data, want_rows.ctypes.data, n)
    for plain in (False, True):
        d = device.array(shuffled.ravel())
        rows = device.factor(d, n, plain=plain)
        d.free()
        assert np.array_equal(rows, want_rows), plain

    g = rng.standard_normal((n, n)).astype(np.float32)
    d = device.array(g.ravel())
    rows = device.factor(d, n)
    lu = d.numpy().reshape(n, n)
    d.free()
    assert np.array_equal(np.sort(rows), np.arange(n))
    sample = np.sort(rng.choice(n, 64, replace=False))
    upper = np.triu(lu.astype(np.float64))
    columns = np.arange(n)
    lower = np.where(columns[None, :] < sample[:, None], lu[sample].astype(np.float64), 0.0)
    lower[np.arange(len(sample)), sample] = 1.0  # rows `sample` of the unit lower triangle L
    err = np.abs(g.astype(np.float64)[rows.astype(np.int64)[sample]] - lower @ upper).max() / np.abs(g).max()
    assert err <= 1e-6 * n


# ---- gradients ---------------------------------------------------------------------------------------
def c4(a, b, c):
    return C.unary("exponential", -a * a) * C.unary("sin", b) + C.unary("logarithm", 1 + c * c)


def fd_gradient(reference, hosts, index, coords, step=1e-5):
    """Central differences of the C4 summand with respect to argument `index` at `coords`, in double
    on libsci's CPU path (a Precision::wide chunk through oracle/_ref)."""
    base = [np.ascontiguousarray(h[coords].astype(np.float64)) for h in hosts]
    h = step * np.maximum(1.0, np.abs(base[index]))

    def run(arrays):
        refs = [C.Reference(v.ctypes.data, len(coords), np.float64) for v in arrays]
        return _oracle.execute(reference, C.record_output(C._operand(c4(*refs), None)), len(coords), np.float64)

    plus, minus = [v.copy() for v in base], [v.copy() for v in base]
    plus[index] = base[index] + h
    minus[index] = base[index] - h
    return (run(plus) - run(minus)) / (plus[index] - minus[index])


def relative_to(got, want, tol):
    floor = 1e-3 * np.abs(want).max()
    return bool(np.all(np.abs(got - want) <= tol * np.maximum(np.abs(want), floor)))


@pytest.mark.parametrize("stored", [False, True], ids=["recompute", "stored"])
def test_chunk_gradient_at_full_size(device, reference, stored):
    n = 1 << 26
    rng = np.random.default_rng(0)
    hosts = [rng.standard_normal(n, dtype=np.float32) for _ in range(3)]
    arrays = [device.array(h) for h in hosts]
    value, grads = device.gradient(c4(*[v.expression() for v in arrays]), arrays, stored=stored)
    got = [g.numpy() for g in grads]
    for v in arrays + grads:
        v.free()

    def closed_form(begin, end):
        a, b, c = (h[begin:end].astype(np.float64) for h in hosts)
        e = np.exp(-a * a)
        return [-2.0 * a * e * np.sin(b), e * np.cos(b), 2.0 * c / (1.0 + c * c)], \
            float(np.sum(e * np.sin(b) + np.log1p(c * c)))

    # two passes: the largest gradient of each argument first (it sets the floor), then the check
    first = blockwise(n, lambda s, e: (lambda w: ([float(np.abs(v).max()) for v in w[0]], w[1]))(closed_form(s, e)))
    largest = [max(f[0][i] for f in first) for i in range(3)]
    want_value = sum(f[1] for f in first)
    assert abs(value - want_value) <= 1e-6 * abs(want_value)

    def check(begin, end):
        want, _ = closed_form(begin, end)
        return [bool(np.all(np.abs(got[i][begin:end] - want[i]) <= 1e-6 * np.maximum(np.abs(want[i]), 1e-3 * largest[i])))
                for i in range(3)]

    assert all(all(ok) for ok in blockwise(n, check))

    coords = np.sort(np.random.default_rng(3).choice(n, 256, replace=False))
    for index in range(3):
        assert relative_to(got[index][coords].astype(np.float64), fd_gradient(reference, hosts, index, coords), 1e-6), index


def test_solve_gradient_at_full_size(device, reference):
    n, width = 4096, 64
    rng = np.random.default_rng(1)
    a = rng.standard_normal((n, n)) + n * np.eye(n)
    b = rng.standard_normal((n, width))
    g = rng.standard_normal((n, width))
    operands = [device.array(v.ravel()) for v in (a, b, g)]
    outputs = device.solve_gradient(*operands, n, width, refine=True)
    x, dA, dB = outputs[0].numpy().reshape(n, width), outputs[1].numpy().reshape(n, n), outputs[2].numpy().reshape(n, width)
    berr, iterations = outputs[3], outputs[4]
    for v in operands + list(outputs[:3]):
        v.free()
    want_x = np.linalg.solve(a, b)
    lam = np.linalg.solve(a.T, g)
    want_dA = -lam @ want_x.T

    def normwise(got, want):
        return np.abs(got - want).max() / np.abs(want).max()

    assert berr <= 1e-14 and iterations >= 1
    assert normwise(x, want_x) <= 1e-10
    assert normwise(dB, lam) <= 1e-10
    assert normwise(dA, want_dA) <= 1e-10

    def loss(mat, rhs):
        out = np.empty((n, width))
        reference.sci_ref_solve_f64(np.ascontiguousarray(mat).ctypes.data, np.ascontiguousarray(rhs).ctypes.data,
                                    out.ctypes.data, n, width)
        return float(np.sum(g * out))

    # central differences through libsci's solve<double> (two solves of 4096 per coordinate). A
    # step of 0.5 against a diagonal of 4096 keeps the truncation error near (0.5/4096)^2 relative,
    # while a step of 1e-4 would drown the ~1e-7 derivative in the loss's own rounding; the loss is
    # linear in B, so there any step is exact up to rounding.
    for _ in range(2):
        i, j = rng.integers(n), rng.integers(n)
        h = 0.5 * max(1.0, abs(a[i, j]))
        ap, am = a.copy(), a.copy()
        ap[i, j] += h
        am[i, j] -= h
        fd = (loss(ap, b) - loss(am, b)) / (ap[i, j] - am[i, j])
        assert abs(dA[i, j] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(dA).max())
    i, c = rng.integers(n), rng.integers(width)
    h = 1.0
    bp, bm = b.copy(), b.copy()
    bp[i, c] += h
    bm[i, c] -= h
    fd = (loss(a, bp) - loss(a, bm)) / (bp[i, c] - bm[i, c])
    assert abs(dB[i, c] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(dB).max())


# ---- batches -----------------------------------------------------------------------------------------
def test_expression_batch_at_full_size(device, reference):
    """8192 items, lengths log-uniform in [256, 2^20] (1.03e9 elements), checked item by item."""
    import torch

    import bench

    items = 8192
    rng = np.random.default_rng(0)
    counts = np.exp(rng.uniform(np.log(256), np.log(1 << 20), items)).astype(np.int64)
    offsets = np.concatenate([[0], np.cumsum((counts + 63) // 64 * 64)])
    total = int(offsets[-1])
    generator = torch.Generator(device="cuda").manual_seed(0)
    inputs = [torch.randn(total, generator=generator, device="cuda", dtype=torch.float32) for _ in range(3)]
    t_out = torch.empty(total, device="cuda", dtype=torch.float32)
    results = torch.zeros(items, device="cuda", dtype=torch.float64)
    pointers = np.array([[v.data_ptr() + 4 * int(o) for v in inputs] for o in offsets[:-1]], np.uint64)
    outputs = np.array([t_out.data_ptr() + 4 * int(o) for o in offsets[:-1]], np.uint64)

    class Results:
        pointer = results.data_ptr()

    batch = device.batch(bench.batch_chunk(C), C.SUM, pointers, counts, outputs, Results)
    batch.launch()
    device.synchronize()
    got = results.cpu().numpy()
    t_host = t_out.cpu().numpy()
    host = [v.cpu().numpy() for v in inputs]
    batch.close()
    del inputs, t_out, results

    def check(k):
        o, n = int(offsets[k]), int(counts[k])
        a, b, c = (np.ascontiguousarray(h[o:o + n]) for h in host)
        refs = [C.Reference(v.ctypes.data, n, np.float32) for v in (a, b, c)]
        t = _oracle.execute(reference, C.record_output(refs[0] * refs[1] + refs[2]), n, np.float32)
        tr = C.Reference(t.ctypes.data, n, np.float32)
        values = _oracle.execute(reference, C.record_output(C.unary("tanh", tr)), n, np.float32).astype(np.float64)
        same = _oracle.mismatches(t_host[o:o + n], t).size == 0
        return same, abs(got[k] - values.sum()) <= 1e-6 * np.abs(values).sum()

    # one item at a time: libsci's CPU path runs each call on its own process-wide thread pool
    checks = [check(k) for k in range(items)]
    assert all(c[0] for c in checks), [k for k, c in enumerate(checks) if not c[0]][:10]
    assert all(c[1] for c in checks), [k for k, c in enumerate(checks) if not c[1]][:10]


def test_solve_batch_at_full_size(device, reference):
    """4096 systems, n ~ U[8, 256], A = G + nI, one right-hand side: every system checked."""
    count = 4096
    rng = np.random.default_rng(0)
    orders = rng.integers(8, 257, count)
    mats = [rng.standard_normal((n, n)) + n * np.eye(n) for n in orders]
    rhs = [rng.standard_normal(n) for n in orders]
    offsets_a = np.concatenate([[0], np.cumsum(orders * orders)])
    offsets_b = np.concatenate([[0], np.cumsum(orders)])
    flat_a = device.array(np.concatenate([m.ravel() for m in mats]))
    flat_b = device.array(np.concatenate(rhs))
    flat_x = device.empty(int(offsets_b[-1]), np.float64)
    errors = device.empty(count, np.float64)
    iterations = device.empty(count, np.int32)
    batch = device.solve_batch(orders, [flat_a.pointer + 8 * int(o) for o in offsets_a[:-1]],
                               [flat_b.pointer + 8 * int(o) for o in offsets_b[:-1]],
                               [flat_x.pointer + 8 * int(o) for o in offsets_b[:-1]], errors, iterations)
    batch.launch()
    x, berr, its = flat_x.numpy(), errors.numpy(), iterations.numpy()
    batch.close()
    for arr in (flat_a, flat_b, flat_x, errors, iterations):
        arr.free()

    def check(k):
        n = int(orders[k])
        xk = x[offsets_b[k]:offsets_b[k + 1]]
        a, b = mats[k], rhs[k]
        mine = np.abs(b - a @ xk).max() / (np.abs(a).sum(axis=1).max() * np.abs(xk).max() + np.abs(b).max())
        want = np.empty(n)
        reference.sci_ref_solve_f64(a.ctypes.data, b.ctypes.data, want.ctypes.data, n, 1)
        return mine <= 1e-14 and berr[k] <= 1e-14 and 1 <= its[k] <= 30, \
            np.abs(xk - want).max() <= 1e-10 * np.abs(want).max()

    checks = [check(k) for k in range(count)]  # one at a time, as above
    assert all(c[0] for c in checks), [k for k, c in enumerate(checks) if not c[0]][:10]
    assert all(c[1] for c in checks), [k for k, c in enumerate(checks) if not c[1]][:10]

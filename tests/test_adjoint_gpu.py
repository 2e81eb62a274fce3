"""Adjoints of linear::product and linear::solve on the device (new; no reference pins).

product: dL/dleft = G right^T and dL/dright = left^T G, checked against FP64 products with the
error bounds of each product mode (tests/test_product_gpu.py) and against libsci's own CPU product
of the transposed operands.
solve: for X = A^-1 B, dL/dB = lambda = A^-T G and dL/dA = -lambda X^T, checked against FP64 numpy
and against central differences of L = sum(G * solve(A, B)) through libsci's own CPU solve<double>.
Refined solves reach a backward error <= 1e-14 in both the forward and the transposed system, so
their gradients match FP64 to 1e-10 relative (normwise) on these well-conditioned systems.
"""
import numpy as np
import pytest

from tests import _oracle
from tests.test_product_gpu import BF16, FP32, NAMES, SPLIT, SPLIT3, bound

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(128, 96, 64), (129, 70, 257), (300, 200, 500), (1, 1, 1)])
@pytest.mark.parametrize("mode", [BF16, SPLIT, SPLIT3, FP32], ids=NAMES.get)
def test_product_gradient(device, mode, shape):
    m, n, k = shape
    rng = np.random.default_rng(m + 3 * n + 7 * k)
    a = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    b = rng.uniform(-1, 1, (k, n)).astype(np.float32)
    g = rng.uniform(-1, 1, (m, n)).astype(np.float32)
    da, db = device.product_gradient(device.array(a.ravel()), device.array(b.ravel()), device.array(g.ravel()), m, n, k,
                                     mode=mode)
    da, db = da.numpy().reshape(m, k), db.numpy().reshape(k, n)
    a64, b64, g64 = a.astype(np.float64), b.astype(np.float64), g.astype(np.float64)
    assert np.all(np.abs(da - g64 @ b64.T) <= bound(mode, n, np.abs(g64) @ np.abs(b64).T))
    assert np.all(np.abs(db - a64.T @ g64) <= bound(mode, m, np.abs(a64).T @ np.abs(g64)))


def test_product_gradient_matches_the_reference_product(device, reference):
    """FP32 mode against libsci's CPU multiply of the explicitly transposed operands."""
    m, n, k = 64, 48, 80
    rng = np.random.default_rng(9)
    a = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    b = rng.uniform(-1, 1, (k, n)).astype(np.float32)
    g = rng.uniform(-1, 1, (m, n)).astype(np.float32)
    da, db = device.product_gradient(device.array(a.ravel()), device.array(b.ravel()), device.array(g.ravel()), m, n, k,
                                     mode=FP32)
    for got, left, right, rows, cols, inner in ((da, g, np.ascontiguousarray(b.T), m, k, n),
                                               (db, np.ascontiguousarray(a.T), g, k, n, m)):
        want = np.empty((rows, cols), np.float32)
        reference.sci_ref_product(0, left.ctypes.data, right.ctypes.data, want.ctypes.data, rows, cols, inner)
        s = np.abs(left.astype(np.float64)) @ np.abs(right.astype(np.float64))
        assert np.all(np.abs(got.numpy().reshape(rows, cols) - want) <= 2 * inner * 2.0 ** -23 * s + 1e-30)


def test_double_product_gradient(device):
    rng = np.random.default_rng(10)
    a, b, g = rng.standard_normal((40, 30)), rng.standard_normal((30, 20)), rng.standard_normal((40, 20))
    da, db = device.product_gradient(device.array(a.ravel()), device.array(b.ravel()), device.array(g.ravel()), 40, 20, 30)
    np.testing.assert_allclose(da.numpy().reshape(40, 30), g @ b.T, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(db.numpy().reshape(30, 20), a.T @ g, rtol=1e-12, atol=1e-12)


def solve_case(n, width, shift, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + (n * np.eye(n) if shift else 0.0)
    b = rng.standard_normal((n, width))
    g = rng.standard_normal((n, width))
    return a, b, g


def fp64_adjoint(a, b, g):
    x = np.linalg.solve(a, b)
    lam = np.linalg.solve(a.T, g)
    return x, -lam @ x.T, lam


def normwise(got, want):
    return np.abs(got - want).max() / np.abs(want).max()


@pytest.mark.parametrize("n,width,shift", [(512, 64, True), (300, 5, False), (1000, 16, True), (129, 33, False)])
def test_refined_solve_gradient(device, n, width, shift):
    a, b, g = solve_case(n, width, shift, seed=n + width)
    x, dA, dB, berr, iterations = device.solve_gradient(device.array(a.ravel()), device.array(b.ravel()),
                                                        device.array(g.ravel()), n, width, refine=True)
    want_x, want_dA, want_dB = fp64_adjoint(a, b, g)
    assert berr <= 1e-14 and iterations >= 2
    assert normwise(x.numpy().reshape(n, width), want_x) <= 1e-10
    assert normwise(dB.numpy().reshape(n, width), want_dB) <= 1e-10
    assert normwise(dA.numpy().reshape(n, n), want_dA) <= 1e-10


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-9), (np.float32, 2e-3)])
def test_plain_solve_gradient(device, dtype, tol):
    n, width = 257, 7
    a, b, g = solve_case(n, width, True, seed=21)
    a, b, g = a.astype(dtype), b.astype(dtype), g.astype(dtype)
    x, dA, dB, _, _ = device.solve_gradient(device.array(a.ravel()), device.array(b.ravel()), device.array(g.ravel()), n,
                                            width)
    want_x, want_dA, want_dB = fp64_adjoint(*(v.astype(np.float64) for v in (a, b, g)))
    assert normwise(x.numpy().reshape(n, width), want_x) <= tol
    assert normwise(dB.numpy().reshape(n, width), want_dB) <= tol
    assert normwise(dA.numpy().reshape(n, n), want_dA) <= tol


def test_solve_gradient_against_central_differences(device, reference):
    """L = sum(G * solve(A, B)); d L / d A[i, j] and d L / d B[i, c] by central differences through
    libsci's own CPU solve<double> (factor + substitute, solve.hpp:60-76) on 24 seeded coordinates."""
    n, width = 96, 4
    a, b, g = solve_case(n, width, True, seed=5)
    _, dA, dB, _, _ = device.solve_gradient(device.array(a.ravel()), device.array(b.ravel()), device.array(g.ravel()), n,
                                            width, refine=True)
    dA, dB = dA.numpy().reshape(n, n), dB.numpy().reshape(n, width)

    def loss(mat, rhs):
        out = np.empty((n, width))
        reference.sci_ref_solve_f64(np.ascontiguousarray(mat).ctypes.data, np.ascontiguousarray(rhs).ctypes.data,
                                    out.ctypes.data, n, width)
        return float(np.sum(g * out))

    rng = np.random.default_rng(6)
    for _ in range(12):
        i, j = rng.integers(n), rng.integers(n)
        h = 1e-4 * max(1.0, abs(a[i, j]))
        ap, am = a.copy(), a.copy()
        ap[i, j] += h
        am[i, j] -= h
        fd = (loss(ap, b) - loss(am, b)) / (ap[i, j] - am[i, j])
        assert abs(dA[i, j] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(dA).max())
    for _ in range(12):
        i, c = rng.integers(n), rng.integers(width)
        h = 1e-4 * max(1.0, abs(b[i, c]))
        bp, bm = b.copy(), b.copy()
        bp[i, c] += h
        bm[i, c] -= h
        fd = (loss(a, bp) - loss(a, bm)) / (bp[i, c] - bm[i, c])
        assert abs(dB[i, c] - fd) <= 1e-6 * max(abs(fd), 1e-3 * np.abs(dB).max())

"""linear::factor and linear::solve on the device, against libsci's own CPU factor and FP64.

Pins restated from the reference: a 3 x 3 matrix with a zero first pivot factors with rows
[1, 2, 0] and P A = L U (tests/linear/test_decompose.cpp:21-36); a 3 x 3 SPD system is solved for
one and two right-hand sides within 1e-9 (tests/linear/test_solve.cpp:8-25). Beyond them:
- pivot sequences equal the reference's factor<T> (oracle/_ref) on seeded matrices, in FP64 and in
  plain FP32; with the tensor-core trailing update (split-bf16, about 16 bits per product) they
  agree on at least 99% of positions, and P A = L U holds to 1e-4 relative;
- FP32 LU + FP64 refinement reaches a normwise backward error <= 1e-14 for A = G + n I and A = G.
"""
import ctypes

import numpy as np
import pytest

from tests import _oracle

pytestmark = pytest.mark.gpu


def reference_factor(reference, a):
    m = np.ascontiguousarray(a.copy())
    rows = np.zeros(m.shape[0], np.uint64)
    fn = reference.sci_ref_factor_f64 if m.dtype == np.float64 else reference.sci_ref_factor_f32
    fn(m.ctypes.data, rows.ctypes.data, m.shape[0])
    return m, rows


def device_factor(device, a, plain=False):
    d = device.array(a.ravel())
    rows = device.factor(d, a.shape[0], plain=plain)
    return d.numpy().reshape(a.shape), rows


def reconstruction_error(a, lu, rows):
    n = a.shape[0]
    lower = np.tril(lu.astype(np.float64), -1) + np.eye(n)
    upper = np.triu(lu.astype(np.float64))
    return np.abs(a.astype(np.float64)[rows.astype(np.int64)] - lower @ upper).max() / np.abs(a).max()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_zero_first_pivot(device, dtype):
    a = np.array([[0, 2, 1], [4, 1, 3], [2, 5, 7]], dtype)
    lu, rows = device_factor(device, a)
    assert list(rows) == [1, 2, 0]
    assert reconstruction_error(a, lu, rows) < 1e-6


def test_solve_pins(device):
    a = np.array([[4, -2, 1], [-2, 4, -2], [1, -2, 4]], np.float64)
    for b in (np.array([11, -16, 17], np.float64).reshape(3, 1), np.array([[11, 1], [-16, 0], [17, 2]], np.float64)):
        x, _, _ = device.solve(device.array(a.ravel()), device.array(b.ravel()), 3, b.shape[1])
        assert np.all(np.abs(a @ x.numpy().reshape(b.shape) - b) < 1e-9)


@pytest.mark.parametrize("n", [1, 2, 17, 64, 100, 257, 512, 1000, 1500])
@pytest.mark.parametrize("kind", ["f64", "f32_plain"])
def test_pivots_match_the_reference(device, reference, n, kind):
    dtype = np.float64 if kind == "f64" else np.float32
    a = np.random.default_rng(n).standard_normal((n, n)).astype(dtype)
    want_lu, want_rows = reference_factor(reference, a)
    lu, rows = device_factor(device, a, plain=(kind == "f32_plain"))
    assert np.array_equal(rows, want_rows)
    tol = 1e-12 if dtype == np.float64 else 1e-4
    assert reconstruction_error(a, lu, rows) < tol * n
    assert np.abs(lu - want_lu).max() <= (1e-9 if dtype == np.float64 else 1e-2) * max(1.0, np.abs(want_lu).max())


@pytest.mark.parametrize("n", [300, 1000, 2048])
def test_tensor_core_factor(device, reference, n):
    """Split-bf16 trailing updates carry about 16 bits per product: P A = L U to ~1e-6 n relative.
    Pivot sequences are compared on tie-free input: a row-shuffled diagonally dominant matrix, whose
    every column has one entry far above the rest, so rounding cannot reorder the candidates."""
    rng = np.random.default_rng(7 + n)
    a = rng.standard_normal((n, n)).astype(np.float32)
    lu, rows = device_factor(device, a)
    assert reconstruction_error(a, lu, rows) < 1e-6 * n
    shuffled = (rng.standard_normal((n, n)) + 4 * n * np.eye(n))[rng.permutation(n)].astype(np.float32)
    _, want_rows = reference_factor(reference, shuffled)
    _, rows = device_factor(device, shuffled)
    assert np.array_equal(rows, want_rows)


def test_diagonally_dominant_does_not_pivot(device):
    n = 1024
    a = (np.random.default_rng(3).standard_normal((n, n)) + n * np.eye(n)).astype(np.float32)
    _, rows = device_factor(device, a)
    assert np.array_equal(rows, np.arange(n))


@pytest.mark.parametrize("n,shift", [(1000, True), (1000, False), (2048, True), (2048, False)])
def test_refined_solve(device, n, shift):
    rng = np.random.default_rng(n + int(shift))
    a = rng.standard_normal((n, n)) + (n * np.eye(n) if shift else 0.0)
    b = rng.standard_normal((n, 16))
    x, berr, iterations = device.solve(device.array(a.ravel()), device.array(b.ravel()), n, 16, refine=True)
    x = x.numpy().reshape(n, 16)
    assert berr <= 1e-14
    assert 1 <= iterations <= 30
    r = b - a @ x
    mine = np.abs(r).max(axis=0) / (np.abs(a).sum(axis=1).max() * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))
    assert mine.max() <= 2e-14
    plain, plain_berr, _ = device.solve(device.array(a.ravel()), device.array(b.ravel()), n, 16, refine=False)
    assert plain_berr <= 1e-14
    assert np.abs(plain.numpy().reshape(n, 16) - x).max() <= 1e-9 * np.abs(x).max() * (1 if shift else 1e3)


@pytest.mark.parametrize("n", [130, 600])
def test_refined_solve_at_unaligned_addresses(device, n):
    """Systems packed one after another in one buffer (as a caller batching them keeps them) start
    on 8-byte boundaries only: the refined solve reads A, b and writes x at such addresses, for an
    order without (130) and with (600) the look-ahead's second stream."""
    from libsci_b200.native import SolveReport, check, lib

    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + n * np.eye(n)
    b = rng.standard_normal((n, 2))
    flat_a = device.array(np.concatenate([[0.0], a.ravel()]))
    flat_b = device.array(np.concatenate([[0.0], b.ravel()]))
    flat_x = device.array(np.zeros(2 * n + 1))
    assert flat_a.pointer % 16 == 0  # so A itself sits 8 bytes past a 16-byte boundary
    report = SolveReport()
    check(lib.sci_cuda_solve(device.handle, 1, 1, flat_a.pointer + 8, flat_b.pointer + 8, flat_x.pointer + 8, n, 2,
                             ctypes.byref(report)), device.handle)
    x = flat_x.numpy()[1:].reshape(n, 2)
    assert report.backward_error <= 1e-14
    r = b - a @ x
    mine = np.abs(r).max(axis=0) / (np.abs(a).sum(axis=1).max() * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))
    assert mine.max() <= 2e-14


def test_float_solve_without_refinement(device):
    n = 500
    rng = np.random.default_rng(1)
    a = (rng.standard_normal((n, n)) + n * np.eye(n)).astype(np.float32)
    b = rng.standard_normal((n, 3)).astype(np.float32)
    x, _, _ = device.solve(device.array(a.ravel()), device.array(b.ravel()), n, 3)
    want = np.linalg.solve(a.astype(np.float64), b.astype(np.float64))
    assert np.abs(x.numpy().reshape(n, 3) - want).max() <= 1e-5 * np.abs(want).max()


@pytest.mark.parametrize("width", [1, 8, 20, 64])
def test_float_solve_column_groups(device, width):
    """The substitution sweeps take the right-hand sides in column groups of 8 or 16 (a partial last
    group zero-filled): every group's columns match FP64 at FP32 accuracy."""
    n = 1024
    rng = np.random.default_rng(width)
    a = (rng.standard_normal((n, n)) + n * np.eye(n)).astype(np.float32)
    b = rng.standard_normal((n, width)).astype(np.float32)
    x, _, _ = device.solve(device.array(a.ravel()), device.array(b.ravel()), n, width)
    want = np.linalg.solve(a.astype(np.float64), b.astype(np.float64))
    assert np.abs(x.numpy().reshape(n, width) - want).max() <= 1e-5 * np.abs(want).max()

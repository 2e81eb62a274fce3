"""decompose and transpose on the device.

decompose (include/linear/decompose.hpp:77-103) against the reference's own factor (oracle/_ref,
linear::factor, the same split done here in numpy): the plain factorisation follows the reference's
pivot order step for step, so P is identical on these tie-free inputs, L and U agree to the
precision's tolerance, and P L U reproduces A. transpose (include/operations/manipulations.hpp:33-62)
against numpy.transpose, which it is named after: a copy, so bit for bit, ranks 1 to 4."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def reference_factors(reference, a, dtype):
    n = a.shape[0]
    packed = np.array(a, dtype, copy=True)  # factor works in place
    rows = np.zeros(n, np.uint64)
    fn = reference.sci_ref_factor_f64 if dtype == np.float64 else reference.sci_ref_factor_f32
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
    fn(packed.ctypes.data, rows.ctypes.data, n)
    lower = np.tril(packed, -1) + np.eye(n, dtype=dtype)
    upper = np.triu(packed)
    permutation = np.zeros((n, n), dtype)
    permutation[rows.astype(np.int64), np.arange(n)] = 1
    return permutation, lower, upper


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n", [5, 64, 257])
def test_decompose_matches_the_reference(device, reference, dtype, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)).astype(dtype)
    p, l, u = device.decompose(device.array(a.ravel()), n, plain=True)
    p, l, u = (m.numpy().reshape(n, n) for m in (p, l, u))
    rp, rl, ru = reference_factors(reference, a, dtype)
    assert np.array_equal(p, rp)
    tol = 1e-4 if dtype == np.float32 else 1e-11
    assert np.abs(l - rl).max() <= tol * n and np.abs(u - ru).max() <= tol * n * np.abs(ru).max()
    assert np.array_equal(np.triu(l, 1), np.zeros_like(l)) and np.array_equal(np.diag(l), np.ones(n, dtype))
    assert np.array_equal(np.tril(u, -1), np.zeros_like(u))
    residual = np.abs(p.astype(np.float64) @ l.astype(np.float64) @ u.astype(np.float64) - a).max() / np.abs(a).max()
    assert residual <= (1e-5 if dtype == np.float32 else 1e-13) * n


def test_decompose_tensor_mode_reconstructs(device):
    n = 1024
    a = (np.random.default_rng(3).standard_normal((n, n)) + n * np.eye(n)).astype(np.float32)
    p, l, u = (m.numpy().reshape(n, n).astype(np.float64) for m in device.decompose(device.array(a.ravel()), n))
    assert np.abs(p @ l @ u - a).max() / np.abs(a).max() <= 1e-5


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", [(17,), (1000, 777), (3, 4099), (7, 5, 3), (2, 3, 4, 5), (64, 1, 33)])
def test_transpose_matches_numpy(device, dtype, shape):
    x = np.random.default_rng(len(shape)).standard_normal(shape).astype(dtype)
    got = device.transpose(device.array(x.ravel()), shape).numpy()
    assert np.array_equal(got, np.ascontiguousarray(np.transpose(x)).ravel())


def test_manipulate_rejects_bad_arguments(device):
    from libsci_b200.native import lib

    x = device.array(np.ones(12, np.float32))
    shape = (ctypes.c_uint64 * 9)(*([1] * 9))
    assert lib.sci_cuda_transpose(device.handle, 0, x.pointer, 9, shape, device.empty(12).pointer) != 0  # rank 9
    assert lib.sci_cuda_transpose(device.handle, 0, x.pointer, 2, (ctypes.c_uint64 * 2)(3, 4), x.pointer) != 0  # in place
    with pytest.raises(ValueError):
        device.transpose(x, (5, 5))
    assert lib.sci_cuda_decompose(device.handle, 0, 0, None, None, None, None, 4) != 0

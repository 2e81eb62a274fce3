"""Broadcasting, the roadmap's elementwise functions and axis reductions on the device
(sci_cuda_broadcast, sci_cuda_reduce_axis) against numpy, whose rules they follow.

libsci lists these as next (README.md:149-152) and has no implementation to pin them to, so the
checker is numpy: bit for bit for add / subtract / multiply / divide / minimum / maximum / floor /
ceil / round / clip / where and for minimum / maximum along an axis; power within 1 ulp of
numpy's (glibc's) float powf and 3 ulp of its double pow; sums and means along an axis within the
bounds of a double-precision fold (float: at most 1 ulp from the correctly rounded sum).
"""
import ctypes
import math

import numpy as np
import pytest

from libsci_b200 import chunk as C
from libsci_b200 import device as D
from libsci_b200.native import SciCudaError, lib
from tests import _oracle

pytestmark = pytest.mark.gpu

PAIRS = [((3, 1), (1, 4)), ((5, 4, 3), (3,)), ((2, 1, 7), (6, 1)), ((1,), (1000,)), ((4097, 1), (1, 4099)),
         ((300,), ()), ((2, 3, 1, 5), (3, 4, 1)), ((2, 1, 2, 1, 2, 1, 2, 3), (1, 2, 1, 2, 1, 2, 1, 3)),
         ((64, 1000), (64, 1000)), ((7, 1, 513), (1, 9, 513)), ((5, 1, 1024), (1, 3, 1024)), ((16, 2048), (16, 1)),
         ((4096, 1), ())]
# the last axis decides the kernel: a whole number of 16-byte vectors (1000, 1024, 2048 ...) takes
# the vector form, 4099 / 513 / 1025 the element-wise rows, 1 / 3 / 4 / 7 the flat form
BINARY = {"add": np.add, "subtract": np.subtract, "multiply": np.multiply, "divide": np.divide,
          "minimum": np.minimum, "maximum": np.maximum}


def values(shape, dtype, rng, specials=True):
    data = rng.standard_normal(int(np.prod(shape, dtype=np.int64))).astype(dtype) * dtype(3)
    if specials and data.size >= 16:
        picks = rng.choice(data.size, size=min(data.size // 8, 64), replace=False)
        pool = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 1.0, -1.0, 0.5, -0.5, 2.5], dtype)
        data[picks] = pool[rng.integers(0, pool.size, picks.size)]
    return data.reshape(shape)


def same_bits(got, want):
    """Bit for bit, NaN by position: the GPU's float operations return the canonical NaN where
    numpy carries an operand's payload (as the chunk tests compare NaNs)."""
    got, want = np.ascontiguousarray(got).ravel(), np.ascontiguousarray(want).ravel()
    nan = np.isnan(want)
    if not np.array_equal(np.isnan(got), nan):
        return False
    unsigned = np.uint32 if got.dtype == np.float32 else np.uint64
    return np.array_equal(got[~nan].view(unsigned), want[~nan].view(unsigned))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_broadcast_binary_ops_match_numpy_bit_for_bit(device, dtype):
    rng = np.random.default_rng(1)
    with np.errstate(all="ignore"):
        for left_shape, right_shape in PAIRS:
            left, right = values(left_shape, dtype, rng), values(right_shape, dtype, rng)
            a, b = device.array(left.ravel()), device.array(right.ravel())
            for name, fn in BINARY.items():
                out, shape = device.broadcast(name, [(a, left_shape), (b, right_shape)])
                want = fn(left, right)
                assert shape == want.shape, (name, left_shape, right_shape)
                assert same_bits(out.numpy().reshape(shape), want), (name, left_shape, right_shape)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_floor_ceil_round_clip_where(device, dtype):
    rng = np.random.default_rng(2)
    x = values((257, 129), dtype, rng)
    x.ravel()[:8] = np.array([0.5, 1.5, 2.5, -0.5, -1.5, -2.5, -0.4, 0.49999997], dtype)
    a = device.array(x.ravel())
    for name, fn in (("floor", np.floor), ("ceil", np.ceil), ("round", np.round)):
        out, shape = getattr(D, name)((a, x.shape))
        assert same_bits(out.numpy().reshape(shape), fn(x)), name
        even = x[:256, :128].copy()  # a vector-form shape
        out, shape = getattr(D, name)((device.array(even.ravel()), even.shape))
        assert same_bits(out.numpy().reshape(shape), fn(even)), name
    lower, upper = values((1, 129), dtype, rng, specials=False) - 1, values((257, 1), dtype, rng, specials=False) + 1
    lo, hi = device.array(lower.ravel()), device.array(upper.ravel())
    out, shape = D.clip((a, x.shape), (lo, lower.shape), (hi, upper.shape))
    with np.errstate(all="ignore"):
        assert same_bits(out.numpy().reshape(shape), np.clip(x, lower, upper))
    out, shape = D.clip((a, x.shape), -1.25, 0.75)  # scalar bounds
    assert same_bits(out.numpy().reshape(shape), np.clip(x, dtype(-1.25), dtype(0.75)))
    condition = np.where(rng.random((257, 1)) < 0.5, 0.0, rng.standard_normal((257, 1))).astype(dtype)
    condition[3, 0] = np.nan  # NaN is true
    other = values((129,), dtype, rng)
    c, o = device.array(condition.ravel()), device.array(other)
    out, shape = D.where((c, condition.shape), (a, x.shape), (o, other.shape))
    assert same_bits(out.numpy().reshape(shape), np.where(condition != 0, x, other))


def ulps(got, want):
    return _oracle.ulp_distance(np.ascontiguousarray(got).ravel(), np.ascontiguousarray(want).ravel())


# float: a double pow rounded once to float, against glibc's powf; double: CUDA's pow (at most 2
# ulp) against glibc's pow (under 1 ulp), so up to 3 apart
@pytest.mark.parametrize("dtype,bound", [(np.float32, 1), (np.float64, 3)])
def test_power_within_ulps_of_numpy(device, dtype, bound):
    rng = np.random.default_rng(3)
    base = np.concatenate([rng.uniform(0, 10, 20000), rng.uniform(-10, 0, 2000), [0.0, -0.0, 1.0, -1.0, np.inf,
                                                                                  -np.inf, np.nan, 2.0, 0.5]])
    base = base.astype(dtype).reshape(-1, 1)
    exponent = np.array([0.0, 1.0, 2.0, 3.0, -1.0, -2.0, 0.5, -0.5, 1.0 / 3.0, 7.25, -13.5, 40.0, np.nan, np.inf,
                         -np.inf], dtype)
    b, e = device.array(base.ravel()), device.array(exponent)
    out, shape = D.power((b, base.shape), (e, exponent.shape))
    got = out.numpy().reshape(shape)
    with np.errstate(all="ignore"):
        want = np.power(base, exponent)
    nan = np.isnan(want)
    assert np.array_equal(np.isnan(got), nan)
    assert np.all(ulps(got[~nan], want[~nan]) <= bound), np.max(ulps(got[~nan], want[~nan]))


AXES = [((7, 5000), 0), ((7, 5000), 1), ((3, 4, 5), 0), ((3, 4, 5), 1), ((3, 4, 5), 2), ((1 << 20,), 0),
        ((2, 3_000_001), 1), ((1000, 3), 1), ((4096, 4096), 0), ((4096, 4096), 1), ((9, 1, 11), 1), ((5, 130, 33), 1)]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_axis_reductions_against_numpy(device, dtype):
    rng = np.random.default_rng(4)
    for shape, axis in AXES:
        data = rng.standard_normal(shape).astype(dtype)
        array = device.array(data.ravel())
        exact = np.sum(data.astype(np.longdouble), axis=axis)
        magnitude = np.sum(np.abs(data.astype(np.float64)), axis=axis)
        for fold, fn in ((C.MINIMUM, np.min), (C.MAXIMUM, np.max)):
            out, kept = device.reduce_axis(array, shape, axis, fold)
            assert kept == fn(data, axis=axis).shape and same_bits(out.numpy().reshape(kept), fn(data, axis=axis))
        out, kept = device.reduce_axis(array, shape, axis, C.SUM)
        got = out.numpy().reshape(kept)
        if dtype == np.float32:
            assert np.all(ulps(got, exact.astype(np.float32)) <= 1), (shape, axis)
        else:
            n = shape[axis]
            assert np.all(np.abs(got - exact.astype(np.float64)) <= n * 2.0 ** -52 * magnitude + 1e-300), (shape, axis)
        out, kept = device.reduce_axis(array, shape, axis, C.AXIS_MEAN)
        mean = out.numpy().reshape(kept)
        want = (exact.astype(dtype) / dtype(shape[axis])).astype(dtype)
        if dtype == np.float32:
            assert np.all(ulps(mean, want) <= 2), (shape, axis)
        else:
            assert np.allclose(mean, want, rtol=0, atol=float(np.max(magnitude)) * 1e-13 / shape[axis] + 1e-300)


def test_axis_reductions_propagate_nan_and_handle_empty_axes(device):
    data = np.arange(60, dtype=np.float32).reshape(3, 4, 5)
    data[1, 2, 3] = np.nan
    array = device.array(data.ravel())
    for fold, fn in ((C.SUM, np.sum), (C.MINIMUM, np.min), (C.MAXIMUM, np.max)):
        for axis in range(3):
            out, kept = device.reduce_axis(array, data.shape, axis, fold)
            assert np.array_equal(np.isnan(out.numpy().reshape(kept)), np.isnan(fn(data, axis=axis))), (fold, axis)
    empty = device.empty(0, np.float32)
    out, kept = device.reduce_axis(empty, (5, 0, 3), 1, C.SUM)
    assert kept == (5, 3) and np.array_equal(out.numpy(), np.zeros(15, np.float32))
    out, _ = device.reduce_axis(empty, (5, 0, 3), 1, C.MAXIMUM)
    assert np.all(np.isnan(out.numpy()))
    out, _ = device.reduce_axis(empty, (5, 0, 3), 1, C.AXIS_MEAN)
    assert np.array_equal(out.numpy(), np.zeros(15, np.float32))


def test_broadcast_to_and_shape_errors(device):
    row = np.arange(5, dtype=np.float64)
    row[0] = -0.0
    a = device.array(row)
    out, shape = D.broadcast_to((a, (5,)), (3, 5))
    assert shape == (3, 5) and same_bits(out.numpy().reshape(shape), np.broadcast_to(row, (3, 5)))
    with pytest.raises(ValueError):
        device.broadcast("add", [(a, (5,)), (a, (5, 1)), (device.array(np.zeros(4)), (4,))])
    # the C ABI checks extents itself
    inputs = (ctypes.c_void_p * 2)(a.pointer, a.pointer)
    extents = (ctypes.c_uint64 * 4)(1, 5, 1, 4)
    out_extents = (ctypes.c_uint64 * 2)(3, 5)
    target = device.empty(15, np.float64)
    status = lib.sci_cuda_broadcast(device.handle, 1, C.CODE["add"], 2, out_extents, 2, inputs, extents, target.pointer)
    assert status != 0
    status = lib.sci_cuda_broadcast(device.handle, 1, C.CODE["add"], 2, out_extents, 3, inputs, extents, target.pointer)
    assert status != 0  # add takes two operands
    with pytest.raises(SciCudaError):
        device.reduce_axis(a, (5,), 0, 7)
    assert math.isnan(float(D.maximum_axis((device.array(np.array([1.0, np.nan])), (2,)), 0)[0].numpy()[0]))

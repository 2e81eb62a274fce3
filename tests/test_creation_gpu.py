"""Arrays made on the device (include/operations/creation.hpp through sci_cuda_fill / linspace /
range / eye / grid) against the oracle's restatement, which test_oracle.py pins to the reference's
own creation functions: bit for bit, in float and double, at sizes past 2^24 (where a float index
stops being exact) and at the edges the reference handles (no values, one value, a step that
overshoots, a descending range)."""
import numpy as np
import pytest

from tests import _oracle
from tests.test_oracle import LINSPACES, RANGES, creation_functions

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def made(oracle):
    return creation_functions(oracle, "sci_oracle")


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_full_zeros_ones(device, made, dtype):
    precision = 1 if dtype == np.float64 else 0
    for count in (1, 1003, (1 << 24) + 5):
        for value in (0.0, 1.0, 2.5, -0.0, float("nan"), 1e40):
            got = device.full(count, value, dtype).numpy()
            want = np.empty(count, dtype)
            made["fill"](precision, want.ctypes.data, count, value)
            assert _oracle.mismatches(got, want).size == 0, (count, value)
    assert np.array_equal(device.zeros(77, dtype).numpy(), np.zeros(77, dtype))
    assert np.array_equal(device.ones(77, dtype).numpy(), np.ones(77, dtype))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_linspace_and_range(device, made, dtype):
    precision = 1 if dtype == np.float64 else 0
    for start, stop, count in LINSPACES + [(-1.0, 3.0, (1 << 25) + 7)]:
        got = device.linspace(start, stop, count, dtype).numpy()
        want = np.empty(max(count, 1), dtype)
        made["linspace"](precision, want.ctypes.data, count, start, stop)
        assert got.size == count and _oracle.mismatches(got, want[:count]).size == 0, (start, stop, count)
    for start, stop, step in RANGES:
        got = device.range(start, stop, step, dtype).numpy()
        count = made["range_count"](precision, start, stop, step)
        want = np.empty(max(count, 1), dtype)
        made["range"](precision, want.ctypes.data, count, start, step)
        assert got.size == count and _oracle.mismatches(got, want[:count]).size == 0, (start, stop, step)
    assert np.array_equal(device.range(5, dtype=dtype).numpy(), np.arange(5, dtype=dtype))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_eye_and_grid(device, made, dtype):
    for rows, columns in ((3, 3), (4, 7), (7, 4), (1, 1), (4099, 4097)):
        got = device.eye(rows, columns, dtype).numpy().reshape(rows, columns)
        assert np.array_equal(got, np.eye(rows, columns, dtype=dtype)), (rows, columns)
    x = np.linspace(-1, 1, 1001).astype(dtype)
    y = np.linspace(0, 5, 333).astype(dtype)
    xx, yy = device.grid(device.array(x), device.array(y))
    gx, gy = np.meshgrid(x, y)
    assert np.array_equal(xx.numpy().reshape(333, 1001), gx) and np.array_equal(yy.numpy().reshape(333, 1001), gy)


def test_creation_rejects_bad_arguments(device):
    from libsci_b200.native import lib

    host = np.empty(4, np.float32)
    assert lib.sci_cuda_fill(device.handle, 7, device.empty(4).pointer, 4, 1.0) != 0       # unknown precision
    assert lib.sci_cuda_fill(device.handle, 0, host.ctypes.data, 4, 1.0) != 0              # host memory
    assert lib.sci_cuda_eye(device.handle, 0, None, 3, 3) != 0                              # no output
    with pytest.raises(TypeError):
        device.grid(device.array(np.ones(3, np.float32)), device.array(np.ones(3, np.float64)))
    assert lib.sci_cuda_fill(device.handle, 0, None, 0, 1.0) == 0                           # nothing to make

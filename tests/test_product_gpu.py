"""linear::product on the device, every mode, against an FP64 product of the same float inputs.

Bounds, with S = |A| @ |B| (elementwise absolute values) and k the depth:
- FP32 SIMT: |C - C64| <= k 2^-23 S (k roundings of a float accumulator);
- BF16 tensor cores: <= (2^-7 + k 2^-22) S (each operand rounded to 8 bits);
- split BF16: <= (2^-14 + k 2^-22) S (hi + lo keeps about 16 bits per operand; lo*lo dropped);
- three-term split BF16: <= (2^-21 + k 2^-22) S (hi + mid + lo, six products);
- FP64: <= k 2^-51 S.
The reference pins its product at 37 x 53 x 29 with patterned values within 1e-3 of a double
loop (tests/linear/test_product.cpp:8-33); that case is exact in every mode here.
"""
import numpy as np
import pytest

from tests import _oracle

pytestmark = pytest.mark.gpu

BF16, SPLIT, FP32, SPLIT3 = 0, 1, 2, 3
NAMES = {BF16: "bf16", SPLIT: "split_bf16", FP32: "fp32", SPLIT3: "split3_bf16"}


def bound(mode, k, s, wide=False):
    if wide:
        return k * 2.0 ** -51 * s + 1e-300
    return {FP32: k * 2.0 ** -23, BF16: 2.0 ** -7 + k * 2.0 ** -22, SPLIT: 2.0 ** -14 + k * 2.0 ** -22,
            SPLIT3: 2.0 ** -21 + k * 2.0 ** -22}[mode] * s + 1e-30


def run(device, a, b, mode):
    m, k = a.shape
    n = b.shape[1]
    da, db = device.array(a.ravel()), device.array(b.ravel())
    out = device.product(da, db, m, n, k, mode=mode)
    return out.numpy().reshape(m, n)


@pytest.mark.parametrize("mode", [BF16, SPLIT, SPLIT3, FP32], ids=NAMES.get)
def test_reference_pin(device, mode):
    rows, inner, columns = 37, 53, 29
    left = np.fromfunction(lambda r, c: ((r * 7 + c * 3) % 11) - 5.0, (rows, inner)).astype(np.float32)
    right = np.fromfunction(lambda r, c: ((r * 5 + c) % 13) * 0.25, (inner, columns)).astype(np.float32)
    got = run(device, left, right, mode)
    want = left.astype(np.float64) @ right.astype(np.float64)
    assert np.all(np.abs(got - want) < 1e-3)


@pytest.mark.parametrize("shape", [(128, 256, 64), (129, 257, 70), (300, 500, 200), (64, 8, 1000), (1024, 1024, 1024),
                                   (1, 1, 1), (700, 9, 3)])
@pytest.mark.parametrize("mode", [BF16, SPLIT, SPLIT3, FP32], ids=NAMES.get)
def test_product_against_fp64(device, mode, shape):
    m, n, k = shape
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    a = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    b = rng.uniform(-1, 1, (k, n)).astype(np.float32)
    got = run(device, a, b, mode)
    a64, b64 = a.astype(np.float64), b.astype(np.float64)
    want = a64 @ b64
    s = np.abs(a64) @ np.abs(b64)
    assert np.all(np.abs(got - want) <= bound(mode, k, s))


def test_split_is_more_accurate_than_bf16(device):
    rng = np.random.default_rng(3)
    a = rng.uniform(-1, 1, (512, 768)).astype(np.float32)
    b = rng.uniform(-1, 1, (768, 384)).astype(np.float32)
    want = a.astype(np.float64) @ b.astype(np.float64)
    plain = np.abs(run(device, a, b, BF16) - want).max()
    split = np.abs(run(device, a, b, SPLIT) - want).max()
    assert split < plain / 50


def test_large_product_rows_against_the_oracle(device, oracle):
    """4096^3 in split mode: 64 seeded rows checked against the oracle's FP64 rows."""
    m = n = k = 4096
    rng = np.random.default_rng(11)
    a = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    b = rng.uniform(-1, 1, (k, n)).astype(np.float32)
    got = run(device, a, b, SPLIT)
    rows = np.sort(rng.choice(m, 64, replace=False))
    for r in rows:
        want = np.zeros(n, np.float64)
        oracle.sci_oracle_product_rows(a.ctypes.data, b.ctypes.data, want.ctypes.data, m, n, k, int(r), int(r) + 1)
        s = np.abs(a[r].astype(np.float64)) @ np.abs(b.astype(np.float64))
        assert np.all(np.abs(got[r] - want) <= bound(SPLIT, k, s))


def test_double_product_and_empty_depth(device):
    rng = np.random.default_rng(5)
    a = rng.standard_normal((77, 131))
    b = rng.standard_normal((131, 45))
    got = run(device, a, b, FP32)
    want = a @ b
    s = np.abs(a) @ np.abs(b)
    assert np.all(np.abs(got - want) <= bound(FP32, 131, s, wide=True))
    da, db = device.array(np.ones(6, np.float32)), device.array(np.ones(6, np.float32))
    out = device.array(np.full(6, 7.0, np.float32))
    device.product(da, db, 2, 3, 0, mode=BF16, out=out)
    assert np.array_equal(out.numpy(), np.zeros(6, np.float32))

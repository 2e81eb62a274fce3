"""Batched small solves on the device (new; no reference batch API).

Every system is also solvable by libsci's own CPU solve<double> (include/linear/solve.hpp:60-76,
oracle/_ref): the batch's FP32 LU + FP64 refinement must reach a normwise backward error of at most
1e-14 (checked here in numpy) and agree with the reference's solution to 1e-10 relative on these
well-conditioned systems.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EDGES = [1, 2, 7, 8, 31, 32, 33, 63, 64, 65, 127, 128, 129, 207, 208, 209, 255, 256]


def systems(count, seed, shift=True):
    rng = np.random.default_rng(seed)
    orders = np.concatenate([EDGES, rng.integers(8, 257, count - len(EDGES))]).astype(np.int64)
    mats, rhs = [], []
    for n in orders:
        a = rng.standard_normal((n, n))
        if shift:
            a += n * np.eye(n)
        mats.append(a)
        rhs.append(rng.standard_normal(n))
    return orders, mats, rhs


def run(device, orders, mats, rhs, launches=1):
    da = [device.array(m.ravel()) for m in mats]
    db = [device.array(b) for b in rhs]
    dx = [device.empty(len(b), np.float64) for b in rhs]
    errors = device.empty(len(orders), np.float64)
    iterations = device.empty(len(orders), np.int32)
    batch = device.solve_batch(orders, [a.pointer for a in da], [b.pointer for b in db], [x.pointer for x in dx],
                               errors, iterations)
    for _ in range(launches):
        batch.launch()
    out = [x.numpy() for x in dx], errors.numpy(), iterations.numpy(), batch.shapes()
    batch.close()
    return out


def backward_error(a, b, x):
    return np.abs(b - a @ x).max() / (np.abs(a).sum(axis=1).max() * np.abs(x).max() + np.abs(b).max())


@pytest.mark.parametrize("shift", [True, False], ids=["G+nI", "G"])
def test_batched_solves(device, reference, shift):
    orders, mats, rhs = systems(160 if shift else 60, seed=1 + int(shift), shift=shift)
    xs, errors, iterations, shapes = run(device, orders, mats, rhs, launches=2)
    assert all(t in (0, 32, 64, 128, 256, 512) for t in shapes)
    for k, (a, b, x) in enumerate(zip(mats, rhs, xs)):
        mine = backward_error(a, b, x)
        assert mine <= 1e-14, (k, orders[k], mine)
        assert errors[k] <= 1e-14 and 1 <= iterations[k] <= 30, (k, errors[k], iterations[k])
        if k % 7 == 0:
            want = np.empty(len(b))
            reference.sci_ref_solve_f64(np.ascontiguousarray(a).ctypes.data, np.ascontiguousarray(b).ctypes.data,
                                        want.ctypes.data, len(b), 1)
            assert np.abs(x - want).max() <= 1e-10 * np.abs(want).max(), k


def test_replay_is_deterministic_and_singular_systems_report(device):
    orders, mats, rhs = systems(40, seed=9)
    mats[5] = np.zeros_like(mats[5])  # singular: zero pivots are skipped, the solution is not finite
    first = run(device, orders, mats, rhs)
    second = run(device, orders, mats, rhs, launches=3)
    for k in range(len(orders)):
        if k == 5:
            assert not np.isfinite(first[1][k]) or first[1][k] > 1e-3
            continue
        assert np.array_equal(first[0][k], second[0][k])
        assert first[1][k] <= 1e-14


def test_invalid_solve_batches(device):
    import ctypes

    from libsci_b200.native import SolveItems, lib

    orders = np.array([300], np.uint32)  # above 256
    table = np.zeros(1, np.uint64)
    items = SolveItems(1, orders.ctypes.data, table.ctypes.data, table.ctypes.data, table.ctypes.data, None, None)
    handle = ctypes.c_void_p()
    assert lib.sci_cuda_solve_batch_create(device.handle, ctypes.byref(items), ctypes.byref(handle)) != 0
    assert lib.sci_cuda_solve_batch_launch(None) != 0

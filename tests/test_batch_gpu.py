"""Batched launches on the device (new; no reference batch API, so no reference pins).

The oracle is libsci's own CPU path run item by item (what a reference user writes: one assign and
one reduce per instance). Stored outputs must be bit-identical to it; reduced results must match the
double sum of its per-element values to 1e-6 of the sum of their magnitudes (the batch folds eight
lanes in the element type before switching to double, like the single-chunk reduction).
"""
import ctypes
import os
import tempfile
from pathlib import Path

import numpy as np
import pytest

from libsci_b200 import chunk as C
from tests import _oracle

pytestmark = pytest.mark.gpu

# The tuning cache of this test process: read once, at the first batch the library creates.
CACHE = Path(tempfile.mkdtemp()) / "tune.txt"
os.environ["SCI_CUDA_TUNE_CACHE"] = str(CACHE)


def store_and_reduce(precision=C.SINGLE, reduce_code=C.CODE["tanh"]):
    """t = a*b + c stored, tanh(t) reduced: fuse(in0, in1, in2) -> T0; copy(T0) -> out; tanh(T0) -> T1."""
    chunk = C.Chunk(precision)
    chunk.arguments = 3
    chunk.temporaries = 2
    chunk.length = 3
    for index, (code, target, sources) in enumerate(((C.CODE["fuse"], C.TEMPORARY | 0, (0, 1, 2)),
                                                     (C.CODE["copy"], C.OUTPUT, (C.TEMPORARY | 0, C.NONE, C.NONE)),
                                                     (reduce_code, C.TEMPORARY | 1, (C.TEMPORARY | 0, C.NONE, C.NONE)))):
        ins = chunk.instructions[index]
        ins.code, ins.target = code, target
        ins.sources[0], ins.sources[1], ins.sources[2] = sources
    chunk.result = C.TEMPORARY | 1
    return chunk


def lengths(items, seed, low=1, high=200_000):
    rng = np.random.default_rng(seed)
    out = np.exp(rng.uniform(np.log(low), np.log(high), items)).astype(np.int64)
    out[:9] = [0, 1, 15, 16, 17, 255, 256, 257, 4096]
    return out


class Items:
    """Per-item inputs carved from three device buffers (with a one-element shift on every
    third item, so unaligned items take the element-wise path)."""

    def __init__(self, device, counts, dtype, seed):
        self.counts = counts
        rng = np.random.default_rng(seed)
        shift = (np.arange(len(counts)) % 3 == 2).astype(np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(counts + shift + 8)])[:-1] + shift
        total = int(self.offsets[-1] + counts[-1] + 8)
        self.host = [rng.standard_normal(total).astype(dtype) for _ in range(3)]
        self.arrays = [device.array(h) for h in self.host]
        self.out = device.empty(total, dtype)
        size = np.dtype(dtype).itemsize
        self.pointers = np.array([[a.pointer + int(o) * size for a in self.arrays] for o in self.offsets], np.uint64)
        self.outputs = np.array([self.out.pointer + int(o) * size for o in self.offsets], np.uint64)

    def item(self, k):
        o, n = int(self.offsets[k]), int(self.counts[k])
        return [h[o:o + n] for h in self.host]


def oracle_item(reference, a, b, c, reduce_name="tanh"):
    """libsci's CPU path on one item: t = a*b + c (assign), then the values of reduce_name(t)."""
    n = len(a)
    refs = [C.Reference(x.ctypes.data, n, x.dtype) for x in (a, b, c)]
    t = _oracle.execute(reference, C.record_output(refs[0] * refs[1] + refs[2]), n, a.dtype)
    tr = C.Reference(t.ctypes.data, n, a.dtype)
    values = _oracle.execute(reference, C.record_output(C.unary(reduce_name, tr)), n, a.dtype)
    return t, values


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_store_and_reduce_batch(device, reference, dtype):
    counts = lengths(300, seed=1 if dtype == np.float32 else 2)
    items = Items(device, counts, dtype, seed=3)
    results = device.empty(len(counts), np.float64)
    chunk = store_and_reduce(C.WIDE if dtype == np.float64 else C.SINGLE)
    batch = device.batch(chunk, C.SUM, items.pointers, counts, items.outputs, results)
    batch.launch()
    spans, specialized = batch.spans()
    assert specialized and all(s in (256, 1024, 4096, 16384, 65536) for s in spans)
    first = results.numpy()
    out = items.out.numpy()
    batch.launch()
    assert np.array_equal(results.numpy(), first)  # deterministic per item
    for k in range(len(counts)):
        a, b, c = items.item(k)
        t, values = oracle_item(reference, a, b, c)
        o, n = int(items.offsets[k]), int(counts[k])
        assert _oracle.mismatches(out[o:o + n], t).size == 0, k
        want = float(np.sum(values.astype(np.float64)))
        assert abs(first[k] - want) <= 1e-6 * float(np.sum(np.abs(values.astype(np.float64)))) + 1e-12, k
    batch.close()


def test_extreme_folds_and_nan(device, reference):
    counts = lengths(64, seed=4, high=20_000)
    items = Items(device, counts, np.float32, seed=5)
    o = int(items.offsets[20])
    items.host[2][o + 3] = np.nan  # one NaN in item 20's c
    items.arrays[2].upload(items.host[2])
    for fold, pick in ((C.MAXIMUM, np.max), (C.MINIMUM, np.min)):
        results = device.empty(len(counts), np.float64)
        batch = device.batch(store_and_reduce(reduce_code=C.CODE["sin"]), fold, items.pointers, counts, items.outputs,
                             results)
        batch.launch()
        got = results.numpy()
        for k in range(len(counts)):
            _, values = oracle_item(reference, *items.item(k), reduce_name="sin")
            if counts[k] == 0 or np.isnan(values).any():
                assert np.isnan(got[k]), k  # empty extremes and NaN items are NaN
            else:
                assert got[k] == float(pick(values)), k
        batch.close()


def test_store_only_and_tuning_cache(device, reference):
    """A batch without results stores only; the tuner's choices land in the cache file and a second
    batch of the same chunk and buckets reads them instead of tuning again."""
    counts = lengths(40, seed=6, high=100_000)
    items = Items(device, counts, np.float32, seed=7)
    x = [C.Reference(0x1000 * (i + 1), 16, np.float32) for i in range(3)]
    chunk = C.record_output(x[0] * x[1] + x[2])
    batch = device.batch(chunk, C.SUM, items.pointers, counts, items.outputs, None)
    batch.launch()
    out = items.out.numpy()
    for k in (0, 5, 17, 39):
        t, _ = oracle_item(reference, *items.item(k))
        o, n = int(items.offsets[k]), int(counts[k])
        assert _oracle.mismatches(out[o:o + n], t).size == 0
    spans, _ = batch.spans()
    batch.close()
    lines = CACHE.read_text().splitlines()
    assert len(lines) >= 3
    again = device.batch(chunk, C.SUM, items.pointers, counts, items.outputs, None)
    assert again.spans()[0] == spans
    assert CACHE.read_text().splitlines() == lines
    again.close()


def test_invalid_batches(device):
    from libsci_b200.native import BatchItems, lib

    chunk = store_and_reduce()
    handle = ctypes.c_void_p()
    counts = np.array([4], np.uint64)
    pointers = np.zeros((1, 3), np.uint64)  # null inputs
    items = BatchItems(1, pointers.ctypes.data, None, counts.ctypes.data, None)
    assert lib.sci_cuda_batch_create(device.handle, ctypes.byref(chunk), C.SUM, ctypes.byref(items), ctypes.byref(handle)) != 0
    assert lib.sci_cuda_batch_create(device.handle, ctypes.byref(chunk), 7, ctypes.byref(items), ctypes.byref(handle)) != 0
    assert lib.sci_cuda_batch_launch(None) != 0

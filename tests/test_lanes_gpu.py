"""Copy lanes (sci_cuda_upload_lane / download_lane / join): pieces of three arrays go up on the
upload lane, a chunk runs over each piece on the main stream, and the results come back on the
download lane, all queued before one wait. The outputs equal the single-pass result bit for bit,
and a piece's kernel never runs before its upload nor its download before its kernel."""
import ctypes

import numpy as np
import pytest

from libsci_b200 import chunk as C
from libsci_b200.native import check, lib

pytestmark = pytest.mark.gpu


def test_pieces_through_the_lanes_match_one_pass(device):
    import torch

    n, pieces = 1 << 22, 8
    span = n // pieces
    rng = np.random.default_rng(17)
    hosts = [torch.from_numpy(rng.standard_normal(n).astype(np.float32)).pin_memory() for _ in range(3)]
    back = torch.empty(n, dtype=torch.float32).pin_memory()
    x, y, z = (device.empty(n, np.float32) for _ in range(3))
    out = device.empty(n, np.float32)
    partial = device.empty(pieces, np.float64)
    for p in range(pieces):
        o = p * span
        for host, dev in zip(hosts, (x, y, z)):
            check(lib.sci_cuda_upload_lane(device.handle, dev.pointer + 4 * o, host.data_ptr() + 4 * o, 4 * span),
                  device.handle)
        a, b, c = (v.offset(o, span).expression() for v in (x, y, z))
        device.execute(C.record_output(a * b + C.unary("sin", c)), out.pointer + 4 * o, span)
        device.reduce_async(C.record_reduce(a * c), C.SUM, span, partial.pointer + 8 * p)
        check(lib.sci_cuda_download_lane(device.handle, back.data_ptr() + 4 * o, out.pointer + 4 * o, 4 * span),
              device.handle)
    check(lib.sci_cuda_join(device.handle), device.handle)
    device.synchronize()

    a, b, c = (v.expression() for v in (x, y, z))
    whole = device.evaluate(a * b + C.unary("sin", c)).numpy()
    assert np.array_equal(back.numpy().view(np.uint32), whole.view(np.uint32))
    total = device.reduce_chunk(C.record_reduce(a * c), C.SUM, n)
    assert abs(partial.numpy().sum() - total) <= 1e-12 * np.abs(hosts[0].numpy().astype(np.float64)
                                                            * hosts[2].numpy()).sum()

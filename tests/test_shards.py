"""The N > 1 path's only exchange (libsci_b200/shards.py), on CPU: two gloo ranks, each folding its
own shard, must give the single-device fold of the whole array, NaN winning as in
core::Accumulator (include/core/bytecode/accumulator.hpp:28-34)."""
import datetime
import os
import socket

import numpy as np
import torch.multiprocessing as mp

SUM, MINIMUM, MAXIMUM = 0, 1, 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fold(x, kind):
    if np.isnan(x).any():
        return float("nan")
    return float({SUM: np.sum, MINIMUM: np.min, MAXIMUM: np.max}[kind](x.astype(np.float64)))


def _rank(rank, world, port, shards, kinds, queue):
    import torch
    import torch.distributed as dist

    from libsci_b200.shards import combine

    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local = torch.tensor([_fold(x, k) for x, k in zip(shards[rank], kinds)], dtype=torch.float64)
        queue.put((rank, combine(local, kinds).tolist()))
    finally:
        dist.destroy_process_group()


def run(shards, kinds, world=2):
    context = mp.get_context("spawn")
    queue = context.Queue()
    port = _free_port()
    procs = [context.Process(target=_rank, args=(r, world, port, shards, kinds, queue)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(queue.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0] == out[1] or (np.isnan(out[0]).tolist() == np.isnan(out[1]).tolist())
    return out[0]


def test_two_ranks_fold_like_one_device():
    rng = np.random.default_rng(0)
    whole = [rng.standard_normal(1000).astype(np.float32) for _ in range(3)]
    kinds = (SUM, MAXIMUM, MINIMUM)
    shards = [[w[:600] for w in whole], [w[600:] for w in whole]]
    got = run(shards, kinds)
    want = [_fold(w, k) for w, k in zip(whole, kinds)]
    np.testing.assert_allclose(got, want, rtol=1e-12)


def test_a_nan_on_one_rank_wins():
    rng = np.random.default_rng(1)
    whole = [rng.standard_normal(64).astype(np.float32) for _ in range(3)]
    whole[1][50] = np.nan  # on rank 1 only
    kinds = (SUM, MAXIMUM, MINIMUM)
    shards = [[w[:32] for w in whole], [w[32:] for w in whole]]
    got = run(shards, kinds)
    assert not np.isnan(got[0]) and np.isnan(got[1]) and not np.isnan(got[2])
    assert abs(got[0] - _fold(whole[0], SUM)) <= 1e-12 * abs(got[0]) + 1e-12

"""Multi-process paths on CPU (gloo): replica throughput aggregation and tempering decisions
across ranks.  The hot path itself does not shard (one lattice per GPU); only scalars move."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from lettuce_b200 import replicas  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _potential(q):
    return 2.0 * np.cos(q) + 0.3 * q * q


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # replica throughput: rank r did (r + 1) * 100 units in (10 + r) ms
        value, ms = replicas.job_rate((rank + 1) * 100.0, 10.0 + rank, dist)
        # tempering: stream r has charge q_r and scale s_r
        q, s = replicas.gather_streams(0.7 * rank - 1.0, 1.0 - rank / max(world - 1, 1), dist)
        from lettuce_b200.tempering import swap_decisions
        rng = np.random.default_rng(1234)          # shared seed: every rank draws the same numbers
        scales = s
        history = []
        for sweep in range(6):
            u = rng.random(world)
            scales, acc = swap_decisions(q, scales, _potential, sweep % 2, u)
            history.append(tuple(scales))
        out[rank] = (value, ms, tuple(q), history)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_replicas_and_tempering_across_ranks(world):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    results = [out[r] for r in range(world)]
    total = sum((r + 1) * 100.0 for r in range(world))
    for value, ms, q, history in results:
        assert ms == pytest.approx(10.0 + world - 1)
        assert value == pytest.approx(total / ((10.0 + world - 1) / 1000.0))
    # every rank reached the same decisions, and they match a single-process run
    assert all(r[3] == results[0][3] for r in results)
    from lettuce_b200.tempering import swap_decisions
    q = list(results[0][2])
    scales = [1.0 - r / max(world - 1, 1) for r in range(world)]
    rng = np.random.default_rng(1234)
    for sweep in range(6):
        scales, _ = swap_decisions(q, scales, _potential, sweep % 2, rng.random(world))
        assert tuple(scales) == results[0][3][sweep]
        assert sorted(scales) == sorted(1.0 - r / max(world - 1, 1) for r in range(world))


def test_swap_rule_matches_reference_two_streams():
    """s_a = 0 (plain stream), s_b = 1 (biased): dE = V(Q_a) - V(Q_b), the reference's
    dV = V(CV_new) - V(CV_old) (updates/tempering.hpp:57-60)."""
    from lettuce_b200.tempering import swap_decisions
    q = [0.5, 1.5]
    dV = _potential(0.5) - _potential(1.5)
    u_accept, u_reject = 0.999 * np.exp(-dV), 1.001 * np.exp(-dV)
    s, acc = swap_decisions(q, [0.0, 1.0], _potential, 0, [min(u_accept, 0.999999), 0])
    assert acc == [0] and s == [1.0, 0.0]
    if u_reject < 1.0:
        s, acc = swap_decisions(q, [0.0, 1.0], _potential, 0, [u_reject, 0])
        assert acc == [] and s == [0.0, 1.0]

"""Host logic of the multi-GPU replicas, on CPU: draw sharding, the LPT partition
and the per-step reduction across two gloo ranks (the same collectives bench.py
issues over NCCL)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import rans_uq_b200.replicas as rp


def test_shard_ids_disjoint():
    a, b = rp.shard_ids(0, 2, 5), rp.shard_ids(1, 2, 5)
    assert list(a) == [0, 1, 2, 3, 4] and list(b) == [5, 6, 7, 8, 9]
    with pytest.raises(ValueError):
        rp.shard_ids(2, 2, 5)


def test_partition_lpt_covers_and_balances():
    rng = np.random.default_rng(3)
    # the channel ensemble's classes: cells x reference iterations per class
    cls = np.arange(256) % 3
    cost = np.array([384 * 12460, 768 * 58690, 1536 * 258900])[cls] * rng.uniform(0.9, 1.1, 256)
    for world in (1, 2, 3, 8):
        parts = rp.partition_lpt(cost, world)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(256))
        loads = [cost[p].sum() for p in parts]
        # LPT bound: max load <= mean + the largest single cost
        assert max(loads) <= np.mean(loads) + cost.max() + 1e-6


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [120.0, 250.5][rank]
        conv = [85, 84][rank]
        ll = np.arange(3 + rank, dtype=np.float64) + 10 * rank
        out = rp.reduce_step(ms, conv, ll)
        # the timed-step plan: every rank must reach the same count of timed steps
        import bench

        est = rp.reduce_max([148.0, 151.0][rank])
        elapsed = rp.reduce_max([400.0, 420.0][rank])
        k = bench.plan_timed_steps(20, elapsed, est, 1400.0)
        e2e = rp.reduce_count([80, 81][rank])
        q.put((rank, out[0], out[1], out[2].tolist(), k, e2e))
    finally:
        dist.destroy_process_group()


def bench_plan(*a):
    import bench

    return bench.plan_timed_steps(*a)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_reduce_step_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, conv, ll, k, e2e in res:
        assert ms == 250.5 and conv == 169
        assert ll == [0.0, 1.0, 2.0, 10.0, 11.0, 12.0, 13.0]
        assert k == bench_plan(20, 420.0, 151.0, 1400.0) and e2e == 161


def _reference_weights(ll):
    """cfdr.statistics.posterior_weights' rule on the host: exp(l - max) / fsum."""
    import math

    m = max(ll)
    w = [math.exp(v - m) for v in ll]
    s = math.fsum(w)
    return np.asarray(w) / s, m + math.log(s)


def _reference_parts(ll):
    import math

    m = max(ll)
    w = [math.exp(v - m) for v in ll]
    s = math.fsum(w)
    return np.asarray(w) / s, m, s


def _weights_worker(rank, world, port, q, parts):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # the per-rank step is the device kernel on a GPU; the host rule stands in here
        w, g = rp.sharded_posterior_weights(parts[rank],
                                            local=lambda ll, lq: _reference_parts(list(ll)))
        q.put((rank, w.tolist(), g))
    finally:
        dist.destroy_process_group()


def test_sharded_posterior_weights_two_gloo_ranks():
    """Two ranks holding 70 and 30 draws normalise their own weights with one MAX and one
    SUM all-reduce: the concatenation equals the single-process weights and the log
    evidence agrees. The tolerance is the rounding of l - max itself: a shard subtracts
    its own maximum, so exp sees an argument rounded differently by up to an ulp of
    |l| (4 ulp of the largest |l| here, relative)."""
    rng = np.random.default_rng(5)
    ll = -0.5 * rng.chisquare(30, 100) * 12.0
    parts = [ll[:70], ll[70:]]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_weights_worker, args=(r, 2, port, q, parts)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want, g_ref = _reference_weights(list(ll))
    got = np.concatenate([np.asarray(r[1]) for r in res])
    rtol = 4 * np.max(np.abs(ll)) * np.finfo(float).eps
    np.testing.assert_allclose(got, want, rtol=rtol, atol=0)
    assert abs(got.sum() - 1.0) < 1e-14
    for r in res:
        assert abs(r[2] - g_ref) <= 1e-14 * abs(g_ref)

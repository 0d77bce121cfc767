"""Multi-rank SMC exchange (particle sharding) on CPU with gloo, world size 2."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from smccat import distributed as sd
from smccat import workload


def test_systematic_resample_matches_reference_walk():
    rng = np.random.default_rng(0)
    for n in (1, 5, 64):
        w = rng.random(n)
        w /= w.sum()
        u = rng.random()
        a = sd.systematic_resample(w, u)
        # each index appears floor/ceil of n * w_i times and the output is sorted
        assert np.all(np.diff(a) >= 0)
        counts = np.bincount(a, minlength=n)
        assert np.all(np.abs(counts - n * w) <= 1.0 + 1e-9)


def test_next_step_matches_oracle():
    rng = np.random.default_rng(1)
    lnl = rng.normal(size=40) * 30 - 500
    raw = np.full(40, -np.log(40))
    w, nw, ess, temp = sd.next_step(raw, lnl, 24.0, 0.0)
    rw, onw, oess, otemp = oracle.next_step(raw, lnl, 24.0, 0.0)
    assert temp == otemp
    np.testing.assert_allclose(nw, onw, rtol=1e-12)
    assert ess == pytest.approx(oess, rel=1e-12)


def test_pack_roundtrip():
    cfg = workload.CONFIGS[1]
    st = workload.make_particles(cfg, 3, np.random.default_rng(2), kmax=4)
    packed = sd.pack_states(st, cfg.T, cfg.S, 4)
    back = sd.unpack_states(packed, cfg.T, cfg.S, 4)
    for k in sd.STATE_KEYS:
        np.testing.assert_array_equal(np.asarray(back[k]).reshape(np.asarray(st[k]).shape), st[k])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, assign, per_rank, width, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # global particle g carries the value g in every field
        local = np.tile(np.arange(rank * per_rank, (rank + 1) * per_rank, dtype=np.float64)[:, None],
                        (1, width))
        lnl = np.arange(rank * per_rank, (rank + 1) * per_rank, dtype=np.float64) * -1.0
        gathered = sd.all_gather_lnl(lnl)
        out = sd.exchange_states(local, np.asarray(assign))
        q.put((rank, gathered.tolist(), out[:, 0].tolist(), bool(np.all(out == out[:, :1]))))
    finally:
        dist.destroy_process_group()


def test_two_rank_exchange_with_gloo():
    world, per_rank, width = 2, 5, 7
    rng = np.random.default_rng(3)
    w = rng.random(world * per_rank) ** 4
    w /= w.sum()
    assign = sd.systematic_resample(w, 0.37).tolist()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, assign, per_rank, width, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, g, vals, uniform = q.get(timeout=120)
        res[r] = (g, vals, uniform)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        g, vals, uniform = res[r]
        assert g == [-float(i) for i in range(world * per_rank)]
        assert uniform
        # destination slot d of rank r now holds the state of particle assign[d]
        assert vals == [float(assign[r * per_rank + i]) for i in range(per_rank)]


def test_oracle_resampling_agrees_with_the_distributed_module():
    """Both restate main.cpp:178-192; uniform weights keep every particle once,
    a point mass copies one particle everywhere."""
    from oracle import tuning
    from smccat import distributed
    rng = np.random.default_rng(2)
    for _ in range(20):
        n = int(rng.integers(1, 40))
        w = rng.random(n)
        w /= w.sum()
        u = float(rng.random())
        assert list(distributed.systematic_resample(w, u)) == tuning.systematic_resample(w, u)
    assert tuning.systematic_resample(np.full(8, 1 / 8), 0.5) == list(range(8))
    assert tuning.systematic_resample(np.eye(5)[3], 0.2) == [3] * 5

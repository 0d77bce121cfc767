"""The sharded SMC loop (smccat.smc.run_sharded) with real engine states: two
ranks, each a process with its own engine context on the device, the
log-likelihood all-gather and the particle-state exchange over gloo. Both
ranks must see the same temperatures, resampling rounds and log Z, every
particle's log-likelihood must be the oracle's for the state it ends with, and
after the first resampling each rank's states must be exactly the ancestors
the global systematic walk picked."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

PER_RANK, WORLD = 6, 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _cfg():
    from smccat import workload
    return workload.WorkloadConfig("sharded", T=8, S=150, R=4, particles=PER_RANK * WORLD,
                                   iterations=2, lg=False, invar=False, cat=True,
                                   dp_concentration=2.0, k_range=(1, 3), seed=81)


def _worker(rank, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD,
                            timeout=datetime.timedelta(seconds=120))
    try:
        import smccat
        from smccat import distributed as sd
        from smccat import smc, workload
        cfg = _cfg()
        rng = np.random.default_rng(cfg.seed)
        codes, _ = workload.simulate_alignment(cfg, rng)
        st = workload.make_particles(cfg, cfg.particles, rng, kmax=12)
        sl = slice(rank * PER_RANK, (rank + 1) * PER_RANK)
        eng = smccat.Engine(codes, cfg.R, PER_RANK, max_classes=12, cat=True)
        eng.set_particles(0, st["parent"][sl], st["branch"][sl], st["base"][sl],
                          st["num_classes"][sl], st["logits"][sl], st["assign"][sl],
                          st["pinv"][sl], st["shape"][sl])
        eng.refresh(full=True)
        # One weight step by hand, with a resample forced: the exchanged
        # states must be the ancestors' exactly.
        n = cfg.particles
        raw = np.full(n, -np.log(n))
        w, temp, ess, res = sd.resample_engine(eng, raw, 0.99 * n, 0.0, 0.3)
        first = eng.get_particles()
        out = smc.run_sharded(eng, cat=True, iterations=cfg.iterations, seed=5, max_steps=6)
        fin = eng.get_particles()
        q.put((rank, {"temp": temp, "resampled": res, "first": {k: v.tolist() for k, v in first.items()},
                      "fin": {k: v.tolist() for k, v in fin.items()}, "lnl": eng.lnl().tolist(),
                      "out": out}))
        eng.close()
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_smc_with_engines():
    import oracle
    from smccat import distributed as sd
    from smccat import workload
    cfg = _cfg()
    rng = np.random.default_rng(cfg.seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng, kmax=12)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(WORLD):
        r, d = q.get(timeout=600)
        res[r] = d
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # The forced first step: the global ancestors, from the oracle's
    # likelihoods of the initial states.
    rates = np.stack([oracle.discretize_gamma(s, cfg.R) for s in st["shape"]])
    lnl0 = oracle.lnl_batch(codes, st["parent"], st["branch"], st["base"], st["num_classes"],
                            st["logits"], st["assign"], st["pinv"], rates)
    n = cfg.particles
    w, nw, ess, temp = sd.next_step(np.full(n, -np.log(n)), lnl0, 0.99 * n, 0.0)
    anc = sd.systematic_resample(nw, 0.3)
    for r in range(WORLD):
        d = res[r]
        assert d["resampled"] and d["temp"] == pytest.approx(temp, abs=1e-12)
        for i in range(PER_RANK):
            a = anc[r * PER_RANK + i]
            np.testing.assert_array_equal(d["first"]["parent"][i], st["parent"][a])
            np.testing.assert_allclose(d["first"]["branch"][i], st["branch"][a], rtol=0, atol=0)
            np.testing.assert_array_equal(d["first"]["assign"][i], st["assign"][a])
    # The loop: identical global quantities on both ranks, exact likelihoods.
    o0, o1 = res[0]["out"], res[1]["out"]
    assert o0["steps"] == o1["steps"] and o0["resamples"] == o1["resamples"]
    assert o0["log_z"] == pytest.approx(o1["log_z"], rel=1e-12)
    for r in range(WORLD):
        fin = {k: np.asarray(v) for k, v in res[r]["fin"].items()}
        for i in range(PER_RANK):
            K = int(fin["num_classes"][i])
            rr = oracle.discretize_gamma(fin["shape"][i], cfg.R)
            ref = oracle.lnl(codes, fin["parent"][i].astype(np.int32), fin["branch"][i], fin["base"][i],
                             fin["logits"][i][:K], fin["assign"][i].astype(np.int32), fin["pinv"][i], rr)
            assert res[r]["lnl"][i] == pytest.approx(ref, rel=1e-9)

"""The whole Mcmc::operator() sweep on the device (smccat_mcmc_sweep): the
reference's move registry (main.cpp:55-106) drawn per particle, tree and
parameter moves (Particle.cpp:677-783) proposed, evaluated and accepted on
the device, the sweep captured as one CUDA graph. Final states must carry
exact likelihoods and priors (against the oracle), graph and eager launches
must agree bit for bit, and the host path must continue from the synced
state."""
import numpy as np
import pytest

import oracle
import smccat
from smccat import workload

pytestmark = pytest.mark.gpu

CFGS = [
    workload.WorkloadConfig("sw_cat_i", T=8, S=120, R=4, particles=6, iterations=1, lg=False,
                            invar=True, cat=True, alpha=0.7, pinv=0.1, k_range=(1, 4), seed=201),
    workload.WorkloadConfig("sw_gtr_i", T=20, S=300, R=4, particles=10, iterations=1, lg=False,
                            invar=True, cat=False, alpha=0.5, pinv=0.1, seed=202),
    workload.WorkloadConfig("sw_lg_r1", T=7, S=90, R=1, particles=5, iterations=1, lg=True,
                            invar=False, cat=True, k_range=(2, 3), seed=203),
]


def engine(cfg, precision=smccat.PREC_FP64):
    rng = np.random.default_rng(cfg.seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng)
    st["pinv"] = np.where(cfg.invar, np.maximum(st["pinv"], 0.05), 0.0)
    eng = smccat.Engine(codes, cfg.R, cfg.particles, max_classes=st["logits"].shape[1], lg=cfg.lg,
                        invar=cfg.invar, cat=cfg.cat, precision=precision)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"], st["logits"],
                      st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    eng.compute_split_posteriors()
    return eng, codes, st


def check_exact(eng, codes, cfg, rtol=1e-9, atol=0.0):
    fin = eng.get_particles()
    got = eng.lnl()
    prior = eng.ln_prior()
    for i in range(cfg.particles):
        K = int(fin["num_classes"][i])
        rates = oracle.discretize_gamma(fin["shape"][i], cfg.R) if cfg.R > 1 else [1.0]
        ref = oracle.lnl(codes, fin["parent"][i], fin["branch"][i], fin["base"][i],
                         fin["logits"][i][:K], fin["assign"][i], fin["pinv"][i], rates)
        assert got[i] == pytest.approx(ref, rel=rtol, abs=atol), i
        counts = np.bincount(fin["assign"][i], minlength=K)
        rp = oracle.ln_prior(cfg.T, cfg.S, cfg.R, cfg.lg, fin["branch"][i], fin["shape"][i],
                             fin["base"][i], fin["logits"][i][:K], counts)
        assert prior[i] == pytest.approx(rp, rel=1e-12, abs=1e-9), i
    return fin


@pytest.mark.parametrize("cfg", CFGS, ids=lambda c: c.name)
def test_sweep_keeps_likelihoods_exact(cfg):
    eng, codes, st = engine(cfg)
    start = eng.get_particles()
    stats = eng.mcmc_sweep(iterations=4, temperature=0.7, seed=5)
    fin = check_exact(eng, codes, cfg)
    prop, acc = np.array(stats["proposed"]), np.array(stats["accepted"])
    assert np.all(acc <= prop) and prop.sum() > 0 and acc.sum() > 0
    assert prop.sum() <= cfg.particles * stats["lockstep_steps"]
    # Every registered family proposed something over the particles, and the
    # parameters it owns moved.
    assert prop[:5].sum() > 0                              # tree moves
    assert prop[7] > 0                                     # stationary
    if cfg.R > 1:
        assert prop[6] > 0
        if acc[6] > 0:
            assert np.any(fin["shape"] != start["shape"])
    if cfg.invar:
        assert prop[5] > 0
    if not cfg.lg:
        assert prop[8] + prop[9] > 0
    else:
        assert prop[8] + prop[9] == 0
        np.testing.assert_array_equal(fin["base"], start["base"])
    eng.close()


def test_graph_and_eager_launches_agree():
    cfg = CFGS[0]
    out = []
    for graph in (True, False):
        eng, codes, st = engine(cfg)
        s = eng.mcmc_sweep(iterations=3, temperature=0.9, seed=77, use_graph=graph)
        out.append((s, eng.get_particles(), eng.lnl()))
        eng.close()
    (s1, p1, l1), (s2, p2, l2) = out
    assert s1 == s2
    for k in p1:
        np.testing.assert_array_equal(p1[k], p2[k], err_msg=k)
    np.testing.assert_array_equal(l1, l2)


def test_host_path_continues_from_the_synced_state():
    cfg = CFGS[1]
    eng, codes, st = engine(cfg)
    eng.mcmc_sweep(iterations=3, temperature=1.0, seed=9)
    after = eng.lnl()
    eng.refresh(full=True)
    np.testing.assert_allclose(eng.lnl(), after, rtol=1e-12)
    eng.rejuvenate(iterations=2, temperature=1.0, seed=10)
    eng.mcmc_sweep(iterations=2, temperature=1.0, seed=11)
    check_exact(eng, codes, cfg)
    eng.close()


def test_mixed_precision_sweep():
    cfg = CFGS[1]
    eng, codes, st = engine(cfg, precision=smccat.PREC_FP32)
    eng.mcmc_sweep(iterations=3, temperature=1.0, seed=12)
    check_exact(eng, codes, cfg, rtol=0.0, atol=1e-3)
    eng.close()

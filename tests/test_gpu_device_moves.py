"""Tree rejuvenation (branch scale, subtree scale, NNI) with proposals, plans
and accept/reject on the device (smccat_branch_sweep), captured as one CUDA
graph: final likelihoods exact against the oracle, graph and eager launches
identical, host path consistent afterwards."""
import numpy as np
import pytest

import oracle
import smccat
from smccat import workload

pytestmark = pytest.mark.gpu

CFGS = [
    workload.WorkloadConfig("dm_cat", T=8, S=120, R=4, particles=6, iterations=1, lg=False,
                            invar=True, cat=True, alpha=0.7, pinv=0.1, k_range=(1, 4), seed=101),
    workload.WorkloadConfig("dm_gtr", T=20, S=300, R=4, particles=12, iterations=1, lg=False,
                            invar=True, cat=False, alpha=0.5, pinv=0.1, seed=33),
]


def engine(cfg, seed=None, precision=smccat.PREC_FP64):
    rng = np.random.default_rng(cfg.seed if seed is None else seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng)
    st["pinv"] = np.maximum(st["pinv"], 0.05)
    eng = smccat.Engine(codes, cfg.R, cfg.particles, max_classes=st["logits"].shape[1], lg=cfg.lg,
                        invar=cfg.invar, cat=cfg.cat, precision=precision)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    return eng, codes, st


def oracle_lnl(codes, cfg, s, i):
    K = int(s["num_classes"][i])
    rates = oracle.discretize_gamma(s["shape"][i], cfg.R)
    return oracle.lnl(codes, s["parent"][i], s["branch"][i], s["base"][i], s["logits"][i][:K],
                      s["assign"][i], s["pinv"][i], rates)


@pytest.mark.parametrize("cfg", CFGS, ids=lambda c: c.name)
def test_branch_sweep_keeps_exact_likelihoods(cfg):
    eng, codes, st = engine(cfg)
    before = eng.get_particles()
    stats = eng.branch_sweep(steps=25, temperature=0.7, seed=5)
    n = cfg.particles
    assert stats["branch_proposed"] + stats["subtree_proposed"] + stats["nni_proposed"] == 25 * n
    assert 0 < stats["branch_accepted"] <= stats["branch_proposed"]
    assert stats["subtree_accepted"] <= stats["subtree_proposed"]
    assert stats["nni_accepted"] <= stats["nni_proposed"]
    assert stats["nni_proposed"] > 0
    fin = eng.get_particles()
    assert np.any(fin["branch"] != before["branch"])
    got = eng.lnl()
    for i in range(n):
        assert got[i] == pytest.approx(oracle_lnl(codes, cfg, fin, i), rel=1e-9)
    # the host path continues from the synchronised state
    eng.rejuvenate(iterations=1, temperature=0.7, seed=9)
    fin2 = eng.get_particles()
    got2 = eng.lnl()
    for i in range(n):
        assert got2[i] == pytest.approx(oracle_lnl(codes, cfg, fin2, i), rel=1e-9)
    eng.close()


def _splits(parent, T):
    """Tip sets below every internal node, as frozensets."""
    N = len(parent)
    below = [{n} if n < T else set() for n in range(N)]
    changed = True
    while changed:
        changed = False
        for n in range(N):
            p = parent[n]
            if p >= 0 and not below[n] <= below[p]:
                below[p] |= below[n]
                changed = True
    return {frozenset(b) for n, b in enumerate(below) if n >= T}


@pytest.mark.parametrize("cfg", CFGS, ids=lambda c: c.name)
def test_nni_changes_topology_exactly(cfg):
    # At temperature 0 the target is the prior alone: every NNI (prior and
    # Hastings terms both zero) is accepted, so topologies must move.
    eng, codes, st = engine(cfg, seed=cfg.seed + 1)
    before = eng.get_particles()
    stats = eng.branch_sweep(steps=30, temperature=0.0, seed=12)
    assert stats["nni_proposed"] > 0
    assert stats["nni_accepted"] == stats["nni_proposed"]
    fin = eng.get_particles()
    moved = 0
    for i in range(cfg.particles):
        assert (fin["parent"][i] < 0).sum() == 1
        moved += _splits(fin["parent"][i], cfg.T) != _splits(before["parent"][i], cfg.T)
    assert moved > 0
    got = eng.lnl()
    for i in range(cfg.particles):
        assert got[i] == pytest.approx(oracle_lnl(codes, cfg, fin, i), rel=1e-9)
    # a full refresh of the synchronised trees reproduces the incremental values
    eng.refresh(full=True)
    np.testing.assert_allclose(eng.lnl(), got, rtol=1e-12, atol=0)
    eng.close()


def test_graph_and_eager_launches_agree():
    cfg = CFGS[1]
    a, _, _ = engine(cfg)
    b, _, _ = engine(cfg)
    sa = a.branch_sweep(steps=10, temperature=1.0, seed=77, use_graph=True)
    sb = b.branch_sweep(steps=10, temperature=1.0, seed=77, use_graph=False)
    assert sa == sb
    np.testing.assert_array_equal(a.get_particles()["branch"], b.get_particles()["branch"])
    np.testing.assert_array_equal(a.get_particles()["parent"], b.get_particles()["parent"])
    np.testing.assert_array_equal(a.lnl(), b.lnl())
    a.close()
    b.close()


def test_branch_sweep_fp32_matches_fp64_evaluation():
    cfg = CFGS[1]
    eng, codes, st = engine(cfg, precision=smccat.PREC_FP32)
    eng.branch_sweep(steps=10, temperature=1.0, seed=3)
    fin = eng.get_particles()
    got = eng.lnl()
    for i in range(cfg.particles):
        assert abs(got[i] - oracle_lnl(codes, cfg, fin, i)) < 3e-4
    eng.close()


def test_branch_sweep_refuses_uncommitted_edits():
    cfg = CFGS[0]
    eng, codes, st = engine(cfg)
    eng.set_pinv(0, 0.2)
    with pytest.raises(smccat.SmccatError) as e:
        eng.branch_sweep(steps=1, temperature=1.0, seed=1)
    assert e.value.code == smccat.ESTATE
    eng.close()

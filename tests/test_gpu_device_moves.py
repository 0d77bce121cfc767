"""Tree rejuvenation with the reference's whole treeMove mixture (NNI, adaptive
NNI, SPR, branch scale, subtree scale) proposed, planned and accepted on the
device (smccat_tree_sweep), captured as one CUDA graph: final likelihoods
exact against the oracle, graph and eager launches identical, the adaptive
NNI Hastings ratio driven by the installed split table, host path consistent
afterwards."""
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
KINDS = ("adaptive_nni", "nni", "spr", "branch", "subtree")


def engine(cfg, seed=None, precision=smccat.PREC_FP64, particles=None, parent=None):
    rng = np.random.default_rng(cfg.seed if seed is None else seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    n = particles or cfg.particles
    st = workload.make_particles(cfg, n, rng)
    st["pinv"] = np.maximum(st["pinv"], 0.05)
    if parent is not None:
        st["parent"] = np.tile(np.asarray(parent, np.int32), (n, 1))
    eng = smccat.Engine(codes, cfg.R, n, max_classes=st["logits"].shape[1], lg=cfg.lg,
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


def _clades(parent, T):
    """Tip sets below every node."""
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
    return below


def _splits(parent, T):
    return {frozenset(b) for n, b in enumerate(_clades(parent, T)) if n >= T}


def _canonical_bits(clade, T):
    s = set(clade) if 0 in clade else set(range(T)) - set(clade)
    w = [0, 0]
    for t in s:
        w[t >> 6] |= 1 << (t & 63)
    return w


@pytest.mark.parametrize("cfg", CFGS, ids=lambda c: c.name)
def test_tree_sweep_keeps_exact_likelihoods(cfg):
    eng, codes, st = engine(cfg)
    before = eng.get_particles()
    eng.compute_split_posteriors()  # a non-empty table for adaptive NNI
    stats = eng.tree_sweep(steps=25, temperature=0.7, seed=5)
    n = cfg.particles
    assert sum(stats[k + "_proposed"] for k in KINDS) == 25 * n
    for k in KINDS:
        assert stats[k + "_proposed"] > 0, k
        assert stats[k + "_accepted"] <= stats[k + "_proposed"]
    assert stats["branch_accepted"] > 0
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


@pytest.mark.parametrize("cfg", CFGS, ids=lambda c: c.name)
def test_topology_moves_at_temperature_zero(cfg):
    # At temperature 0 the target is the prior alone: NNI and SPR (prior and
    # Hastings terms both zero) are always accepted, so topologies must move;
    # with no split table adaptive NNI weighs every node alike and is too.
    eng, codes, st = engine(cfg, seed=cfg.seed + 1)
    before = eng.get_particles()
    stats = eng.tree_sweep(steps=30, temperature=0.0, seed=12)
    for k in ("nni", "spr", "adaptive_nni"):
        assert stats[k + "_proposed"] > 0
        assert stats[k + "_accepted"] == stats[k + "_proposed"], k
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


# Balanced 8-taxon tree ((0,1),(2,3)),((4,5),(6,7)): internal nodes 8..14, root 14.
BALANCED8 = [8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13, 14, 14, -1]


def test_adaptive_nni_hastings_follows_split_table():
    # Install every split one NNI away from the balanced tree with posterior 1
    # (and none of its own): every adaptive-NNI proposal then leaves a node of
    # weight 1 + eps for one of weight eps, log Hastings = log(eps / (tot - 1))
    # - log((1 + eps) / tot) ~ -4.4, so at temperature 0 almost all are
    # rejected. Without the table they are all accepted.
    cfg = CFGS[0]
    T = cfg.T
    clades = _clades(BALANCED8, T)
    kids = {}
    for n, p in enumerate(BALANCED8):
        if p >= 0:
            kids.setdefault(p, []).append(n)
    bits = []
    for x in range(T, 2 * T - 1):
        p = BALANCED8[x]
        if p < 0:
            continue
        sib = [c for c in kids[p] if c != x][0]
        for c in kids[x]:
            new = (clades[x] - clades[c]) | clades[sib]
            w = _canonical_bits(new, T)
            if w not in bits:
                bits.append(w)
    rates = {}
    for table in (False, True):
        eng, codes, st = engine(cfg, particles=64, parent=BALANCED8)
        if table:
            eng.set_split_posteriors(np.array(bits, np.uint64), np.ones(len(bits)))
        stats = eng.tree_sweep(steps=2, temperature=0.0, seed=21)
        assert stats["adaptive_nni_proposed"] > 15
        rates[table] = stats["adaptive_nni_accepted"] / stats["adaptive_nni_proposed"]
        fin = eng.get_particles()
        got = eng.lnl()
        for i in range(0, 64, 9):
            assert got[i] == pytest.approx(oracle_lnl(codes, cfg, fin, i), rel=1e-9)
        eng.close()
    assert rates[False] == 1.0
    assert rates[True] < 0.3


def test_graph_and_eager_launches_agree():
    cfg = CFGS[1]
    a, _, _ = engine(cfg)
    b, _, _ = engine(cfg)
    a.compute_split_posteriors()
    b.compute_split_posteriors()
    sa = a.tree_sweep(steps=10, temperature=1.0, seed=77, use_graph=True)
    sb = b.tree_sweep(steps=10, temperature=1.0, seed=77, use_graph=False)
    assert sa == sb
    np.testing.assert_array_equal(a.get_particles()["branch"], b.get_particles()["branch"])
    np.testing.assert_array_equal(a.get_particles()["parent"], b.get_particles()["parent"])
    np.testing.assert_array_equal(a.lnl(), b.lnl())
    a.close()
    b.close()


def test_tree_sweep_fp32_matches_fp64_evaluation():
    cfg = CFGS[1]
    eng, codes, st = engine(cfg, precision=smccat.PREC_FP32)
    eng.tree_sweep(steps=10, temperature=1.0, seed=3)
    fin = eng.get_particles()
    got = eng.lnl()
    for i in range(cfg.particles):
        assert abs(got[i] - oracle_lnl(codes, cfg, fin, i)) < 3e-4
    eng.close()


def test_tree_sweep_refuses_uncommitted_edits():
    cfg = CFGS[0]
    eng, codes, st = engine(cfg)
    eng.set_pinv(0, 0.2)
    with pytest.raises(smccat.SmccatError) as e:
        eng.tree_sweep(steps=1, temperature=1.0, seed=1)
    assert e.value.code == smccat.ESTATE
    eng.close()


def test_tree_sweep_on_three_taxa():
    # The smallest tree: one internal non-root node, so NNI and SPR have a
    # single admissible target node and a single regraft point.
    cfg = workload.WorkloadConfig("dm_t3", T=3, S=40, R=2, particles=4, iterations=1, lg=True,
                                  invar=False, cat=False, alpha=0.9, seed=2)
    eng, codes, st = engine(cfg)
    stats = eng.tree_sweep(steps=20, temperature=0.5, seed=3)
    assert sum(stats[k + "_proposed"] for k in KINDS) == 20 * cfg.particles
    fin = eng.get_particles()
    got = eng.lnl()
    for i in range(cfg.particles):
        assert (fin["parent"][i] < 0).sum() == 1
        assert got[i] == pytest.approx(oracle_lnl(codes, cfg, fin, i), rel=1e-9)
    eng.close()

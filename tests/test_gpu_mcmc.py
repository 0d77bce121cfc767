"""Rejuvenation moves, lnPrior, the lockstep MCMC driver and the SMC weight
step, through the C-ABI, against the oracle and against restatements of the
reference's move rules (Tree.cpp:553-812, Particle.cpp:677-783)."""
import numpy as np
import pytest
from scipy import stats

import oracle
import smccat
from smccat import workload

pytestmark = pytest.mark.gpu

CFG = workload.WorkloadConfig("mcmc_small", T=8, S=120, R=4, particles=6, iterations=3,
                              lg=False, invar=True, cat=True, alpha=0.7, pinv=0.1,
                              k_range=(1, 4), seed=101)


def engine(cfg=CFG, n=None, seed=None):
    n = cfg.particles if n is None else n
    rng = np.random.default_rng(cfg.seed if seed is None else seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, n, rng)
    st["pinv"] = np.maximum(st["pinv"], 0.05) if cfg.invar else st["pinv"]
    eng = smccat.Engine(codes, cfg.R, n, max_classes=st["logits"].shape[1], lg=cfg.lg,
                        invar=cfg.invar, cat=cfg.cat)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    return eng, codes, st


def oracle_lnl_state(codes, cfg, s, i):
    K = int(s["num_classes"][i])
    rates = oracle.discretize_gamma(s["shape"][i], cfg.R) if cfg.R > 1 else [1.0]
    return oracle.lnl(codes, s["parent"][i], s["branch"][i], s["base"][i], s["logits"][i][:K],
                      s["assign"][i], s["pinv"][i], rates)


def subtree(parent, x):
    out = {x}
    changed = True
    while changed:
        changed = False
        for n, p in enumerate(parent):
            if p in out and n not in out:
                out.add(n)
                changed = True
    return out


def test_ln_prior_matches_oracle():
    for cfg in (CFG, workload.WorkloadConfig("lg", T=6, S=50, R=1, particles=3, iterations=1,
                                             lg=True, invar=False, cat=False, seed=5)):
        eng, codes, st = engine(cfg)
        got = eng.ln_prior()
        for i in range(cfg.particles):
            K = int(st["num_classes"][i])
            counts = np.bincount(st["assign"][i], minlength=K)
            ref = oracle.ln_prior(cfg.T, cfg.S, cfg.R, cfg.lg, st["branch"][i], st["shape"][i],
                                  st["base"][i], st["logits"][i][:K], counts)
            assert got[i] == pytest.approx(ref, rel=1e-12)
        eng.close()


@pytest.mark.parametrize("seed", range(12))
def test_tree_proposals_follow_reference_rules(seed):
    eng, codes, st = engine()
    before = eng.get_particles()
    p = seed % CFG.particles
    kind, hastings = eng.propose(p, smccat.FAMILY_TREE, seed * 7919 + 3)
    after = eng.get_particles()
    par0, par1 = before["parent"][p], after["parent"][p]
    br0, br1 = before["branch"][p], after["branch"][p]
    oracle.postorder(par1)  # raises if not a rooted binary tree
    if kind == smccat.MOVE_NAMES.index("Branch Length"):
        ch = np.where(br0 != br1)[0]
        assert len(ch) == 1 and np.array_equal(par0, par1)
        assert hastings == pytest.approx(np.log(br1[ch[0]] / br0[ch[0]]), rel=1e-12)
    elif kind == smccat.MOVE_NAMES.index("Scale Subtree"):
        ch = set(np.where(br0 != br1)[0].tolist())
        x = min(ch, key=lambda n: len(subtree(par0, n)) * -1)  # the subtree root
        assert ch <= subtree(par0, x)
        ratios = br1[list(ch)] / br0[list(ch)]
        np.testing.assert_allclose(ratios, ratios[0], rtol=1e-12)
        n_branches = len(subtree(par0, x))
        assert hastings == pytest.approx(n_branches * np.log(ratios[0]), rel=1e-10)
    elif kind in (smccat.MOVE_NAMES.index("NNI"), smccat.MOVE_NAMES.index("Adaptive NNI")):
        assert np.count_nonzero(par0 != par1) == 2
        assert hastings == pytest.approx(0.0, abs=1e-12)   # no split posteriors loaded
    else:
        assert kind == smccat.MOVE_NAMES.index("SPR") and hastings == 0.0
    # the proposed state evaluates like the oracle, and reject restores the old one
    eng.refresh()
    assert eng.lnl()[p] == pytest.approx(oracle_lnl_state(codes, CFG, after, p), rel=1e-9)
    old = before
    mask = np.ones(CFG.particles, np.uint8)
    mask[p] = 0
    eng.accept(mask)
    assert eng.lnl()[p] == pytest.approx(oracle_lnl_state(codes, CFG, old, p), rel=1e-9)
    eng.close()


def _weights(parent, T, post, eps=0.01):
    N = len(parent)
    kids = [[] for _ in range(N)]
    for n, q in enumerate(parent):
        if q >= 0:
            kids[q].append(n)
    root = int(np.where(parent < 0)[0][0])

    def clade(n):
        if n < T:
            return {n}
        return clade(kids[n][0]) | clade(kids[n][1])

    w = {}
    for n in range(T, N):
        if n == root:
            continue
        c = clade(n)
        if 0 not in c:
            c = set(range(T)) - c
        key = frozenset(c)
        trivial = len(c) == 1 or len(c) == T - 1
        w[n] = eps + ((1.0 - post[key]) if (key in post and not trivial) else 1.0)
    return w


def test_adaptive_nni_hastings_with_split_posteriors():
    eng, codes, st = engine()
    rng = np.random.default_rng(9)
    T = CFG.T
    # posterior probabilities for every clade of particle 0's tree and a few others
    post = {}
    for i in range(CFG.particles):
        par = st["parent"][i]
        for n in range(T, 2 * T - 1):
            w = _weights(par, T, {})
        kids = [[] for _ in range(2 * T - 1)]
        for n, q in enumerate(par):
            if q >= 0:
                kids[q].append(n)

        def clade(n):
            return {n} if n < T else clade(kids[n][0]) | clade(kids[n][1])

        for n in range(T, 2 * T - 1):
            c = clade(n)
            if 0 not in c:
                c = set(range(T)) - c
            post[frozenset(c)] = float(rng.random())
    bits = []
    probs = []
    for c, pr in post.items():
        w = [0, 0]
        for t in c:
            w[t >> 6] |= 1 << (t & 63)
        bits.append(w)
        probs.append(pr)
    eng.set_split_posteriors(np.array(bits, dtype=np.uint64), probs)
    seen = 0
    for seed in range(60):
        p = seed % CFG.particles
        before = eng.get_particles()["parent"][p]
        kind, h = eng.propose(p, smccat.FAMILY_TREE, 1000 + seed)
        after = eng.get_particles()["parent"][p]
        if kind == smccat.MOVE_NAMES.index("Adaptive NNI"):
            seen += 1
            ch = np.where(before != after)[0]
            u, v = ch
            cand = {int(before[u]), int(before[v])}
            x = [c for c in cand if int(before[c]) in cand][0]
            w0 = _weights(before, T, post)
            w1 = _weights(after, T, post)
            ref = np.log(w1[x] / sum(w1.values())) - np.log(w0[x] / sum(w0.values()))
            assert h == pytest.approx(ref, rel=1e-10, abs=1e-12)
        eng.refresh()
        eng.accept(np.zeros(CFG.particles, np.uint8))
    assert seen >= 5
    eng.close()


def test_parameter_proposals():
    eng, codes, st = engine()
    tun = eng.tuning()
    for seed in range(4):
        for fam in (smccat.FAMILY_STATIONARY, smccat.FAMILY_SHAPE, smccat.FAMILY_INVAR,
                    smccat.FAMILY_RATE_MATRIX):
            p = (seed + fam) % CFG.particles
            b = eng.get_particles()
            kind, h = eng.propose(p, fam, 77 + seed * 13 + fam)
            a = eng.get_particles()
            if fam == smccat.FAMILY_STATIONARY:
                assert np.count_nonzero(a["logits"][p] != b["logits"][p]) == 1 and h == 0.0
            elif fam == smccat.FAMILY_SHAPE:
                assert h == pytest.approx(np.log(a["shape"][p] / b["shape"][p]), rel=1e-12)
            elif fam == smccat.FAMILY_INVAR:
                al = tun["invar_alpha"]
                p0, p1 = b["pinv"][p], a["pinv"][p]
                aa = al + 1.0
                ref = (stats.beta.logpdf(p0, aa, al / p1 - aa + 2.0)
                       - stats.beta.logpdf(p1, aa, al / p0 - aa + 2.0))
                assert h == pytest.approx(ref, rel=1e-9)
            else:
                nchg = np.count_nonzero(a["base"][p] != b["base"][p])
                if kind == smccat.MOVE_NAMES.index("Rate Matrix Single"):
                    assert nchg == 1
                else:
                    assert kind == smccat.MOVE_NAMES.index("Rate Matrix Full") and nchg == 190
            eng.refresh()
            assert eng.lnl()[p] == pytest.approx(oracle_lnl_state(codes, CFG, a, p), rel=1e-9)
            eng.accept(np.ones(CFG.particles, np.uint8))
    eng.close()


def test_rejuvenate_keeps_exact_likelihoods():
    eng, codes, st = engine()
    res = eng.rejuvenate(iterations=CFG.iterations, temperature=0.4, seed=12345)
    assert sum(res["proposed"]) > 0 and res["lockstep_steps"] > 0
    got = eng.lnl().copy()
    fin = eng.get_particles()
    for i in range(CFG.particles):
        assert got[i] == pytest.approx(oracle_lnl_state(codes, CFG, fin, i), rel=1e-9)
    eng.refresh(full=True)
    np.testing.assert_allclose(eng.lnl(), got, rtol=1e-12)
    # deterministic for a fixed seed
    eng2, _, _ = engine()
    res2 = eng2.rejuvenate(iterations=CFG.iterations, temperature=0.4, seed=12345)
    assert res2 == res
    np.testing.assert_array_equal(eng2.lnl(), got)
    eng.close()
    eng2.close()


def test_smc_step_matches_oracle():
    eng, codes, st = engine(n=6)
    lnl = eng.lnl()
    raw = np.full(6, -np.log(6))
    w, nw, ess, temp = eng.smc_step(raw, 0.6 * 6, 0.0)
    rw, onw, oess, otemp = oracle.next_step(raw, lnl, 0.6 * 6, 0.0)
    assert temp == pytest.approx(otemp, abs=1e-12)
    np.testing.assert_allclose(w, rw, rtol=1e-12)
    np.testing.assert_allclose(nw, onw, rtol=1e-9, atol=1e-300)
    assert ess == pytest.approx(oess, rel=1e-9)
    eng.close()


def test_gibbs_weights_match_oracle():
    eng, codes, st = engine()
    rng = np.random.default_rng(3)
    for trial in range(6):
        p = trial % CFG.particles
        K = int(st["num_classes"][p])
        site = int(rng.integers(CFG.S))
        aux = np.zeros((5, 20))
        aux[:, :19] = rng.normal(size=(5, 19))
        temp = [1.0, 0.37, 0.0][trial % 3]
        got = eng.gibbs_weights(p, site, aux, temp, K)
        counts = np.bincount(st["assign"][p], minlength=K)
        counts[st["assign"][p][site]] -= 1
        live = counts > 0
        rates = oracle.discretize_gamma(st["shape"][p], CFG.R)
        ref = oracle.gibbs_weights(codes, st["parent"][p], st["branch"][p], st["base"][p],
                                   st["logits"][p][:K][live], counts[live], st["pinv"][p], rates,
                                   site, aux, temp)
        exp_full = np.full(K + 5, -np.inf)
        exp_full[np.where(live)[0]] = ref[:live.sum()]
        exp_full[K:] = ref[live.sum():]
        fin = np.isfinite(exp_full)
        assert np.array_equal(np.isfinite(got), fin)
        np.testing.assert_allclose(got[fin], exp_full[fin], rtol=1e-9, atol=1e-9)
    eng.close()


def test_gibbs_move_keeps_exact_likelihoods():
    eng, codes, st = engine()
    res = eng.gibbs(temperature=0.3, seed=42)
    assert res["particles"] == CFG.particles
    fin = eng.get_particles()
    got = eng.lnl()
    for i in range(CFG.particles):
        K = int(fin["num_classes"][i])
        assert np.all(np.bincount(fin["assign"][i], minlength=K) > 0)
        assert got[i] == pytest.approx(oracle_lnl_state(codes, CFG, fin, i), rel=1e-9)
    # a masked call leaves unselected particles untouched
    before = eng.get_particles()
    mask = np.zeros(CFG.particles, np.uint8)
    mask[1] = 1
    eng.gibbs(temperature=1.0, seed=7, mask=mask)
    after = eng.get_particles()
    for i in range(CFG.particles):
        if i != 1:
            np.testing.assert_array_equal(after["assign"][i], before["assign"][i])
    eng.close()


def test_gibbs_at_zero_temperature_samples_the_crp_prior():
    cfg = workload.WorkloadConfig("crp", T=4, S=60, R=1, particles=24, iterations=1, lg=True,
                                  invar=False, cat=True, k_range=(1, 1), seed=8)
    rng = np.random.default_rng(8)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng, kmax=64)
    eng = smccat.Engine(codes, 1, cfg.particles, max_classes=64, lg=True, cat=True)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    alpha = 8.0
    eng.set_tuning(dpp_alpha=alpha)
    ks = []
    # Starting from one class the chain needs ~15 passes of S/2 site updates to
    # forget its start (a numpy run of the same schedule: mean 17.3 over passes
    # 30..59 against the exact 17.57).
    for call in range(60):
        eng.gibbs(temperature=0.0, seed=100 + call)
        if call >= 30:
            ks.extend(eng.get_particles()["num_classes"].tolist())
    expected = sum(alpha / (alpha + i) for i in range(cfg.S))
    assert abs(np.mean(ks) - expected) < 0.1 * expected, (np.mean(ks), expected)
    eng.close()


def test_split_posteriors_match_oracle_and_drive_adaptive_nni():
    """computeSplitPosteriors (Miscellaneous.hpp:115-150) over the particles'
    clade sets (Tree.cpp:485-541), uniform and weighted, against the oracle;
    the result then sets the adaptive NNI node weights."""
    from oracle import splits
    eng, codes, st = engine()
    T = CFG.T
    w = np.random.default_rng(4).random(CFG.particles)
    w /= w.sum()
    for weights in (w, None):
        bits, prob = eng.compute_split_posteriors(weights)
        ref = splits.split_posteriors(st["parent"], T, weights)
        got = {(int(b[0]), int(b[1])): float(p) for b, p in zip(bits, prob)}
        assert set(got) == set(ref)
        for k, v in ref.items():
            assert got[k] == pytest.approx(v, rel=1e-14, abs=1e-15)
        assert np.all(np.diff(prob) <= 0)
    # The uniform table is now installed: adaptive NNI proposals must carry the
    # Hastings ratio of node weights built from it.
    post = {frozenset(t for t in range(T) if (k[t >> 6] >> (t & 63)) & 1): v for k, v in ref.items()}
    seen = 0
    for seed in range(60):
        p = seed % CFG.particles
        before = eng.get_particles()["parent"][p]
        kind, h = eng.propose(p, smccat.FAMILY_TREE, 5000 + seed)
        after = eng.get_particles()["parent"][p]
        if kind == smccat.MOVE_NAMES.index("Adaptive NNI"):
            seen += 1
            u, v = np.where(before != after)[0]
            cand = {int(before[u]), int(before[v])}
            x = [c for c in cand if int(before[c]) in cand][0]
            w0 = _weights(before, T, post)
            w1 = _weights(after, T, post)
            ref_h = np.log(w1[x] / sum(w1.values())) - np.log(w0[x] / sum(w0.values()))
            assert h == pytest.approx(ref_h, rel=1e-10, abs=1e-12)
        eng.refresh()
        eng.accept(np.zeros(CFG.particles, np.uint8))
    assert seen >= 5
    eng.close()


def test_resample_tune_matches_oracle():
    """Systematic resampling and proposal tuning of the SMC step
    (main.cpp:176-301) against oracle/tuning.py; every slot then carries its
    ancestor's state and, after a refresh, its ancestor's log-likelihood."""
    from oracle import tuning
    eng, codes, st = engine()
    n = CFG.particles
    before = eng.get_particles()
    lnl0 = eng.lnl()
    w = np.random.default_rng(21).random(n) ** 3
    w /= w.sum()
    u = 0.37
    anc = eng.resample_tune(w, u, copy=True)
    ref_anc = tuning.systematic_resample(w, u)
    np.testing.assert_array_equal(anc, ref_anc)
    ref = tuning.tune(before, ref_anc, gtr=not CFG.lg)
    t = eng.tuning()
    for k in ("shape_delta", "scale_delta", "stationary_delta", "rate_matrix_delta"):
        assert t[k] == pytest.approx(ref[k], rel=1e-11), k
    assert t["subtree_scale_delta"] == t["scale_delta"]
    assert t["invar_alpha"] == pytest.approx(0.5 * ref["pinv_mean"], rel=1e-12)
    np.testing.assert_allclose(eng.rate_cholesky(), ref["cholesky"], rtol=1e-9, atol=1e-12)
    after = eng.get_particles()
    for i in range(n):
        np.testing.assert_array_equal(after["parent"][i], before["parent"][anc[i]])
        np.testing.assert_array_equal(after["assign"][i], before["assign"][anc[i]])
        np.testing.assert_array_equal(after["branch"][i], before["branch"][anc[i]])
    eng.refresh()
    np.testing.assert_allclose(eng.lnl(), lnl0[anc], rtol=1e-12)
    eng.close()


@pytest.mark.parametrize("reassign,device_sweep", [("gibbs", False), ("learned", False), ("learned", True)],
                         ids=["gibbs-host", "learned-host", "learned-device"])
def test_smc_driver_reaches_temperature_one(reassign, device_sweep):
    """The reference's SMC loop over the C-ABI (smccat.smc.run): temperatures
    rise monotonically to 1, resampling rounds happen, log Z is finite and the
    particles keep exact likelihoods; rejuvenation host-driven or as the device
    sweep."""
    from smccat import smc
    rng = np.random.default_rng(CFG.seed)
    codes, _ = workload.simulate_alignment(CFG, rng)
    n = 8
    st = workload.make_particles(CFG, n, rng, kmax=12)
    eng = smccat.Engine(codes, CFG.R, n, max_classes=12, lg=CFG.lg, invar=CFG.invar, cat=CFG.cat)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], np.maximum(st["pinv"], 0.05), st["shape"])
    eng.refresh(full=True)
    res = smc.run(eng, cat=True, iterations=2, alg8_probability=0.5, reassign=reassign,
                  learned_warmup=1, learned_updates=30, seed=4, device_sweep=device_sweep)
    temps = res["temperatures"]
    assert temps[-1] == 1.0 and all(b >= a for a, b in zip(temps, temps[1:]))
    assert res["resamples"] >= 1 and np.isfinite(res["log_z"])
    fin = eng.get_particles()
    got = eng.lnl()
    for i in range(n):
        assert got[i] == pytest.approx(oracle_lnl_state(codes, CFG, fin, i), rel=1e-9)
    eng.close()


def test_gibbs_class_table_matches_per_site_evaluation():
    """Gibbs reads the site log-likelihoods of the classes a particle enters
    with from a table the SIMT pruning kernels fill beforehand; with a kernel
    variant that has no evaluation mode (the FP64 tensor-path kernels) every
    class is pruned per site inside the Gibbs kernel instead. Same state, same
    seed: the same draws, hence the same assignments and likelihoods."""
    cfg = workload.WorkloadConfig("gibbs_table", T=10, S=300, R=4, particles=6, iterations=1,
                                  lg=False, invar=True, cat=True, pinv=0.1, k_range=(2, 7), seed=71)
    rng = np.random.default_rng(cfg.seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng, kmax=24)
    out = []
    for variant in (None, "dmma"):
        eng = smccat.Engine(codes, cfg.R, cfg.particles, max_classes=24, invar=True, cat=True)
        eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                          st["logits"], st["assign"], st["pinv"], st["shape"])
        eng.refresh(full=True)
        if variant == "dmma":
            n, _ = eng.kernel_variants()
            eng.set_kernel_variant(n - 1)
        eng.gibbs(temperature=0.8, seed=13)
        out.append((eng.get_particles(), eng.lnl()))
        eng.close()
    (a, la), (b, lb) = out
    np.testing.assert_array_equal(a["num_classes"], b["num_classes"])
    np.testing.assert_array_equal(a["assign"], b["assign"])
    np.testing.assert_allclose(la, lb, rtol=1e-12)


def test_reassignment_groups_do_not_change_results():
    """Gibbs and the learned move run their particles in device passes sized
    to the free memory; the random streams are keyed by particle, so passes
    of two particles give the same assignments and likelihoods as one pass of
    all of them."""
    cfg = workload.WorkloadConfig("groups", T=10, S=300, R=4, particles=6, iterations=1,
                                  lg=False, invar=True, cat=True, pinv=0.1, k_range=(2, 7), seed=72)
    rng = np.random.default_rng(cfg.seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng, kmax=24)
    params = (np.random.default_rng(8).normal(size=smccat.MLP_PARAMS) * 0.1).astype(np.float32)
    out = []
    for group in (0, 2):
        eng = smccat.Engine(codes, cfg.R, cfg.particles, max_classes=24, invar=True, cat=True)
        eng.set_reassign_group(group)
        eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                          st["logits"], st["assign"], st["pinv"], st["shape"])
        eng.refresh(full=True)
        g = eng.gibbs(temperature=0.8, seed=21)
        eng.learned_params(set_to=params)
        lm = eng.learned_move(updates=100, temperature=0.8, seed=22)
        out.append((eng.get_particles(), eng.lnl(), g, lm))
        eng.close()
    (a, la, ga, ma), (b, lb, gb, mb) = out
    assert ga == gb and ma == mb
    np.testing.assert_array_equal(a["num_classes"], b["num_classes"])
    np.testing.assert_array_equal(a["assign"], b["assign"])
    np.testing.assert_allclose(la, lb, rtol=1e-12)


def test_gibbs_with_no_site_iterations():
    """floor(S/2) = 0 iterations (a one-site alignment): the pass leaves every
    particle as it was, with its likelihood exact."""
    cfg = workload.WorkloadConfig("one_site", T=6, S=1, R=4, particles=3, iterations=1,
                                  lg=True, invar=False, cat=True, k_range=(1, 1), seed=5)
    rng = np.random.default_rng(cfg.seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng, kmax=4)
    eng = smccat.Engine(codes, cfg.R, cfg.particles, max_classes=4, lg=True, cat=True)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    before = eng.lnl().copy()
    res = eng.gibbs(temperature=1.0, seed=3)
    assert res["particles"] == cfg.particles and res["created"] == 0
    fin = eng.get_particles()
    np.testing.assert_array_equal(fin["num_classes"], st["num_classes"])
    np.testing.assert_array_equal(fin["assign"], st["assign"])
    np.testing.assert_allclose(eng.lnl(), before, rtol=1e-12)
    eng.close()

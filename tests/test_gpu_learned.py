"""The learned CAT class proposal: device gradients against the CPU oracle, and
what the trained network gains over an untrained (uniform) proposal."""
import numpy as np
import pytest

import oracle
from oracle import mlp as omlp
import smccat
from smccat import workload

pytestmark = pytest.mark.gpu


def cat_engine(seed=31, n=8, S=240):
    cfg = workload.WorkloadConfig("learned", T=10, S=S, R=4, particles=n, iterations=2,
                                  lg=False, invar=False, cat=True, alpha=0.8,
                                  dp_concentration=3.0, k_range=(4, 6), seed=seed)
    rng = np.random.default_rng(seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, n, rng, kmax=16)
    eng = smccat.Engine(codes, cfg.R, n, max_classes=16, cat=True)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    return eng, codes, cfg


def test_gradients_match_cpu_oracle():
    eng, codes, cfg = cat_engine(n=2)
    rng = np.random.default_rng(4)
    params = (rng.normal(size=omlp.N_PARAMS) * 0.1).astype(np.float32)
    eng.learned_params(set_to=params)
    sizes = [3, 5, 2, 6, 4, 1, 7]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    X = rng.normal(size=(off[-1], omlp.IN)).astype(np.float32)
    labels = np.array([rng.integers(s) for s in sizes], dtype=np.int32)
    loss, g = eng.learned_gradients(X, off, labels)
    rloss, rg = omlp.loss_and_grad(params.astype(np.float64), X.astype(np.float64), off, labels)
    assert loss == pytest.approx(rloss, rel=1e-4)
    scale = np.abs(rg).max()
    np.testing.assert_allclose(g, rg, atol=2e-4 * scale, rtol=1e-3)
    # finite-difference check of the oracle itself on a few coordinates
    for idx in (0, omlp.IN * omlp.HID + 3, omlp.N_PARAMS - 1):
        e = np.zeros(omlp.N_PARAMS)
        e[idx] = 1e-6
        p64 = params.astype(np.float64)
        fd = (omlp.loss_and_grad(p64 + e, X, off, labels)[0]
              - omlp.loss_and_grad(p64 - e, X, off, labels)[0]) / 2e-6
        assert fd == pytest.approx(rg[idx], rel=1e-4, abs=1e-7)
    eng.close()


def test_trained_proposal_beats_uniform_and_keeps_exact_likelihoods():
    eng, codes, cfg = cat_engine()
    # Gibbs warm-up produces the training assignments.
    for call in range(4):
        eng.gibbs(temperature=1.0, seed=10 + call)
    # Untrained network (all-zero weights): a uniform proposal over classes.
    eng.learned_params(set_to=np.zeros(smccat.MLP_PARAMS, np.float32))
    base = eng.learned_move(updates=400, temperature=1.0, seed=5)
    # Train from a fresh initialisation (Glorot) on the Gibbs samples.
    eng.learned_params(set_to=(np.random.default_rng(1).normal(size=smccat.MLP_PARAMS) * 0.05)
                       .astype(np.float32))
    loss = eng.learned_train(epochs=30, batch_sites=256, lr=3e-3, seed=2)
    k_mean = eng.get_particles()["num_classes"].mean()
    assert loss < 0.9 * np.log(k_mean), (loss, np.log(k_mean))   # better than chance
    trained = eng.learned_move(updates=400, temperature=1.0, seed=5)
    acc_base = base["accepted"] / base["proposed"]
    acc_trained = trained["accepted"] / trained["proposed"]
    assert acc_trained > acc_base, (acc_trained, acc_base)
    fin = eng.get_particles()
    got = eng.lnl()
    for i in range(cfg.particles):
        K = int(fin["num_classes"][i])
        assert np.all(np.bincount(fin["assign"][i], minlength=K) > 0)
        rates = oracle.discretize_gamma(fin["shape"][i], cfg.R)
        ref = oracle.lnl(codes, fin["parent"][i], fin["branch"][i], fin["base"][i],
                         fin["logits"][i][:K], fin["assign"][i], fin["pinv"][i], rates)
        assert got[i] == pytest.approx(ref, rel=1e-9)
    eng.close()


def test_learned_move_at_zero_temperature_samples_the_crp_prior():
    """At temperature 0 the target is the CRP prior alone. The learned move
    keeps K fixed (it never opens or empties a class), so over labelled
    assignments with all K classes non-empty the chain must sample
    p(z) ~ prod_k (n_k - 1)!, i.e. a class-size vector c with probability
    ~ S! prod_k (c_k - 1)! / c_k! = S! prod_k 1 / c_k. Any proposal network
    works here: the Metropolis-Hastings ratio (prior n_b / (n_a - 1), proposal
    q_rev / q_fwd, site selection 1/S both ways) is what is tested. 2,048
    independent chains of 6 sites and 3 classes, chi-square over the 10
    size vectors."""
    from itertools import product
    from scipy import stats
    S, K, n = 6, 3, 2048
    cfg = workload.WorkloadConfig("crp_learned", T=4, S=S, R=4, particles=n, iterations=1,
                                  lg=True, invar=False, cat=True, k_range=(K, K), seed=9)
    rng = np.random.default_rng(9)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, n, rng, kmax=K)
    st["assign"][:] = np.arange(S) % K
    eng = smccat.Engine(codes, cfg.R, n, max_classes=K, lg=True, cat=True)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    # An arbitrary (random) scoring network: non-uniform, state-dependent proposals.
    eng.learned_params(set_to=(np.random.default_rng(3).normal(size=smccat.MLP_PARAMS) * 0.3)
                       .astype(np.float32))
    vecs = [c for c in product(range(1, S + 1), repeat=K) if sum(c) == S]
    index = {c: i for i, c in enumerate(vecs)}
    p = np.array([np.prod([1.0 / x for x in c]) for c in vecs])
    p /= p.sum()
    obs = np.zeros(len(vecs))
    eng.learned_move(updates=200, temperature=0.0, seed=1)   # burn-in
    for snap in range(3):   # 3 snapshots, 100 updates apart
        eng.learned_move(updates=100, temperature=0.0, seed=2 + snap)
        a = eng.get_particles()["assign"]
        for i in range(n):
            obs[index[tuple(np.bincount(a[i], minlength=K))]] += 1
    stat, pval = stats.chisquare(obs, p * obs.sum())
    assert pval > 1e-3, (pval, obs.tolist(), (p * obs.sum()).tolist())
    eng.close()


def test_learned_move_table_matches_per_update_pruning():
    """The learned move reads its two classes' site log-likelihoods from the
    class table the SIMT pruning kernels fill before the pass; with a kernel
    variant that has no evaluation mode (the FP64 tensor-path kernels) it
    prunes the site under both classes at every update instead. Same state,
    network and seed: the same proposals and decisions, hence the same
    assignments."""
    out = []
    for variant in (None, "dmma"):
        eng, codes, cfg = cat_engine(seed=33, n=6)
        eng.learned_params(set_to=(np.random.default_rng(5).normal(size=smccat.MLP_PARAMS) * 0.1)
                           .astype(np.float32))
        if variant == "dmma":
            n, _ = eng.kernel_variants()
            eng.set_kernel_variant(n - 1)
        r = eng.learned_move(updates=300, temperature=1.0, seed=9)
        out.append((eng.get_particles()["assign"], r["accepted"], r["proposed"], eng.lnl()))
        eng.close()
    (a, acc_a, prop_a, la), (b, acc_b, prop_b, lb) = out
    assert prop_a == prop_b and acc_a == acc_b
    np.testing.assert_array_equal(a, b)
    np.testing.assert_allclose(la, lb, rtol=1e-9)


def _bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def test_tensor_core_scores_match_cpu_oracle():
    """The learned move scores every class with two tcgen05 BF16 products
    (feature rows, weights and hidden activations in BF16, FP32 accumulation).
    Against the float64 oracle forward pass on the same features, with the same
    BF16 roundings applied, for a particle with more classes than one 128-row
    product holds."""
    K, S, T = 150, 400, 8
    cfg = workload.WorkloadConfig("scores", T=T, S=S, R=4, particles=1, iterations=1, lg=False,
                                  invar=False, cat=True, k_range=(K, K), seed=12)
    rng = np.random.default_rng(12)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, 1, rng, kmax=K)
    eng = smccat.Engine(codes, cfg.R, 1, max_classes=K, cat=True)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    params = (np.random.default_rng(6).normal(size=omlp.N_PARAMS) * 0.15).astype(np.float32)
    eng.learned_params(set_to=params)
    q = omlp.unpack(_bf16(params).astype(np.float64))
    lg = st["logits"][0][:K]
    pi = np.exp(lg - lg.max(axis=1, keepdims=True))
    pi /= pi.sum(axis=1, keepdims=True)
    pi32 = pi.astype(np.float32)
    lpi32 = np.log(pi).astype(np.float32)
    counts = np.bincount(st["assign"][0], minlength=K)
    for site in (0, 17, 233, S - 1):
        col = codes[:, site]
        res = col[col < 20]
        sf = np.zeros(21, np.float32)
        sf[:20] = np.bincount(res, minlength=20)[:20] / max(len(res), 1)
        sf[20] = 1.0 - len(res) / T
        X = np.zeros((K, omlp.IN), np.float32)
        X[:, :21] = sf
        X[:, 21:41] = pi32
        X[:, 41] = np.log(np.maximum(counts, 1)).astype(np.float32)
        X[:, 42] = (lpi32 * sf[:20]).sum(axis=1)
        Xq = _bf16(X).astype(np.float64)
        H1 = _bf16(np.maximum(Xq @ q["W1"] + q["b1"], 0)).astype(np.float64)
        H2 = np.maximum(H1 @ q["W2"] + q["b2"], 0)
        ref = H2 @ q["w3"] + q["b3"][0]
        got = eng.learned_scores(0, site, K)
        scale = np.abs(ref).max()
        np.testing.assert_allclose(got, ref, atol=3e-3 * scale, rtol=0)
    eng.close()

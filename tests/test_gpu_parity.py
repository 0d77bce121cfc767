"""GPU parity of the FP64 likelihood path against the FP64 oracle.

Every test drives the CUDA path through the C-ABI (``smccat.Engine``) and
checks it against ``oracle`` on the same particle states. Tolerance: the FP64
path must match to 1e-9 relative log-likelihood (per particle) and 1e-9
relative + 1e-9 absolute per site.
"""
import json
import os

import numpy as np
import pytest

import oracle
import smccat
from smccat import workload

pytestmark = pytest.mark.gpu

RTOL = 1e-9
GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def oracle_lnl(codes, st, i, rates_R):
    K = int(st["num_classes"][i])
    rates = oracle.discretize_gamma(st["shape"][i], rates_R) if rates_R > 1 else [1.0]
    return oracle.lnl(codes, st["parent"][i], st["branch"][i], st["base"][i],
                      st["logits"][i][:K], st["assign"][i], st["pinv"][i], rates, site_out=True)


def make_engine(cfg, n, seed, kmax=None):
    rng = np.random.default_rng(seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, n, rng, kmax=kmax)
    eng = smccat.Engine(codes, cfg.R, n, max_classes=st["logits"].shape[1], lg=cfg.lg,
                        invar=cfg.invar, cat=cfg.cat)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    return eng, codes, st


SMALL = [
    workload.WorkloadConfig("small_lg_r1", T=6, S=70, R=1, particles=4, iterations=1, lg=True,
                            invar=False, cat=False, seed=11),
    workload.WorkloadConfig("small_gtr_g4_i", T=9, S=150, R=4, particles=5, iterations=1,
                            lg=False, invar=True, cat=False, alpha=0.5, pinv=0.1, seed=12),
    workload.WorkloadConfig("small_cat", T=7, S=200, R=4, particles=4, iterations=1, lg=False,
                            invar=True, cat=True, dp_concentration=3.0, k_range=(2, 9), seed=13),
    workload.WorkloadConfig("small_r3_cat", T=5, S=90, R=3, particles=3, iterations=1, lg=True,
                            invar=False, cat=True, k_range=(1, 4), seed=14),
    workload.WorkloadConfig("odd_r8", T=3, S=33, R=8, particles=2, iterations=1, lg=False,
                            invar=True, cat=False, seed=15),
]


@pytest.mark.parametrize("cfg", SMALL, ids=lambda c: c.name)
def test_full_refresh_matches_oracle(cfg):
    eng, codes, st = make_engine(cfg, cfg.particles, cfg.seed)
    got = eng.lnl()
    for i in range(cfg.particles):
        ref, ref_sites = oracle_lnl(codes, st, i, cfg.R)
        assert got[i] == pytest.approx(ref, rel=RTOL), i
        np.testing.assert_allclose(eng.site_lnl(i), ref_sites, rtol=RTOL, atol=1e-9)
    eng.close()


@pytest.mark.parametrize("case", GOLD["likelihood"], ids=lambda c: f"T{c['T']}S{c['S']}R{c['R']}K{c['K']}")
def test_golden_cases(case):
    T, S, K, R = case["T"], case["S"], case["K"], case["R"]
    codes = np.array(case["codes"], dtype=np.uint8).reshape(T, S)
    eng = smccat.Engine(codes, R, 1, max_classes=K, lg=case["lg"], invar=case["pinv"] > 0,
                        cat=K > 1)
    eng.set_particles(0, np.array([case["parent"]]), np.array([case["branch"]]),
                      np.array([case["base"]]), np.array([K]),
                      np.array(case["logits"]).reshape(1, K, 20), np.array([case["assign"]]),
                      np.array([case["pinv"]]), np.array([case["shape"]]))
    eng.refresh(full=True)
    assert eng.lnl()[0] == pytest.approx(case["lnl"], rel=RTOL)
    np.testing.assert_allclose(eng.site_lnl(0), case["site_lnl"], rtol=RTOL, atol=1e-9)
    eng.close()


def test_transition_matrices_match_oracle():
    """Device spectral decomposition + P(t r) against the oracle, every edge."""
    cfg = SMALL[2]
    eng, codes, st = make_engine(cfg, 2, 31)
    worst = 0.0
    for p in range(2):
        rates = oracle.discretize_gamma(st["shape"][p], cfg.R)
        root = int(np.where(st["parent"][p] < 0)[0][0])
        for k in range(int(st["num_classes"][p])):
            pi = oracle.softmax20(st["logits"][p, k])
            for node in range(2 * cfg.T - 1):
                if node == root:
                    continue
                for r in range(cfg.R):
                    ref = oracle.transition(st["base"][p], pi, st["branch"][p, node] * rates[r])
                    got = eng.transition_matrix(p, k, node, r)
                    worst = max(worst, np.abs(got - ref).max())
    assert worst < 1e-13
    eng.close()


def _nni(parent, rng):
    """Swap a child of an internal non-root node p with its sibling's side."""
    parent = parent.copy()
    N = len(parent)
    T = (N + 1) // 2
    kids = [[] for _ in range(N)]
    for n, p in enumerate(parent):
        if p >= 0:
            kids[p].append(n)
    cands = [n for n in range(T, N) if parent[n] >= 0]
    p = cands[rng.integers(len(cands))]
    a = parent[p]
    n1 = kids[p][rng.integers(2)]
    n2 = [x for x in kids[a] if x != p][0]
    parent[n1], parent[n2] = a, p
    return parent


def _spr(parent, rng):
    parent = parent.copy()
    N = len(parent)
    T = (N + 1) // 2
    kids = [[] for _ in range(N)]
    for n, p in enumerate(parent):
        if p >= 0:
            kids[p].append(n)
    root = int(np.where(parent < 0)[0][0])
    while True:
        p = int(rng.integers(T, N))
        if p != root and parent[p] != -1:
            break
    s = kids[p][rng.integers(2)]
    sib = [x for x in kids[p] if x != s][0]

    def in_sub(x, r):
        while x >= 0:
            if x == r:
                return True
            x = parent[x]
        return False

    while True:
        a = int(rng.integers(0, N))
        if a != root and not in_sub(a, p) and parent[a] != p:
            break
    g = parent[p]
    parent[sib] = g
    ap = parent[a]
    parent[p] = ap
    parent[a] = p
    return parent


@pytest.mark.parametrize("cfg", SMALL[1:3], ids=lambda c: c.name)
def test_dirty_edits_accept_reject(cfg):
    n = cfg.particles
    eng, codes, st = make_engine(cfg, n, cfg.seed + 100)
    rng = np.random.default_rng(cfg.seed + 7)
    cur = {k: v.copy() for k, v in st.items()}
    committed = eng.lnl().copy()
    N = 2 * cfg.T - 1
    for step in range(24):
        prop = {k: v.copy() for k, v in cur.items()}
        kind = step % 8
        for i in range(n):
            root = int(np.where(prop["parent"][i] < 0)[0][0])
            if kind == 0:      # one branch
                x = int(rng.integers(0, N - 1))
                x = x if x != root else N - 1
                prop["branch"][i, x] *= np.exp(rng.random() - 0.5)
                eng.set_branch_lengths(i, [x], [prop["branch"][i, x]])
            elif kind == 1:    # subtree scale: a set of branches
                xs = [x for x in range(N) if x != root and rng.random() < 0.4]
                prop["branch"][i, xs] *= 1.3
                eng.set_branch_lengths(i, xs, prop["branch"][i, xs])
            elif kind == 2:
                prop["parent"][i] = _nni(prop["parent"][i], rng)
                eng.set_topology(i, prop["parent"][i], prop["branch"][i])
            elif kind == 3:
                prop["parent"][i] = _spr(prop["parent"][i], rng)
                eng.set_topology(i, prop["parent"][i], prop["branch"][i])
            elif kind == 4:
                prop["pinv"][i] = rng.random() * 0.9
                eng.set_pinv(i, prop["pinv"][i])
            elif kind == 5:
                prop["shape"][i] *= np.exp(rng.random() - 0.5)
                eng.set_shape(i, prop["shape"][i])
            elif kind == 6:
                prop["base"][i] += 0.2 * rng.normal(size=190)
                eng.set_base(i, prop["base"][i])
            else:
                k = int(rng.integers(prop["num_classes"][i]))
                prop["logits"][i, k, :19] += 0.3 * rng.normal(size=19)
                eng.set_class_logits(i, k, prop["logits"][i, k])
        eng.refresh()
        got = eng.lnl()
        for i in range(n):
            ref, _ = oracle_lnl(codes, prop, i, cfg.R)
            assert got[i] == pytest.approx(ref, rel=RTOL), (step, kind, i)
        mask = rng.random(n) < 0.5
        eng.accept(mask.astype(np.uint8))
        after = eng.lnl()
        for i in range(n):
            if mask[i]:
                for k in cur:
                    cur[k][i] = prop[k][i]
                assert after[i] == got[i]
            else:
                assert after[i] == committed[i]
        committed = after.copy()
        back = eng.get_particles()
        np.testing.assert_array_equal(back["parent"], cur["parent"])
        np.testing.assert_array_equal(back["branch"], cur["branch"])
    # A full rebuild of the final state reproduces the incrementally kept value.
    eng.refresh(full=True)
    np.testing.assert_allclose(eng.lnl(), committed, rtol=1e-12)
    eng.close()


def test_two_refreshes_before_reject_restore_committed_state():
    cfg = SMALL[1]
    eng, codes, st = make_engine(cfg, 2, 77)
    base_lnl = eng.lnl().copy()
    eng.set_branch_lengths(0, [0], [st["branch"][0, 0] * 3])
    eng.refresh()
    eng.set_branch_lengths(0, [1], [st["branch"][0, 1] * 0.2])
    eng.refresh()
    eng.accept(np.array([0, 0], np.uint8))
    np.testing.assert_array_equal(eng.lnl(), base_lnl)
    eng.refresh(full=True)
    np.testing.assert_allclose(eng.lnl(), base_lnl, rtol=1e-12)
    eng.close()


def test_autotune_keeps_likelihoods():
    cfg = SMALL[1]
    eng, codes, st = make_engine(cfg, 3, 41)
    before = eng.lnl().copy()
    res = eng.autotune(reps=1)
    assert 0 <= res["variant"] < max(1, len(res["ms"]))
    np.testing.assert_array_equal(eng.lnl(), before)
    # edits and reject after the tuner's refreshes still restore the committed state
    eng.set_branch_lengths(1, [0], [st["branch"][1, 0] * 2])
    eng.refresh()
    eng.accept(np.array([1, 0, 1], np.uint8))
    np.testing.assert_array_equal(eng.lnl(), before)
    eng.close()


def test_protocol_errors():
    cfg = SMALL[0]
    eng, codes, st = make_engine(cfg, 2, 5)
    eng.set_pinv(0, 0.0)
    with pytest.raises(smccat.SmccatError) as e:
        eng.accept(np.array([1, 1], np.uint8))
    assert e.value.code == smccat.ESTATE
    with pytest.raises(smccat.SmccatError):
        bad = st["parent"][0].copy()
        bad[0] = bad[1] = bad[2] = cfg.T   # three children
        eng.set_topology(0, bad, st["branch"][0])
    eng.close()


@pytest.mark.parametrize("cfg", [SMALL[1], SMALL[3], SMALL[4]], ids=lambda c: c.name)
def test_every_kernel_variant_matches_oracle(cfg):
    """Each pruning-kernel variant (SIMT register caps, FP64 tensor path) on a
    full refresh and on dirty re-evaluation after branch and NNI edits."""
    rng = np.random.default_rng(cfg.seed + 55)
    codes, _ = workload.simulate_alignment(cfg, rng)
    n = cfg.particles
    st = workload.make_particles(cfg, n, rng)
    eng = smccat.Engine(codes, cfg.R, n, max_classes=st["logits"].shape[1], lg=cfg.lg,
                        invar=cfg.invar, cat=cfg.cat)
    nv, _ = eng.kernel_variants()
    assert nv >= 2
    for v in range(nv):
        eng.set_kernel_variant(v)
        eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                          st["logits"], st["assign"], st["pinv"], st["shape"])
        eng.refresh(full=True)
        cur = {k: x.copy() for k, x in st.items()}
        for i in range(n):
            ref, sites = oracle_lnl(codes, cur, i, cfg.R)
            assert eng.lnl()[i] == pytest.approx(ref, rel=RTOL), (v, i)
            np.testing.assert_allclose(eng.site_lnl(i), sites, rtol=RTOL, atol=1e-9)
        for step in range(3):
            for i in range(n):
                if step == 1:
                    cur["parent"][i] = _nni(cur["parent"][i], rng)
                    eng.set_topology(i, cur["parent"][i], cur["branch"][i])
                else:
                    x = int(rng.integers(0, cfg.T))  # a tip's branch
                    cur["branch"][i, x] *= 1.7
                    eng.set_branch_lengths(i, [x], [cur["branch"][i, x]])
            eng.refresh()
            eng.accept(np.ones(n, np.uint8))
            got = eng.lnl()
            for i in range(n):
                ref, _ = oracle_lnl(codes, cur, i, cfg.R)
                assert got[i] == pytest.approx(ref, rel=RTOL), (v, step, i)
    eng.close()


MIXED_ATOL = 3e-4  # |dlogL| per particle (nats) allowed for the FP32 path (sites <= 2,000)


@pytest.mark.parametrize("cfg", SMALL, ids=lambda c: c.name)
def test_mixed_precision_full_refresh(cfg):
    rng = np.random.default_rng(cfg.seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng)
    eng = smccat.Engine(codes, cfg.R, cfg.particles, max_classes=st["logits"].shape[1],
                        lg=cfg.lg, invar=cfg.invar, cat=cfg.cat, precision=smccat.PREC_FP32)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    got = eng.lnl()
    for i in range(cfg.particles):
        ref, _ = oracle_lnl(codes, st, i, cfg.R)
        assert abs(got[i] - ref) <= MIXED_ATOL, (i, got[i] - ref)
    eng.close()


def test_mixed_precision_dirty_edits():
    cfg = SMALL[2]
    rng = np.random.default_rng(5)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, 3, rng)
    eng = smccat.Engine(codes, cfg.R, 3, max_classes=st["logits"].shape[1], invar=True, cat=True,
                        precision=smccat.PREC_FP32)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    cur = {k: v.copy() for k, v in st.items()}
    for step in range(6):
        for i in range(3):
            x = int(rng.integers(0, 2 * cfg.T - 2))
            x = x if cur["parent"][i][x] >= 0 else x + 1
            cur["branch"][i, x] *= 1.5
            eng.set_branch_lengths(i, [x], [cur["branch"][i, x]])
        eng.refresh()
        eng.accept(np.ones(3, np.uint8))
        got = eng.lnl()
        for i in range(3):
            ref, _ = oracle_lnl(codes, cur, i, cfg.R)
            assert abs(got[i] - ref) <= MIXED_ATOL
    eng.close()


@pytest.mark.parametrize("cid", [1, 2])
def test_reference_configs_full_size(cid):
    """Configs 1 and 2 at full size: every particle against the oracle."""
    cfg = workload.CONFIGS[cid]
    rng = np.random.default_rng(cfg.seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    n = cfg.particles if cid == 1 else 32
    st = workload.make_particles(cfg, n, rng)
    eng = smccat.Engine(codes, cfg.R, n, lg=cfg.lg, invar=cfg.invar, cat=cfg.cat)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    got = eng.lnl()
    rates = np.stack([oracle.discretize_gamma(s, cfg.R) for s in st["shape"]])
    ref = oracle.lnl_batch(codes, st["parent"], st["branch"], st["base"], st["num_classes"],
                           st["logits"], st["assign"], st["pinv"], rates)
    np.testing.assert_allclose(got, ref, rtol=RTOL)
    eng.close()


@pytest.mark.parametrize("cfg", SMALL, ids=lambda c: c.name)
def test_every_fp32_variant_matches_oracle(cfg):
    """Each FP32 pruning variant (SIMT register caps and the tcgen05 3xTF32
    kernel) within the FP32 tolerance, R = 1 .. 8 and T = 3 included."""
    rng = np.random.default_rng(cfg.seed + 7)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng)
    eng = smccat.Engine(codes, cfg.R, cfg.particles, max_classes=st["logits"].shape[1],
                        lg=cfg.lg, invar=cfg.invar, cat=cfg.cat, precision=smccat.PREC_FP32)
    nv, _ = eng.kernel_variants()
    refs = [oracle_lnl(codes, st, i, cfg.R)[0] for i in range(cfg.particles)]
    for v in range(nv):
        eng.set_kernel_variant(v)
        eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                          st["logits"], st["assign"], st["pinv"], st["shape"])
        eng.refresh(full=True)
        got = eng.lnl()
        for i in range(cfg.particles):
            assert abs(got[i] - refs[i]) <= MIXED_ATOL, (v, i, got[i] - refs[i])
    eng.close()


@pytest.mark.parametrize("precision", [smccat.PREC_FP64, smccat.PREC_FP32], ids=["fp64", "fp32"])
def test_persistent_variant_over_many_tiles(precision):
    """The persistent pruning variant (one wave of CTAs walking ~1,000 tiles,
    several per CTA) gives the same values as the one-tile-per-CTA kernel it
    wraps, on full refreshes and on lockstep rejuvenation with finished
    (inactive) particles."""
    cfg = workload.WorkloadConfig("many_tiles", T=12, S=2000, R=4, particles=16, iterations=1,
                                  lg=False, invar=True, cat=False, alpha=0.5, pinv=0.1, seed=21)
    rng = np.random.default_rng(cfg.seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng)
    fp32 = precision == smccat.PREC_FP32
    base_v, pers_v = (4, 12) if fp32 else (3, 9)
    outs = []
    for v in (base_v, pers_v):
        eng = smccat.Engine(codes, cfg.R, cfg.particles, max_classes=st["logits"].shape[1],
                            lg=cfg.lg, invar=cfg.invar, cat=cfg.cat, precision=precision)
        eng.set_kernel_variant(v)
        eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                          st["logits"], st["assign"], st["pinv"], st["shape"])
        eng.refresh(full=True)
        full = eng.lnl()
        eng.rejuvenate(iterations=2, temperature=0.8, seed=5)
        outs.append((full, eng.lnl(), eng.get_particles()))
        eng.close()
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    fin = outs[1][2]
    for i in range(0, cfg.particles, 5):
        ref, _ = oracle_lnl(codes, fin, i, cfg.R)
        if fp32:
            assert abs(outs[1][1][i] - ref) <= MIXED_ATOL
        else:
            assert outs[1][1][i] == pytest.approx(ref, rel=RTOL)

"""Pin the FP64 oracle against the golden fixtures (tests/golden/golden.json).

The fixtures come from tests/golden/make_golden.py, an independent restatement
that uses the reference's own numerical route (general eigendecomposition +
inverse for P(t), scipy's gamma quantile for Boost's, the LG table parsed out
of the reference source).
"""
import json
import os

import numpy as np
import pytest

import oracle

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def test_lg_table_matches_reference_source():
    np.testing.assert_array_equal(oracle.lg_base(), np.array(GOLD["lg_base"]))


@pytest.mark.parametrize("case", GOLD["gamma_ppf"], ids=lambda c: f"a{c['a']}-p{c['p']}")
def test_gamma_quantile(case):
    x = oracle.gamma_quantile(case["a"], 1.0, case["p"])
    assert x == pytest.approx(case["x"], rel=1e-12, abs=1e-300)


@pytest.mark.parametrize("case", GOLD["discretize_gamma"],
                         ids=lambda c: f"shape{c['shape']}-R{c['R']}")
def test_discretize_gamma(case):
    r = oracle.discretize_gamma(case["shape"], case["R"])
    np.testing.assert_allclose(r, case["rates"], rtol=1e-11, atol=0)
    assert r.mean() == pytest.approx(1.0, rel=1e-14)


def test_transition_matches_general_eigensolver():
    worst = 0.0
    for c in GOLD["transition"]:
        pi = oracle.softmax20(c["logits"])
        P = oracle.transition(c["base"], pi, c["t"])
        ref = np.array(c["P"]).reshape(20, 20)
        worst = max(worst, np.abs(P - ref).max())
    assert worst < 1e-12


def test_transition_known_answers():
    rng = np.random.default_rng(3)
    base = rng.normal(size=190)
    lg = np.zeros(20)
    lg[:19] = rng.normal(size=19)
    pi = oracle.softmax20(lg)
    np.testing.assert_allclose(oracle.transition(base, pi, 0.0), np.eye(20), atol=1e-14)
    for t in [0.01, 0.3, 3.0]:
        P = oracle.transition(base, pi, t)
        np.testing.assert_allclose(P.sum(axis=1), 1.0, atol=1e-13)        # rows sum to 1
        D = pi[:, None] * P
        np.testing.assert_allclose(D, D.T, atol=1e-14)                      # detailed balance
    P = oracle.transition(base, pi, 400.0)
    np.testing.assert_allclose(P, np.tile(pi, (20, 1)), atol=1e-12)         # P(inf) = 1 pi^T
    Q = oracle.rate_matrix(base, pi)
    assert -np.sum(np.diag(Q) * pi) == pytest.approx(1.0, rel=1e-14)        # mean rate 1


@pytest.mark.parametrize("case", GOLD["likelihood"], ids=lambda c: f"T{c['T']}S{c['S']}R{c['R']}K{c['K']}")
def test_lnl_matches_golden(case):
    T, S = case["T"], case["S"]
    codes = np.array(case["codes"], dtype=np.uint8).reshape(T, S)
    logits = np.array(case["logits"]).reshape(case["K"], 20)
    v, site = oracle.lnl(codes, case["parent"], case["branch"], case["base"], logits,
                         case["assign"], case["pinv"], case["rates"], site_out=True)
    assert v == pytest.approx(case["lnl"], rel=1e-12)
    np.testing.assert_allclose(site, case["site_lnl"], rtol=1e-11, atol=1e-12)


@pytest.mark.parametrize("case", GOLD["likelihood"], ids=lambda c: f"T{c['T']}S{c['S']}")
def test_tip_encoding_matches_golden(case):
    T, S = case["T"], case["S"]
    codes = np.array(case["codes"], dtype=np.uint8).reshape(T, S)
    inv, ch = oracle.tip_encode(codes)
    np.testing.assert_array_equal(inv, case["is_inv"])
    np.testing.assert_array_equal(ch, case["inv_char"])


def test_tip_encoding_quirks():
    codes = np.array([[20, 5, 20, 21, 3],
                      [20, 5, 5, 21, 3],
                      [20, 5, 5, 21, 4]], dtype=np.uint8)
    inv, ch = oracle.tip_encode(codes)
    # all-gap column is invariant with character 0; gap differs from residue
    np.testing.assert_array_equal(inv, [1, 1, 0, 1, 0])
    np.testing.assert_array_equal(ch, [0, 5, 0, 0, 0])


@pytest.mark.parametrize("case", GOLD["likelihood"], ids=lambda c: f"T{c['T']}S{c['S']}")
def test_ln_prior_matches_golden(case):
    v = oracle.ln_prior(case["T"], case["S"], case["R"], case["lg"], case["branch"],
                        case["shape"], case["base"], np.array(case["logits"]).reshape(case["K"], 20),
                        case["counts"])
    assert v == pytest.approx(case["ln_prior"], rel=1e-12)


@pytest.mark.parametrize("case", GOLD["next_step"], ids=lambda c: f"n{len(c['lnl'])}")
def test_next_step_matches_golden(case):
    rw, nw, ess, temp = oracle.next_step(case["raw_w"], np.array(case["lnl"]), case["target"],
                                         case["last"])
    assert temp == case["temp"]
    np.testing.assert_allclose(rw, case["raw_w_out"], rtol=1e-13)
    np.testing.assert_allclose(nw, case["norm_w"], rtol=1e-10, atol=1e-300)
    assert ess == pytest.approx(case["ess"], rel=1e-10)


def test_two_taxon_pulley_closed_form():
    # 2 tips under the root: L = sum_i pi_i P(t1)_{i a} P(t2)_{i b} = pi_a P(t1+t2)_{a b}
    rng = np.random.default_rng(11)
    base = rng.normal(size=190)
    lg = np.zeros(20)
    lg[:19] = rng.normal(size=19)
    pi = oracle.softmax20(lg)
    S = 20 * 20
    codes = np.array([[a for a in range(20) for b in range(20)],
                      [b for a in range(20) for b in range(20)]], dtype=np.uint8)
    # a 2-taxon tree is not buildable by the particle code (T >= 3), so use T=3
    # with a zero-length third tip that is a gap everywhere.
    codes3 = np.vstack([codes, np.full((1, S), 20, dtype=np.uint8)])
    parent = np.array([3, 4, 4, -1, 3], dtype=np.int32)   # (t0,(t1,t2)) rooted at 3
    branch = np.array([0.13, 0.21, 0.05, 0.0, 0.0])
    v, site = oracle.lnl(codes3, parent, branch, base, lg[None, :], np.zeros(S, np.int32), 0.0,
                         [1.0], site_out=True)
    P = oracle.transition(base, pi, 0.13 + 0.21)
    expect = np.log(np.array([pi[a] * P[a, b] for a in range(20) for b in range(20)]))
    np.testing.assert_allclose(site, expect, rtol=1e-12, atol=1e-12)


def test_reroot_invariance():
    # moving the root along an edge leaves a reversible model's likelihood unchanged
    rng = np.random.default_rng(5)
    T, S = 4, 60
    codes = rng.integers(0, 21, size=(T, S)).astype(np.uint8)
    base = rng.normal(size=190)
    lg = np.zeros((1, 20))
    lg[0, :19] = rng.normal(size=19)
    assign = np.zeros(S, np.int32)
    # ((0,1)5,(2,3)6)4 with the internal edge split 0.1 + 0.2
    p1 = np.array([5, 5, 6, 6, -1, 4, 4], dtype=np.int32)
    b1 = np.array([0.1, 0.2, 0.3, 0.05, 0.0, 0.1, 0.2])
    # same unrooted tree, internal edge split 0.25 + 0.05
    b2 = b1.copy()
    b2[5], b2[6] = 0.25, 0.05
    l1 = oracle.lnl(codes, p1, b1, base, lg, assign, 0.0, [1.0])
    l2 = oracle.lnl(codes, p1, b2, base, lg, assign, 0.0, [1.0])
    assert l1 == pytest.approx(l2, rel=1e-12)


def test_all_gap_site_is_zero_without_invariants():
    T, S = 5, 3
    codes = np.full((T, S), 20, dtype=np.uint8)
    parent = np.array([5, 5, 6, 7, 7, 6, 8, 8, -1], dtype=np.int32)
    branch = np.full(9, 0.1)
    branch[8] = 0.0
    lg = np.zeros((1, 20))
    v, site = oracle.lnl(codes, parent, branch, oracle.lg_base(), lg, np.zeros(S, np.int32),
                         0.0, [0.5, 1.5], site_out=True)
    # log(sum_r exp(0)) = log R: the reference has no 1/R weight
    np.testing.assert_allclose(site, np.log(2.0), atol=1e-13)


def test_split_set_known_answer():
    """((0,1),(2,3)) rooted at node 6: tips and both cherries; the root's two
    children give the same canonical split, counted once (Tree.cpp:485-541)."""
    from oracle import splits
    parent = [4, 4, 5, 5, 6, 6, -1]
    got = splits.split_set(parent, 4)
    want = {0b0001, 0b1101, 0b1011, 0b0111, 0b0011}
    assert got == {(b, 0) for b in want}
    post = splits.split_posteriors([parent, parent, [4, 5, 4, 5, 6, 6, -1]], 4)
    assert post[(0b0011, 0)] == pytest.approx(2 / 3)
    assert post[(0b0101, 0)] == pytest.approx(1 / 3)
    assert post[(0b0001, 0)] == pytest.approx(1.0)

"""Class-local refreshes: an edit of one class's stationary logits (the
stationary move, Particle.cpp:734-742) rebuilds that class alone -- its
spectral decomposition, its matrices and its sites' partials, into that
class's other workspaces -- while the node workspace indices, and every other
class, stay put. Every step of a random walk of class edits, branch edits and
both together, with random accepts and rejects, must give the oracle's
log-likelihood, per particle and per site, and the matrices the oracle builds."""
import numpy as np
import pytest

import oracle
import smccat
from smccat import workload

pytestmark = pytest.mark.gpu

CFG = workload.WorkloadConfig("cls_local", T=9, S=160, R=4, particles=4, iterations=1, lg=False,
                              invar=True, cat=True, pinv=0.1, k_range=(3, 6), seed=61)


def ref(codes, st, i):
    K = int(st["num_classes"][i])
    rates = oracle.discretize_gamma(st["shape"][i], CFG.R)
    return oracle.lnl(codes, st["parent"][i], st["branch"][i], st["base"][i], st["logits"][i][:K],
                      st["assign"][i], st["pinv"][i], rates, site_out=True)


@pytest.mark.parametrize("precision", [smccat.PREC_FP64, smccat.PREC_FP32], ids=["fp64", "fp32"])
def test_class_edits_with_accept_reject(precision):
    rng = np.random.default_rng(CFG.seed)
    codes, _ = workload.simulate_alignment(CFG, rng)
    st = workload.make_particles(CFG, CFG.particles, rng)
    eng = smccat.Engine(codes, CFG.R, CFG.particles, max_classes=st["logits"].shape[1],
                        invar=True, cat=True, precision=precision)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"], st["logits"],
                      st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    tol = dict(rel=1e-9) if precision == smccat.PREC_FP64 else dict(abs=1e-3)
    committed = {k: v.copy() for k, v in st.items()}
    g = np.random.default_rng(5)
    for step in range(40):
        trial = {k: v.copy() for k, v in committed.items()}
        kind = ["class", "class", "class", "branch", "class+branch"][step % 5]
        for i in range(CFG.particles):
            K = int(trial["num_classes"][i])
            if "class" in kind:
                k = int(g.integers(K))
                trial["logits"][i, k, g.integers(20)] += g.normal() * 0.5
                eng.set_class_logits(i, k, trial["logits"][i, k])
            if "branch" in kind:
                n = int(g.integers(2 * CFG.T - 1))
                if trial["parent"][i, n] >= 0:
                    trial["branch"][i, n] *= np.exp(g.normal() * 0.3)
                    eng.set_branch_lengths(i, [n], [trial["branch"][i, n]])
        eng.refresh()
        got = eng.lnl()
        for i in range(CFG.particles):
            lnl, site = ref(codes, trial, i)
            assert got[i] == pytest.approx(lnl, **tol), (step, kind, i)
            if precision == smccat.PREC_FP64:
                np.testing.assert_allclose(eng.site_lnl(i), site, rtol=1e-9, atol=1e-9)
        mask = (g.random(CFG.particles) < 0.5).astype(np.uint8)
        eng.accept(mask)
        for i in range(CFG.particles):
            if mask[i]:
                for key in committed:
                    committed[key][i] = trial[key][i]
        got = eng.lnl()
        for i in range(CFG.particles):
            assert got[i] == pytest.approx(ref(codes, committed, i)[0], **tol), (step, "after accept", i)
    # The matrices of every class, after all the flips, are the oracle's.
    if precision == smccat.PREC_FP64:
        for i in range(CFG.particles):
            K = int(committed["num_classes"][i])
            rates = oracle.discretize_gamma(committed["shape"][i], CFG.R)
            for k in range(K):
                pi = oracle.softmax20(committed["logits"][i, k])
                for n in (0, CFG.T + 1):
                    if committed["parent"][i, n] < 0:
                        continue
                    P = eng.transition_matrix(i, k, n, 2)
                    Q = oracle.transition(committed["base"][i], pi, committed["branch"][i, n] * rates[2])
                    np.testing.assert_allclose(P, Q, atol=1e-13)
    # A full rebuild reproduces the value kept incrementally.
    before = eng.lnl()
    eng.refresh(full=True)
    np.testing.assert_allclose(eng.lnl(), before, rtol=1e-12 if precision == smccat.PREC_FP64 else 1e-6)
    eng.close()

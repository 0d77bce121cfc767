"""Generate the golden fixtures that pin the oracle (tests/golden/*.json).

This script is an independent numpy/scipy restatement of the reference's
likelihood path that follows the reference's own numerical route wherever a
third-party library does the work there:

* LG exchangeabilities are parsed from the reference source itself
  (src/analysis/RateMatrices.hpp:7-95) and flattened in its lower-triangle
  order (RateMatrices.hpp:97-111).
* discretizeGamma (src/core/Miscellaneous.hpp:22-37) uses Boost's gamma
  quantile; here scipy.stats.gamma.ppf stands in for it.
* recomputeEigens / recomputeTransitionProbs
  (src/analysis/TransitionProbabilityClass.cpp:50-95) use Eigen's general
  complex EigenSolver and an explicit inverse; here numpy.linalg.eig (LAPACK
  dgeev) and numpy.linalg.inv, then P = Re(V diag(exp(lambda t r)) V^-1).
* refreshLikelihood(true) (src/analysis/Particle.cpp:530-675): per-node
  max-rescaling, log-sum-exp over rates without a 1/R weight, +I mixing.
* Tip encoding / invariance (Particle.cpp:44-73), lnPrior (Particle.cpp:484-517)
  and computeNextStep (Miscellaneous.hpp:42-109).

Run from the repository root:
    python tests/golden/make_golden.py <Smc-CAT checkout>
(or with the checkout in the environment variable SMCCAT_REFERENCE). It needs
the reference checkout only for the LG table, read from
src/analysis/RateMatrices.hpp inside it; the fixtures it writes are committed
so the tests never read the reference.
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np
from scipy import stats

HERE = os.path.dirname(os.path.abspath(__file__))
LG_SOURCE = os.path.join("src", "analysis", "RateMatrices.hpp")


def reference_root():
    """The Smc-CAT checkout: the first argument, else $SMCCAT_REFERENCE."""
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SMCCAT_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py <Smc-CAT checkout>  (or set SMCCAT_REFERENCE)")
    return root


def parse_lg(path):
    txt = open(path).read()
    m = np.full((20, 20), np.nan)
    for i, j, v in re.findall(r"m\(\s*(\d+),\s*(\d+)\)\s*=\s*([0-9.]+);", txt):
        m[int(i), int(j)] = float(v)
    assert not np.isnan(m).any()
    vec = [m[i, j] for i in range(1, 20) for j in range(i)]
    return np.array(vec)


def discretize_gamma(shape, R):
    q = stats.gamma.ppf((2 * np.arange(R) + 1) / (2.0 * R), shape, scale=1.0 / shape)
    return q * (R / q.sum())


def rate_matrix(base, pi):
    Q = np.zeros((20, 20))
    c = 0
    for i in range(1, 20):
        for j in range(i):
            Q[i, j] = Q[j, i] = np.exp(base[c])
            c += 1
    Q = Q * pi[None, :]
    np.fill_diagonal(Q, 0.0)
    np.fill_diagonal(Q, -Q.sum(axis=1))
    mean = np.sum(-np.diag(Q) * pi)
    return Q / mean


def softmax(lg):
    e = np.exp(lg)
    return e / e.sum()


def transition_general(Q, t):
    w, V = np.linalg.eig(Q)
    Vi = np.linalg.inv(V)
    return np.real(V @ np.diag(np.exp(w * t)) @ Vi)


def random_tree(rng, T):
    """Reference-style random rooted binary tree (Tree.cpp:10-77): start from a
    root with tips 0 and 1, then repeatedly split the branch above a random
    existing tip. Internal ids follow creation order from T (root = T)."""
    parent = {}
    nodes_internal = ["root"]
    parent[0] = "root"
    parent[1] = "root"
    tips = [0, 1]
    for i in range(2, T):
        tip = tips[int(rng.random() * i)]
        new_int = "n%d" % i
        nodes_internal.append(new_int)
        parent[new_int] = parent[tip]
        parent[tip] = new_int
        parent[i] = new_int
        tips.append(i)
    ids = {name: T + k for k, name in enumerate(nodes_internal)}
    N = 2 * T - 1
    par = np.full(N, -1, dtype=np.int64)
    for ch, p in parent.items():
        cid = ch if isinstance(ch, int) else ids[ch]
        par[cid] = ids[p]
    branch = rng.exponential(0.1, size=N)
    branch[ids["root"]] = 0.0
    return par, branch


def postorder(par):
    N = len(par)
    kids = [[] for _ in range(N)]
    root = -1
    for n, p in enumerate(par):
        if p < 0:
            root = n
        else:
            kids[p].append(n)
    out = []

    def rec(n):
        for c in sorted(kids[n]):
            rec(c)
        out.append(n)

    rec(root)
    return out, kids, root


def tip_encode(codes):
    T, S = codes.shape
    inv = np.all(codes == codes[0:1, :], axis=0).astype(float)
    ch = np.where((inv == 1.0) & (codes[0] < 20), codes[0], 0).astype(int)
    return inv, ch


def lnl_reference(codes, par, branch, base, logits, assign, pinv, rates):
    T, S = codes.shape
    R = len(rates)
    N = 2 * T - 1
    K = logits.shape[0]
    post, kids, root = postorder(par)
    pis = [softmax(logits[k]) for k in range(K)]
    P = np.zeros((K, N, R, 20, 20))
    for k in range(K):
        Q = rate_matrix(base, pis[k])
        for n in range(N):
            for r in range(R):
                P[k, n, r] = transition_general(Q, branch[n] * rates[r])
    CL = np.zeros((N, S, R, 20))
    resc = np.zeros((N, S, R))
    for t in range(T):
        for s in range(S):
            c = codes[t, s]
            if c < 20:
                CL[t, s, :, c] = 1.0
            else:
                CL[t, s, :, :] = 1.0
    for n in post:
        if n < T:
            continue
        acc = np.ones((S, R, 20))
        for d in kids[n]:
            for k in range(K):
                mem = np.where(assign == k)[0]
                for r in range(R):
                    acc[mem, r, :] *= CL[d, mem, r, :] @ P[k, d, r].T
        mx = acc.max(axis=2)
        CL[n] = acc / mx[:, :, None]
        resc[n] = np.log(mx)
    inv, ch = tip_encode(codes)
    site = np.zeros(S)
    for s in range(S):
        k = assign[s]
        pik = pis[k]
        logs = np.log(CL[root, s] @ pik) + resc[:, s, :].sum(axis=0)
        mx = logs.max()
        lse = mx + np.log(np.exp(logs - mx).sum())
        v = np.exp(lse) * (1 - pinv) + pinv * pik[ch[s]] * inv[s]
        site[s] = np.log(v)
    return site.sum(), site


def ln_prior_exact(T, S, R, lg, branch, shape, base, logits, counts, alpha=0.01):
    from math import lgamma
    N = 2 * T - 1
    lnp = np.log(stats.gamma.pdf(branch.sum(), N - 1, scale=0.1))
    if R > 1:
        lnp += np.log(stats.gamma.pdf(shape, 3.0, scale=2.0))
    if not lg:
        lnp += np.sum(np.log(stats.norm.pdf(base)))
    lnp += np.log(alpha) * len(counts)
    for k in range(len(counts)):
        lnp += np.sum(np.log(stats.norm.pdf(logits[k])))
        lnp += lgamma(counts[k])
    lnp += lgamma(alpha) - lgamma(alpha + S)
    return float(lnp)


def next_step(raw_w, lnl, target, last):
    raw_w = np.array(raw_w, dtype=float)
    n = len(raw_w)

    def ess(temp):
        tw = raw_w + (temp - last) * lnl
        e = np.exp(tw - tw.max())
        e /= e.sum()
        return 1.0 / np.sum(e * e)

    lo, hi = last, 1.0
    while hi - lo > 1e-5:
        mid = 0.5 * (lo + hi)
        if ess(mid) > target:
            lo = mid
        else:
            hi = mid
    raw_w = raw_w + (hi - last) * lnl
    nw = np.exp(raw_w - raw_w.max())
    nw /= nw.sum()
    return raw_w, nw, 1.0 / np.sum(nw * nw), hi


def simulate_codes(rng, T, S, gap_frac=0.05, special=True):
    codes = rng.integers(0, 20, size=(T, S))
    # a few nearly-conserved columns so invariance is exercised
    for s in range(0, S, 7):
        codes[:, s] = codes[0, s]
    mask = rng.random((T, S)) < gap_frac
    codes[mask] = 20
    if special and S >= 6:
        codes[:, 1] = 20            # all-gap column: invariant, invChar 0
        codes[:, 2] = 5             # all-residue column: invariant, invChar 5
        codes[0, 3] = 20            # gap vs residue: not invariant
        codes[1:, 3] = 5
        codes[:, 4] = 21            # all 'X'
        codes[2, 5] = 22            # a '?'
    return codes.astype(np.uint8)


def main():
    rng = np.random.default_rng(20261203)
    out = {}
    lg = parse_lg(os.path.join(reference_root(), LG_SOURCE))
    out["lg_base"] = lg.tolist()

    gam = []
    for shape in [0.05, 0.2, 0.5, 0.8, 1.0, 2.5, 6.0, 30.0]:
        for R in [1, 2, 4, 8]:
            gam.append({"shape": shape, "R": R, "rates": discretize_gamma(shape, R).tolist()})
    out["discretize_gamma"] = gam
    qs = []
    for a in [0.05, 0.5, 0.8, 3.0, 47.0]:
        for p in [1e-6, 0.125, 0.375, 0.5, 0.875, 0.999]:
            qs.append({"a": a, "p": p, "x": float(stats.gamma.ppf(p, a))})
    out["gamma_ppf"] = qs

    trans = []
    for case in range(6):
        base = lg if case % 2 == 0 else rng.normal(size=190)
        logits = np.zeros(20)
        logits[:19] = rng.normal(size=19) * (1.0 + case * 0.3)
        pi = softmax(logits)
        Q = rate_matrix(base, pi)
        for t in [0.0, 1e-3, 0.05, 0.3, 2.0, 10.0]:
            P = transition_general(Q, t)
            trans.append({"base": base.tolist(), "logits": logits.tolist(), "t": t,
                          "P": P.ravel().tolist()})
    out["transition"] = trans

    cases = []
    specs = [
        dict(T=5, S=30, R=1, K=1, lg=True, pinv=0.0),
        dict(T=6, S=40, R=4, K=1, lg=False, pinv=0.2),
        dict(T=7, S=50, R=4, K=3, lg=False, pinv=0.1),
        dict(T=4, S=12, R=2, K=2, lg=True, pinv=0.35),
        dict(T=9, S=64, R=4, K=5, lg=False, pinv=0.0),
        dict(T=3, S=8, R=3, K=1, lg=False, pinv=0.5),
    ]
    for sp in specs:
        T, S, R, K = sp["T"], sp["S"], sp["R"], sp["K"]
        codes = simulate_codes(rng, T, S)
        par, branch = random_tree(rng, T)
        base = lg.copy() if sp["lg"] else rng.normal(size=190)
        logits = np.zeros((K, 20))
        logits[:, :19] = rng.normal(size=(K, 19))
        assign = np.arange(S) % K
        rng.shuffle(assign)
        shape = float(rng.gamma(3.0, 2.0))
        rates = discretize_gamma(shape, R) if R > 1 else np.ones(1)
        tot, site = lnl_reference(codes, par, branch, base, logits, assign, sp["pinv"], rates)
        inv, ch = tip_encode(codes)
        counts = np.bincount(assign, minlength=K)
        prior = ln_prior_exact(T, S, R, sp["lg"], branch, shape, base, logits, counts)
        cases.append({
            "T": T, "S": S, "R": R, "K": K, "lg": sp["lg"], "pinv": sp["pinv"],
            "codes": codes.ravel().tolist(), "parent": par.tolist(), "branch": branch.tolist(),
            "base": base.tolist(), "logits": logits.ravel().tolist(),
            "assign": assign.tolist(), "shape": shape, "rates": rates.tolist(),
            "lnl": float(tot), "site_lnl": site.tolist(),
            "is_inv": inv.tolist(), "inv_char": ch.tolist(), "counts": counts.tolist(),
            "ln_prior": prior,
        })
    out["likelihood"] = cases

    steps = []
    for n, spread in [(16, 5.0), (64, 50.0), (200, 400.0)]:
        raw = np.full(n, -np.log(n))
        lnl = rng.normal(size=n) * spread - 1000.0
        rw, nw, ess, temp = next_step(raw, lnl, 0.6 * n, 0.0)
        steps.append({"raw_w": raw.tolist(), "lnl": lnl.tolist(), "target": 0.6 * n,
                      "last": 0.0, "raw_w_out": rw.tolist(), "norm_w": nw.tolist(),
                      "ess": float(ess), "temp": float(temp)})
    out["next_step"] = steps

    path = os.path.join(HERE, "golden.json")
    with open(path, "w") as f:
        json.dump(out, f)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()

"""Seeded synthetic workloads for the Smc-CAT likelihood path.

The reference ships no data set (its only input path, Settings.hpp:29, is a
local file that is not distributed), so every workload is simulated from a
seed:

* a random rooted binary tree grown like the reference's ``Tree(rng, n)``
  (Tree.cpp:10-77: repeatedly split the edge above a random existing tip),
  branch lengths ~ Exp(mean 0.1) (Tree.cpp:346);
* site rates drawn uniformly from the discrete-gamma categories
  (``discretizeGamma``), invariant sites with probability pinv;
* root states from pi, child states sampled from the rows of P(t r);
* about 2% of cells replaced by gaps (code 20).

Particle states follow the reference's initialisation (Particle.cpp:81-166):
random tree, LG or N(0,1) exchangeabilities, 19 N(0,1) logits + 0 per class,
pinv ~ U(0,1) with +I, shape ~ Gamma(3, 2) with R > 1.

The gamma discretisation and the LG table come from the engine library by
default. A caller that must not load it (the CPU timing of the reference's
path) passes its own ``gamma_fn(shape, R)`` and ``lg_fn()``; the values are
the same (both restate Miscellaneous.hpp:22-37 and RateMatrices.hpp:7-111).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def _sources(gamma_fn, lg_fn):
    """The gamma-discretisation and LG-table functions to use: the given ones,
    else the engine library's (imported only when one is missing)."""
    if gamma_fn is None or lg_fn is None:
        from . import discretize_gamma, lg_exchangeabilities
        gamma_fn = gamma_fn or discretize_gamma
        lg_fn = lg_fn or lg_exchangeabilities
    return gamma_fn, lg_fn


@dataclass
class WorkloadConfig:
    name: str
    T: int
    S: int
    R: int
    particles: int
    iterations: int
    lg: bool
    invar: bool
    cat: bool
    alpha: float = 0.8
    pinv: float = 0.0
    dp_concentration: float = 1.0
    k_range: tuple | None = None   # per-particle class count range (uneven CAT)
    seed: int = 1
    extra: dict = field(default_factory=dict)


CONFIGS = {
    1: WorkloadConfig("lg_g4_16x500", T=16, S=500, R=4, particles=64, iterations=5, lg=True,
                      invar=False, cat=False, alpha=0.8, seed=1),
    2: WorkloadConfig("gtr_g4_i_48x2000", T=48, S=2000, R=4, particles=256, iterations=10,
                      lg=False, invar=True, cat=False, alpha=0.5, pinv=0.1, seed=2),
    3: WorkloadConfig("cat_gtr_g4_64x5000", T=64, S=5000, R=4, particles=1024, iterations=10,
                      lg=False, invar=False, cat=True, alpha=0.8, dp_concentration=5.0, seed=3),
    4: WorkloadConfig("cat_uneven_100x10000", T=100, S=10000, R=4, particles=2048, iterations=10,
                      lg=False, invar=False, cat=True, alpha=0.8, dp_concentration=5.0,
                      k_range=(8, 120), seed=4),
    5: WorkloadConfig("cat_gtr_g4_i_128x20000", T=128, S=20000, R=4, particles=4096,
                      iterations=10, lg=False, invar=True, cat=True, alpha=0.8, pinv=0.1,
                      dp_concentration=5.0, seed=5),
}


def random_tree(rng: np.random.Generator, T: int):
    """Reference-style random rooted binary tree; returns (parent, branch).

    Tips are 0..T-1, internal nodes T..2T-2 in creation order (root = T).
    """
    N = 2 * T - 1
    parent = np.full(N, -1, dtype=np.int32)
    parent[0] = parent[1] = T
    nxt = T + 1
    for i in range(2, T):
        tip = int(rng.random() * i)
        new = nxt
        nxt += 1
        parent[new] = parent[tip]
        parent[tip] = new
        parent[i] = new
    branch = rng.exponential(0.1, size=N)
    branch[T] = 0.0
    return parent, branch


def rate_matrix(base, pi):
    """Normalised Q(i,j) = exp(b_ij) pi_j (TransitionProbabilityClass.cpp:50-75)."""
    E = np.zeros((20, 20))
    il = np.tril_indices(20, -1)
    # tril_indices enumerates (i, j<i) row by row: the reference's order.
    E[il] = np.exp(base)
    E = E + E.T
    Q = E * pi[None, :]
    np.fill_diagonal(Q, -Q.sum(axis=1))
    return Q / np.sum(-np.diag(Q) * pi)


def transition_batch(base, pi, t):
    """P(t) for a vector of times via the symmetrised eigendecomposition."""
    Q = rate_matrix(base, pi)
    sq = np.sqrt(pi)
    Sm = sq[:, None] * Q / sq[None, :]
    Sm = 0.5 * (Sm + Sm.T)
    lam, U = np.linalg.eigh(Sm)
    L = U / sq[:, None]
    Rm = (U * sq[:, None]).T
    ex = np.exp(np.multiply.outer(np.asarray(t, dtype=float), lam))
    P = np.einsum("im,tm,mj->tij", L, ex, Rm)
    return np.clip(P, 0.0, None)


def _postorder_children(parent):
    N = len(parent)
    kids = [[] for _ in range(N)]
    root = -1
    for n, p in enumerate(parent):
        if p < 0:
            root = n
        else:
            kids[p].append(n)
    order = []
    stack = [root]
    while stack:
        n = stack.pop()
        order.append(n)
        stack.extend(kids[n])
    return order, root  # pre-order


def crp_assign(rng, S, concentration, max_classes=None):
    assign = np.zeros(S, dtype=np.int32)
    counts = []
    for i in range(S):
        w = np.array(counts + [concentration], dtype=float)
        if max_classes is not None and len(counts) >= max_classes:
            w[-1] = 0.0
        k = rng.choice(len(w), p=w / w.sum())
        if k == len(counts):
            counts.append(0)
        counts[k] += 1
        assign[i] = k
    return assign, len(counts)


def simulate_alignment(cfg: WorkloadConfig, rng: np.random.Generator | None = None,
                       gamma_fn=None, lg_fn=None):
    """Simulate (codes [T][S] uint8, truth dict) for a workload config."""
    discretize_gamma, lg_exchangeabilities = _sources(gamma_fn, lg_fn)
    rng = np.random.default_rng(cfg.seed) if rng is None else rng
    T, S, R = cfg.T, cfg.S, cfg.R
    parent, branch = random_tree(rng, T)
    if cfg.lg:
        base = lg_exchangeabilities()
    else:
        base = np.log(rng.dirichlet(np.ones(190)))
    if cfg.cat:
        assign, K = crp_assign(rng, S, cfg.dp_concentration)
        pis = rng.dirichlet(np.ones(20), size=K)
    else:
        assign, K = np.zeros(S, dtype=np.int32), 1
        pis = rng.dirichlet(5.0 * np.ones(20), size=1)
    rates = discretize_gamma(cfg.alpha, R) if R > 1 else np.ones(1)
    rate_cat = rng.integers(0, R, size=S)
    invariant = rng.random(S) < cfg.pinv
    order, root = _postorder_children(parent)
    N = 2 * T - 1
    states = np.zeros((N, S), dtype=np.int64)
    for k in range(K):
        sites = np.where(assign == k)[0]
        if len(sites) == 0:
            continue
        pi = pis[k]
        cum_pi = np.cumsum(pi)
        states[root, sites] = np.minimum(np.searchsorted(cum_pi, rng.random(len(sites))), 19)
        # P for every (node, rate): [N, R, 20, 20]
        tt = (branch[:, None] * rates[None, :]).ravel()
        P = transition_batch(base, pi, tt).reshape(N, R, 20, 20)
        cum = np.cumsum(P, axis=3)
        for n in order:
            if n == root:
                continue
            par = parent[n]
            rows = cum[n, rate_cat[sites], states[par, sites]]     # [len, 20]
            u = rng.random(len(sites))[:, None] * rows[:, -1:]
            states[n, sites] = np.minimum((rows < u).sum(axis=1), 19)
        inv_sites = sites[invariant[sites]]
        if len(inv_sites):
            c = np.minimum(np.searchsorted(cum_pi, rng.random(len(inv_sites))), 19)
            states[:, inv_sites] = c[None, :]
    codes = states[:T].astype(np.uint8)
    gaps = rng.random((T, S)) < 0.02
    codes[gaps] = 20
    truth = dict(parent=parent, branch=branch, base=base, assign=assign, K=K, pis=pis,
                 rates=rates)
    return codes, truth


def make_particles(cfg: WorkloadConfig, n: int, rng: np.random.Generator, kmax: int | None = None,
                   lg_fn=None):
    """Particle states drawn like the reference's initialisation (packed arrays)."""
    lg_exchangeabilities = _sources(None, lg_fn)[1] if cfg.lg else None
    T, S, R = cfg.T, cfg.S, cfg.R
    N = 2 * T - 1
    if cfg.cat:
        if cfg.k_range is not None:
            ks = rng.integers(cfg.k_range[0], cfg.k_range[1] + 1, size=n)
        else:
            ks = np.maximum(1, rng.poisson(cfg.dp_concentration * np.log1p(S / cfg.dp_concentration), size=n))
    else:
        ks = np.ones(n, dtype=np.int64)
    kmax = int(ks.max()) if kmax is None else kmax
    parent = np.zeros((n, N), np.int32)
    branch = np.zeros((n, N))
    base = np.zeros((n, 190))
    logits = np.zeros((n, kmax, 20))
    assign = np.zeros((n, S), np.int32)
    for i in range(n):
        parent[i], branch[i] = random_tree(rng, T)
        base[i] = lg_exchangeabilities() if cfg.lg else rng.normal(size=190)
        K = int(ks[i])
        logits[i, :K, :19] = rng.normal(size=(K, 19))
        if K > 1:
            a = rng.integers(0, K, size=S)
            a[:K] = rng.permutation(K)   # every class non-empty
            assign[i] = a
    pinv = rng.random(n) if cfg.invar else np.zeros(n)
    shape = rng.gamma(3.0, 2.0, size=n) if R > 1 else np.ones(n)
    return dict(parent=parent, branch=branch, base=base, num_classes=ks.astype(np.int32),
                logits=logits, assign=assign, pinv=pinv, shape=shape)

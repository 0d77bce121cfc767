"""Split posteriors of a particle population -- TEST INFRASTRUCTURE ONLY.

A plain-Python restatement, used only by the tests, of:

* ``Tree::computeSplits`` / ``Tree::getSplitSet`` (src/analysis/Tree.cpp:485-541):
  the taxon set below every non-root node, canonicalised so that taxon 0 is a
  member (the set is complemented otherwise), each distinct set once per tree;
* ``computeSplitPosteriors`` (src/core/Miscellaneous.hpp:115-150): the sum over
  particles of each split's weight, weights either given (normalised SMC
  weights) or 1/count (a resampled assignment list).

A split is returned as the pair (bits of taxa 0..63, bits of taxa 64..127).
"""
from __future__ import annotations


def split_set(parent, T: int) -> set:
    """Canonical clade sets of one tree given as a parent array over 2T-1 nodes."""
    N = 2 * T - 1
    kids = [[] for _ in range(N)]
    root = -1
    for n in range(N):
        if parent[n] < 0:
            root = n
        else:
            kids[parent[n]].append(n)
    full = (1 << T) - 1
    clade = [0] * N

    def fill(n):
        if n < T:
            clade[n] = 1 << n
        else:
            for k in kids[n]:
                fill(k)
            clade[n] = clade[kids[n][0]] | clade[kids[n][1]]

    fill(root)
    out = set()
    for n in range(N):
        if n == root:
            continue
        c = clade[n] if clade[n] & 1 else full & ~clade[n]
        out.add((c & ((1 << 64) - 1), c >> 64))
    return out


def split_posteriors(parents, T: int, weights=None) -> dict:
    """{split: posterior} over the trees `parents` (one parent array each)."""
    n = len(parents)
    acc: dict = {}
    for i, par in enumerate(parents):
        w = (1.0 / n) if weights is None else float(weights[i])
        for s in split_set(par, T):
            acc[s] = acc.get(s, 0.0) + w
    return acc

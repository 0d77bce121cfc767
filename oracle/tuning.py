"""Systematic resampling and proposal tuning of the SMC step -- TEST
INFRASTRUCTURE ONLY.

A numpy restatement, used only by the tests, of src/main.cpp:176-291:
systematic resampling with one uniform draw (main.cpp:178-192) and the proposal
tuning over the resampled population (main.cpp:197-291): population variances
(boost::accumulators tag::variance) of log shape, of log branch length over
every non-root branch and of every class's 20 stationary logits, the mean pInvar,
and the uncentred X^T X of the GTR base vectors, scaled by 2.38^2/190 * 0.21,
shrunk by 0.2 toward its mean diagonal, plus 1e-6 I, and its Cholesky factor.
"""
from __future__ import annotations

import numpy as np


def systematic_resample(w, u: float) -> list:
    n = len(w)
    out = []
    cumulative = w[0]
    k = 0
    ruler = u / n
    step = 1.0 / n
    while len(out) < n:
        if ruler <= cumulative:
            out.append(k)
            ruler += step
        else:
            k += 1
            if k >= n:
                k = n - 1
                cumulative = 1.0
            else:
                cumulative += w[k]
    return out


def tune(states: dict, ancestors, gtr: bool) -> dict:
    """states: the engine's packed particle arrays (get_particles layout)."""
    log_shape, log_branch, logits, pinv, X = [], [], [], [], []
    for a in ancestors:
        par = states["parent"][a]
        root = int(np.where(par < 0)[0][0])
        log_shape.append(np.log(states["shape"][a]))
        pinv.append(states["pinv"][a])
        log_branch.extend(np.log(np.delete(states["branch"][a], root)))
        K = int(states["num_classes"][a])
        logits.extend(states["logits"][a][:K].ravel())
        X.append(states["base"][a])
    out = {"shape_delta": max(0.5 * np.var(log_shape), 0.01),
           "scale_delta": max(np.var(log_branch), 0.01),
           "stationary_delta": max(np.var(logits), 0.01),
           "pinv_mean": float(np.mean(pinv))}
    if gtr:
        X = np.array(X)
        cov = X.T @ X * (2.38 * 2.38) / 190.0 * 0.21
        shrink = np.trace(cov) / 190.0 * 0.2
        cov = cov * 0.8 + np.eye(190) * (shrink + 1e-6)
        out["rate_matrix_delta"] = max(shrink, 0.01)
        out["cholesky"] = np.linalg.cholesky(cov)
    return out

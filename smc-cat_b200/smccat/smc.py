"""The SMC loop of the reference (src/main.cpp:147-336) over the engine's C-ABI.

Each step: computeNextStep on the device-resident log-likelihoods (temperature
bisection to the target ESS, weight update; ``Engine.smc_step``); when the ESS
falls to the threshold, systematic resampling with proposal re-tuning and
ancestor copies (``Engine.resample_tune``), a full refresh, ``Mcmc::operator()``
on every particle (``Engine.rejuvenate``) and, for CAT models, a class
reassignment on a random ``alg8_probability`` fraction of the particles
(main.cpp:296-311); the raw weights restart at -log N.

Reassignment is either the reference's Gibbs move (Neal 8) or the learned
proposal: that arm uses Gibbs for its first ``learned_warmup`` rejuvenation
rounds, trains the MLP on the assignments they leave, then proposes with it
(a Metropolis-Hastings move, so the target is unchanged). The learned move
keeps the class count fixed, so that arm still runs the Gibbs move after the
learned one on every ``gibbs_every``-th round: the class count keeps mixing.

Not in the reference: a running estimate of the log marginal likelihood,
log Z = sum over steps of the change of logsumexp(raw weights) -- the standard
tempered-SMC estimator (raw weights start at -log N, and restart there after
each resample).
"""
from __future__ import annotations

import time

import numpy as np


def _lse(x: np.ndarray) -> float:
    m = float(np.max(x))
    return m + float(np.log(np.sum(np.exp(x - m))))


def run(eng, *, cat: bool, iterations: int = 20, threshold: float = 0.6,
        alg8_probability: float = 0.1, reassign: str = "gibbs", learned_warmup: int = 2,
        learned_updates: int | None = None, gibbs_every: int = 4, seed: int = 0,
        max_steps: int = 100000, sync=None, device_sweep: bool = False) -> dict:
    """Run the loop on all of ``eng``'s particles (loaded and refreshed).
    ``sync`` (optional) is called before reading the wall clock.
    ``device_sweep``: rejuvenate with the whole Mcmc::operator() sweep on the
    device (one CUDA graph, ``Engine.mcmc_sweep``) instead of the host-driven
    lockstep (``Engine.rejuvenate``)."""
    n = eng.P
    rng = np.random.default_rng(seed)
    raw = np.full(n, -np.log(n))
    last, log_z = 0.0, 0.0
    steps = resamples = rounds = 0
    ess = float(n)
    history = []
    moves = {"proposed": 0, "accepted": 0}
    trained = False
    t0 = time.perf_counter()
    while last < 1.0 and steps < max_steps:
        before = _lse(raw)
        raw, norm, ess, temp = eng.smc_step(raw, threshold * n, last)
        log_z += _lse(raw) - before
        steps += 1
        if np.isnan(ess):
            raise RuntimeError("NaN ESS: a log-likelihood came out NaN")  # main.cpp:158-174
        if ess <= threshold * n and temp != 1.0:
            eng.resample_tune(norm, float(rng.random()), copy=True)
            eng.refresh(full=True)
            sweep = eng.mcmc_sweep if device_sweep else eng.rejuvenate
            st = sweep(iterations=iterations, temperature=temp, seed=int(rng.integers(1 << 62)))
            moves["proposed"] += int(np.sum(st["proposed"]))
            moves["accepted"] += int(np.sum(st["accepted"]))
            if cat:
                mask = (rng.random(n) < alg8_probability).astype(np.uint8)
                if mask.any():
                    use_learned = reassign == "learned" and rounds >= learned_warmup
                    if use_learned and not trained:
                        eng.learned_train(epochs=1, batch_sites=512, lr=1e-3,
                                          seed=int(rng.integers(1 << 30)), first=0,
                                          count=min(n, 8))
                        trained = True
                    if use_learned:
                        eng.learned_move(updates=learned_updates or eng.S // 2, temperature=temp,
                                         seed=int(rng.integers(1 << 62)), mask=mask)
                    if not use_learned or (rounds - learned_warmup) % gibbs_every == gibbs_every - 1:
                        eng.gibbs(temperature=temp, seed=int(rng.integers(1 << 62)), mask=mask)
            raw = np.full(n, -np.log(n))
            resamples += 1
            rounds += 1
        history.append((float(temp), float(ess)))
        last = temp
    if sync is not None:
        sync()
    seconds = time.perf_counter() - t0
    return {"log_z": log_z, "steps": steps, "resamples": resamples, "final_ess": float(ess),
            "seconds": seconds, "final_ess_per_s": float(ess) / seconds,
            "mh_acceptance": moves["accepted"] / max(moves["proposed"], 1),
            "temperatures": [h[0] for h in history]}


def run_sharded(eng, *, group=None, device="cpu", cat: bool, iterations: int = 20,
                threshold: float = 0.6, alg8_probability: float = 0.1, seed: int = 0,
                max_steps: int = 100000, sync=None) -> dict:
    """The same loop over a population sharded across ranks (one engine per
    rank, each holding the same number of particles; torch.distributed set
    up by the caller). Every rank keeps the global weight vector: the
    log-likelihoods are all-gathered for computeNextStep, resampling is
    systematic over the whole population, and the surviving states move
    between ranks (smccat.distributed.resample_engine); rejuvenation and
    Gibbs reassignment stay local. The random draws that must agree (the
    resampling uniform, the Gibbs mask) come from one stream seeded alike on
    every rank; each rank's moves use its own."""
    import torch.distributed as dist

    from . import distributed as sd
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    n_local = eng.P
    n = n_local * world
    shared = np.random.default_rng(seed)
    own = np.random.default_rng([seed, rank + 1])
    raw = np.full(n, -np.log(n))
    last, log_z = 0.0, 0.0
    steps = resamples = 0
    ess = float(n)
    t0 = time.perf_counter()
    while last < 1.0 and steps < max_steps:
        before = _lse(raw)
        u = float(shared.random())
        w, temp, ess, resampled = sd.resample_engine(eng, raw, threshold * n, last, u, group, device)
        log_z += _lse(w) - before
        steps += 1
        if np.isnan(ess):
            raise RuntimeError("NaN ESS: a log-likelihood came out NaN")  # main.cpp:158-174
        raw = w
        if resampled:
            raw = np.full(n, -np.log(n))
            resamples += 1
            eng.rejuvenate(iterations=iterations, temperature=temp, seed=int(own.integers(1 << 62)))
            mask = (shared.random(n) < alg8_probability).astype(np.uint8)[rank * n_local:(rank + 1) * n_local]
            if cat and mask.any():
                eng.gibbs(temperature=temp, seed=int(own.integers(1 << 62)), mask=mask)
        last = temp
    if sync is not None:
        sync()
    return {"log_z": log_z, "steps": steps, "resamples": resamples, "final_ess": float(ess),
            "seconds": time.perf_counter() - t0}

"""Particle sharding across GPUs for the SMC step (one process per GPU).

Particles are independent between resampling steps (the reference's
rejuvenation loop, main.cpp:295-312, shares nothing across particles), so each
rank owns a contiguous block of particles in its own engine context and the
likelihood path needs no collective. The SMC step itself has two exchange
points, both here:

* an all-gather of every particle's log-likelihood, so each rank can run
  computeNextStep (Miscellaneous.hpp:42-109) on the global weight vector;
* after systematic resampling (main.cpp:180-195), point-to-point transfers of
  the serialized states of the particles a rank must take over from another
  rank. Conditional likelihoods are never sent: the receiver refreshes.

Collectives go through torch.distributed (NCCL between GPUs, gloo on CPU);
states travel as float64 tensors.
"""
from __future__ import annotations

import numpy as np

STATE_KEYS = ("parent", "branch", "base", "num_classes", "logits", "assign", "pinv", "shape")


def state_width(T: int, S: int, kmax: int) -> int:
    N = 2 * T - 1
    return N + N + 190 + 1 + kmax * 20 + S + 1 + 1


def pack_states(st: dict, T: int, S: int, kmax: int) -> np.ndarray:
    """Serialize packed particle states ([n, ...] arrays) to [n, width] float64."""
    n = len(st["pinv"])
    out = np.zeros((n, state_width(T, S, kmax)))
    o = 0
    for k, w in (("parent", 2 * T - 1), ("branch", 2 * T - 1), ("base", 190),
                 ("num_classes", 1), ("logits", kmax * 20), ("assign", S), ("pinv", 1),
                 ("shape", 1)):
        out[:, o:o + w] = np.asarray(st[k], dtype=np.float64).reshape(n, w)
        o += w
    return out


def unpack_states(a: np.ndarray, T: int, S: int, kmax: int) -> dict:
    n = a.shape[0]
    st, o = {}, 0
    for k, w, dt in (("parent", 2 * T - 1, np.int32), ("branch", 2 * T - 1, np.float64),
                     ("base", 190, np.float64), ("num_classes", 1, np.int32),
                     ("logits", kmax * 20, np.float64), ("assign", S, np.int32),
                     ("pinv", 1, np.float64), ("shape", 1, np.float64)):
        v = a[:, o:o + w].astype(dt)
        st[k] = v.reshape(n) if w == 1 else (v.reshape(n, kmax, 20) if k == "logits" else v)
        o += w
    return st


def systematic_resample(weights: np.ndarray, u: float) -> np.ndarray:
    """Systematic resampling exactly as main.cpp:180-195 walks it."""
    n = len(weights)
    out = np.empty(n, dtype=np.int64)
    cum, k, m = weights[0], 0, 0
    ruler, step = u / n, 1.0 / n
    while m < n:
        if ruler <= cum:
            out[m] = k
            m += 1
            ruler += step
        else:
            k += 1
            if k >= n:
                k, cum = n - 1, 1.0
            else:
                cum += weights[k]
    return out


def next_step(raw_w: np.ndarray, lnl: np.ndarray, target_ess: float, last_temp: float):
    """computeNextStep on the all-gathered vectors (identical on every rank)."""
    raw_w = np.asarray(raw_w, dtype=np.float64)

    def ess(temp):
        tw = raw_w + (temp - last_temp) * lnl
        e = np.exp(tw - tw.max())
        e /= e.sum()
        return 1.0 / np.sum(e * e)

    lo, hi = last_temp, 1.0
    while hi - lo > 1e-5:
        mid = 0.5 * (lo + hi)
        if ess(mid) > target_ess:
            lo = mid
        else:
            hi = mid
    w = raw_w + (hi - last_temp) * lnl
    nw = np.exp(w - w.max())
    nw /= nw.sum()
    return w, nw, 1.0 / np.sum(nw * nw), hi


def transfer_plan(assign: np.ndarray, per_rank: int):
    """For global destination slot d (owned by rank d // per_rank) the source
    particle is assign[d] (owned by rank assign[d] // per_rank). Returns
    {(src_rank, dst_rank): [(src_local, dst_local), ...]} in slot order."""
    plan = {}
    for d, s in enumerate(assign):
        key = (int(s) // per_rank, d // per_rank)
        plan.setdefault(key, []).append((int(s) % per_rank, d % per_rank))
    return plan


def all_gather_lnl(local_lnl: np.ndarray, group=None, device="cpu") -> np.ndarray:
    import torch
    import torch.distributed as dist
    t = torch.as_tensor(np.ascontiguousarray(local_lnl), dtype=torch.float64, device=device)
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(parts, t, group=group)
    return torch.cat(parts).cpu().numpy()


def exchange_states(local_packed: np.ndarray, assign: np.ndarray, group=None,
                    device="cpu") -> np.ndarray:
    """New local packed states after resampling: local copies need no
    transfer; the rest arrive by send/recv, one message per rank pair, in a
    fixed order on every rank (lower rank sends first within each pair)."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    per_rank = local_packed.shape[0]
    plan = transfer_plan(assign, per_rank)
    out = np.zeros_like(local_packed)
    for (src, dst), pairs in plan.items():
        if src == dst == rank:
            for sl, dl in pairs:
                out[dl] = local_packed[sl]
    for a in range(world):
        for b in range(a + 1, world):
            if rank not in (a, b):
                continue
            for src, dst in ((a, b), (b, a)):
                pairs = plan.get((src, dst))
                if not pairs:
                    continue
                if rank == src:
                    buf = torch.as_tensor(local_packed[[sl for sl, _ in pairs]], device=device)
                    dist.send(buf.contiguous(), dst, group=group)
                else:
                    buf = torch.empty((len(pairs), local_packed.shape[1]), dtype=torch.float64,
                                      device=device)
                    dist.recv(buf, src, group=group)
                    got = buf.cpu().numpy()
                    for i, (_, dl) in enumerate(pairs):
                        out[dl] = got[i]
    return out


def resample_engine(engine, raw_w, target_ess, last_temp, u, group=None, device="cpu"):
    """One SMC weight step for a sharded population: all-gather the
    log-likelihoods, computeNextStep, and if the ESS fell to the target,
    resample systematically and move the surviving states between ranks,
    reload them into `engine` and refresh. Returns (raw_w, temp, ess,
    resampled) with the raw weights updated to the new temperature; after a
    resample the caller restarts them at -log N (main.cpp:309)."""
    lnl = all_gather_lnl(engine.lnl(), group, device)
    w, nw, ess, temp = next_step(raw_w, lnl, target_ess, last_temp)
    if not (ess <= target_ess and temp != 1.0):
        return w, temp, ess, False
    assign = systematic_resample(nw, u)
    st = engine.get_particles()
    packed = pack_states(st, engine.T, engine.S, engine.Kmax)
    new = unpack_states(exchange_states(packed, assign, group, device), engine.T, engine.S,
                        engine.Kmax)
    engine.set_particles(0, new["parent"], new["branch"], new["base"], new["num_classes"],
                         new["logits"], new["assign"], new["pinv"], new["shape"])
    engine.refresh(full=True)
    return w, temp, ess, True

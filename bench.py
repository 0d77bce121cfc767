#!/usr/bin/env python
"""Throughput of the Smc-CAT likelihood hot path on B200.

Workload (default): the FP64 GTR+G4+I configuration, 48 taxa x 2,000 sites,
4 gamma categories, 256 particles, seeded synthetic data. One step = one full
likelihood refresh (the reference's refreshLikelihood(true) after
copyFromSerialized) of every particle: 256 x 2,000 x 4 = 2,048,000
particle*site*category evaluations.

* ``value``  -- device-timed throughput with the particle states resident in HBM.
* ``e2e``    -- the same metric through the public C-ABI with host buffers:
  every step uploads all particle states (smccat_set_particles), refreshes and
  reads the log-likelihoods back (smccat_get_lnl).
* ``roofline`` -- the pruning kernel's algorithmic HBM bytes per launch over its
  CUDA-event duration, against the measured copy bandwidth.
* ``cpu_baseline`` -- the FP64 oracle (the reference's algorithm with its
  OpenMP-over-particles structure) on a bounded sample, all host threads.

``--impl reference`` times that CPU implementation alone as the reference arm.
Multi-GPU (torchrun): every rank holds its own 256 particles; no collective in
the data path (weak scaling); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "smc-cat_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "particle*site*cat lik evals/s"
UNIT = "evals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--cpu-sample", type=int, default=32,
                    help="particles per CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variant", type=int, default=-1,
                    help="pin this pruning-kernel variant instead of autotuning (profiling)")
    ap.add_argument("--particles", type=int, default=0,
                    help="override the particle count (small cases for ncu captures)")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--sweeps", type=int, default=2,
                    help="timed rejuvenation sweeps (0 to skip)")
    ap.add_argument("--sweep-temp", type=float, default=0.5)
    ap.add_argument("--branch-steps", type=int, default=50,
                    help="device-side branch-length MH steps timed as one graph (0 to skip)")
    ap.add_argument("--patterns", type=int, default=1,
                    help="also time the same particles with site-pattern compression")
    ap.add_argument("--mixed", type=int, default=1,
                    help="also time the FP32 (mixed-precision) path on the same particles")
    ap.add_argument("--extra-configs", default="4,5",
                    help="comma-separated CAT configs (e.g. 3,4) to time in particle waves, at "
                         "their full particle counts ('' to skip)")
    ap.add_argument("--extra-particles", type=int, default=0,
                    help="particles for --extra-configs (default: the configuration's)")
    ap.add_argument("--sampler-config", type=int, default=4,
                    help="CAT config on which to compare sampler sweeps/s and ESS/s: plain FP64 + "
                         "Gibbs against FP32 + device graph sweep + learned proposal (0 to skip)")
    ap.add_argument("--sampler-particles", type=int, default=48)
    ap.add_argument("--sampler-sweeps", type=int, default=4,
                    help="timed sweeps of the plain arm")
    ap.add_argument("--sampler-chosen-sweeps", type=int, default=10,
                    help="timed sweeps of the chosen arm (a whole Gibbs period)")
    ap.add_argument("--smc", type=int, default=0,
                    help="run whole SMC analyses (temperature 0 -> 1) on a 16-taxon x 500-site "
                         "CAT workload: plain FP64 + Gibbs against FP32 + learned proposal, "
                         "this many replicate seeds each")
    ap.add_argument("--smc-particles", type=int, default=64)
    ap.add_argument("--smc-iterations", type=int, default=5,
                    help="rejuvenation iterations per resampling round of the --smc analyses")
    ap.add_argument("--smc-alg8", type=float, default=0.1,
                    help="fraction of particles given a class reassignment per round (alg8Probability)")
    ap.add_argument("--gibbs-particles", type=int, default=0,
                    help="particles of a CAT --extra-configs run timed through one Gibbs pass "
                         "and one learned-proposal pass (0 to skip)")
    ap.add_argument("--reassign", type=int, default=0,
                    help="only time the CAT reassignment passes on --sampler-config with this many "
                         "particles (FP64 Gibbs, FP32 learned proposal; two passes each) and print "
                         "that line")
    return ap.parse_args()


def measure_reassign_only(cid, n, local, torch, reps=2):
    """Reassignment passes alone on a CAT configuration, from the sampler
    comparison's start (its particles and class headroom): `reps` FP64 Gibbs
    passes, then on an FP32 context one Gibbs warm-up pass, one epoch of MLP
    training (untimed) and `reps` learned-proposal passes of floor(S/2) updates
    per particle. Wall clock around device-synchronised calls."""
    import smccat
    from smccat import workload
    cfg = workload.CONFIGS[cid]
    codes, _ = workload.simulate_alignment(cfg, np.random.default_rng(cfg.seed))
    st = workload.make_particles(cfg, n, np.random.default_rng(cfg.seed * 7 + 1))
    kmax = st["logits"].shape[1] + 96
    logits = np.zeros((n, kmax, 20))
    logits[:, :st["logits"].shape[1]] = st["logits"]
    out = {"workload": cfg.name, "particles": n, "site_iterations_per_particle": cfg.S // 2}
    for arm, prec in (("gibbs_fp64", smccat.PREC_FP64), ("learned_fp32", smccat.PREC_FP32)):
        eng = smccat.Engine(codes, cfg.R, n, max_classes=kmax, lg=cfg.lg, invar=cfg.invar,
                            cat=cfg.cat, device=local, precision=prec)
        eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"], logits,
                          st["assign"], st["pinv"], st["shape"])
        eng.refresh(full=True)
        if arm == "learned_fp32":
            eng.gibbs(temperature=1.0, seed=1)
            eng.learned_train(epochs=1, batch_sites=512, lr=1e-3, seed=2, first=0, count=min(n, 8))
        torch.cuda.synchronize()
        secs, info = [], []
        for rep in range(reps):
            t0 = time.perf_counter()
            if arm == "gibbs_fp64":
                r = eng.gibbs(temperature=1.0, seed=200 + rep)
            else:
                r = eng.learned_move(updates=cfg.S // 2, temperature=1.0, seed=300 + rep)
            torch.cuda.synchronize()
            secs.append(time.perf_counter() - t0)
            info.append(r)
        out[arm] = {"seconds": secs, "stats": info}
        eng.close()
    return out


def algorithmic_cost(T: int, R: int, w: int = 8):
    """Per (particle, site, category) unit of one full refresh, stored-CL design.

    Bytes (the roofline's algorithmic figure): per internal node one 20-state
    partial written, two child 20-state partials read and one scaler written,
    B = (T-1) * (3 * 20 * w + 8) with w the partial's element width.
    Also returned: the minimum HBM bytes of this engine's layout, where child
    partials come back from L2 and tips are never stored -- the T-1 partial and
    scaler writes, B_min = (T-1) * (20 * w + 8).
    Flops (the reference's count): two dense 20x20 child mat-vecs, the
    Hadamard product and the rescale per internal node, F = (T-1) * 1660.
    """
    b = (T - 1) * (3 * 20 * w + 8)
    b_min = (T - 1) * (20 * w + 8)
    f = (T - 1) * (2 * 800 + 60)
    return b, f, b_min


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dgemm_peak_tflops():
    """cuBLAS FP64 GEMM throughput as the measured FP64 ceiling."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def cpu_baseline(cfg, codes, st, n_sample, min_seconds=10.0):
    """Time the oracle's OpenMP full refresh on a bounded particle sample."""
    import oracle
    n = min(n_sample, st["parent"].shape[0])
    sl = slice(0, n)
    rates = np.stack([oracle.discretize_gamma(s, cfg.R) for s in st["shape"][sl]])
    args = (codes, st["parent"][sl], st["branch"][sl], st["base"][sl], st["num_classes"][sl],
            st["logits"][sl], st["assign"][sl], st["pinv"][sl], rates)
    threads = oracle.max_threads()
    oracle.lnl_batch(*args, nthreads=threads)  # warm-up
    reps, t0 = 0, time.perf_counter()
    while True:
        oracle.lnl_batch(*args, nthreads=threads)
        reps += 1
        el = time.perf_counter() - t0
        if el >= min_seconds:
            break
    units = reps * n * cfg.S * cfg.R
    return {"value": units / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} particles x {cfg.S} sites x {cfg.R} categories, full refresh, "
                      f"{reps} repetitions in {el:.1f} s: the oracle's speed (FP64 C++ "
                      "restatement of the reference's path, OpenMP over particles)"}


def measure_reassignment(codes, st, cfg, n, local, torch):
    """One Gibbs pass (Neal 8, floor(S/2) site iterations per particle, then
    the re-permutation and full refresh) and one learned-proposal pass of the
    same length on the first n particles, wall-clocked around
    device-synchronised calls; the MLP is trained first (untimed). The context
    has 32 class slots beyond the particles' largest K, since Gibbs opens new
    classes."""
    import smccat
    kmax = st["logits"].shape[1] + 32
    logits = np.zeros((n, kmax, 20))
    logits[:, :st["logits"].shape[1]] = st["logits"][:n]
    eng = smccat.Engine(codes, cfg.R, n, max_classes=kmax, lg=cfg.lg, invar=cfg.invar,
                        cat=cfg.cat, device=local)
    eng.set_particles(0, st["parent"][:n], st["branch"][:n], st["base"][:n],
                      st["num_classes"][:n], logits, st["assign"][:n], st["pinv"][:n],
                      st["shape"][:n])
    eng.refresh(full=True)
    its = cfg.S // 2
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    gs = eng.gibbs(temperature=1.0, seed=11, first=0, count=n)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    loss = eng.learned_train(epochs=1, batch_sites=512, lr=1e-3, seed=3, first=0, count=min(n, 8))
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    ls = eng.learned_move(updates=its, temperature=1.0, seed=12, first=0, count=n)
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    eng.close()
    return {"particles": n, "site_iterations_per_particle": its,
            "gibbs": {"seconds": t1 - t0, "site_iterations_per_s": n * its / (t1 - t0),
                      "classes_before": gs["classes_before"], "classes_after": gs["classes_after"]},
            "learned": {"train_seconds": t2 - t1, "train_loss": loss, "seconds": t3 - t2,
                        "site_updates_per_s": n * its / (t3 - t2),
                        "acceptance": ls["accepted"] / max(ls["proposed"], 1)}}


def multichain_ess(x):
    """Effective sample size of m chains of n draws, x [m][n] (Gelman et al.,
    Bayesian Data Analysis 3rd ed., 11.5): the pooled variance estimate
    var+ = (n-1)/n W + B/n, autocorrelations rho_t = 1 - V_t / (2 var+) from
    the variogram V_t, summed over lags while adjacent pairs stay positive."""
    x = np.asarray(x, dtype=np.float64)
    m, n = x.shape
    if n < 2:
        return float("nan")
    W = x.var(axis=1, ddof=1).mean()
    B_over_n = x.mean(axis=1).var(ddof=1) if m > 1 else 0.0
    var_plus = (n - 1) / n * W + B_over_n
    if not var_plus > 0:
        return float("nan")
    rho = []
    for t in range(1, n):
        V = np.mean((x[:, t:] - x[:, :-t]) ** 2)
        rho.append(1.0 - V / (2.0 * var_plus))
    s = 0.0
    for t in range(0, len(rho), 2):
        pair = rho[t] + (rho[t + 1] if t + 1 < len(rho) else 0.0)
        if pair < 0:
            break
        s += pair
    return float(m * n / (1.0 + 2.0 * s))


def measure_sampler(cid, n, sweeps, local, torch, gibbs_every=10, chosen_sweeps=10):
    """The sampler comparison (plain FP64 path against the mixed-precision,
    graph-captured, learned-proposal sampler) on a CAT configuration.

    One sweep = Mcmc::operator() with the configuration's iterations on every
    particle + one CAT reassignment pass of floor(S/2) site updates per
    particle, at temperature 1.
      plain arm:  FP64 partials; Mcmc::operator() on the host-driven lockstep
                  path (smccat_rejuvenate); Neal-8 Gibbs reassignment.
      chosen arm: FP32 partials; Mcmc::operator() entirely on the device as one
                  CUDA graph (smccat_mcmc_sweep); the learned-proposal
                  reassignment, with the Gibbs move on every `gibbs_every`-th
                  sweep so the class count keeps mixing (every 10th: the
                  reference's rate, alg8Probability = 0.1, main.cpp:303). Its MLP is trained
                  (untimed) on the assignments a Gibbs warm-up pass leaves.
    Both arms start from the same particles and run one untimed warm-up sweep,
    then timed ones (wall clock around device-synchronised calls): `sweeps`
    for the plain arm, `chosen_sweeps` (a whole Gibbs period) for the chosen one.
    After every timed sweep the log-likelihood, tree length and class count of
    every particle are recorded; their multi-chain ESS over the particles
    divided by the arm's seconds is its ESS/s. The chosen arm's final states
    are re-evaluated at FP64 for its |dlogL|."""
    import smccat
    from smccat import workload
    cfg = workload.CONFIGS[cid]
    codes, _ = workload.simulate_alignment(cfg, np.random.default_rng(cfg.seed))
    st = workload.make_particles(cfg, n, np.random.default_rng(cfg.seed * 7 + 1))
    kmax = st["logits"].shape[1] + 96  # room for the classes Gibbs opens
    logits = np.zeros((n, kmax, 20))
    logits[:, :st["logits"].shape[1]] = st["logits"]
    res = {"workload": cfg.name, "particles": n,
           "timed_sweeps": {"plain_fp64_gibbs": sweeps, "fp32_graph_learned": chosen_sweeps},
           "chosen_gibbs_every": gibbs_every,
           "sweep": f"Mcmc::operator() x {cfg.iterations} iterations + {cfg.S // 2} site updates "
                    "per particle, temperature 1",
           "particles_note": f"{n} particles resident per arm (FP64 partials of a "
                             f"{cfg.T}x{cfg.S} particle with {kmax} class slots take ~2 GB)"}
    finals = {}
    for arm, prec in (("plain_fp64_gibbs", smccat.PREC_FP64), ("fp32_graph_learned", smccat.PREC_FP32)):
        eng = smccat.Engine(codes, cfg.R, n, max_classes=kmax, lg=cfg.lg, invar=cfg.invar,
                            cat=cfg.cat, device=local, precision=prec)
        eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"], logits,
                          st["assign"], st["pinv"], st["shape"])
        eng.refresh(full=True)
        eng.compute_split_posteriors()
        chosen = arm != "plain_fp64_gibbs"
        info = {}

        def sweep(k, timed):
            out = {}
            t_a = time.perf_counter()
            if chosen:
                r = eng.mcmc_sweep(iterations=cfg.iterations, temperature=1.0, seed=100 + k)
                torch.cuda.synchronize()
                t_b = time.perf_counter()
                g = eng.learned_move(updates=cfg.S // 2, temperature=1.0, seed=200 + k)
                out["acc"] = g["accepted"] / max(g["proposed"], 1)
                torch.cuda.synchronize()
                t_c = time.perf_counter()
                if timed and k % gibbs_every == gibbs_every - 1:
                    eng.gibbs(temperature=1.0, seed=300 + k)
                    out["gibbs"] = True
            else:
                r = eng.rejuvenate(iterations=cfg.iterations, temperature=1.0, seed=100 + k)
                torch.cuda.synchronize()
                t_b = t_c = time.perf_counter()
                eng.gibbs(temperature=1.0, seed=200 + k)
            torch.cuda.synchronize()
            t_d = time.perf_counter()
            out["parts"] = (t_b - t_a, t_c - t_b, t_d - t_c)  # MCMC, learned move, Gibbs
            out["steps"] = r["lockstep_steps"]
            out["mh"] = (sum(r["accepted"]), sum(r["proposed"]))
            return out

        if chosen:
            eng.gibbs(temperature=1.0, seed=1)
            info["train_loss"] = eng.learned_train(epochs=1, batch_sites=512, lr=1e-3, seed=2,
                                                   first=0, count=min(n, 8))
        sweep(-1, False)  # warm-up (also graph capture of the first kind)
        torch.cuda.synchronize()
        traces = {"lnl": [], "tree_length": [], "classes": []}
        secs, steps, acc, mh_a, mh_p, n_gibbs = 0.0, 0, [], 0, 0, 0
        parts = np.zeros(3)
        nsw = chosen_sweeps if chosen else sweeps
        for k in range(nsw):
            t0 = time.perf_counter()
            o = sweep(k, True)
            torch.cuda.synchronize()
            secs += time.perf_counter() - t0
            steps += o["steps"]
            parts += np.array(o["parts"])
            mh_a += o["mh"][0]
            mh_p += o["mh"][1]
            n_gibbs += 1 if (not chosen or o.get("gibbs")) else 0
            if "acc" in o:
                acc.append(o["acc"])
            print(f"sampler {arm} sweep {k}: {time.perf_counter() - t0:.2f} s, {o['steps']} steps",
                  file=sys.stderr, flush=True)
            g = eng.get_particles()
            traces["lnl"].append(eng.lnl())
            traces["tree_length"].append(g["branch"].sum(axis=1))
            traces["classes"].append(g["num_classes"].astype(np.float64))
        ess = {k: multichain_ess(np.stack(v, axis=1)) for k, v in traces.items()}
        info.update({"sweeps_per_s": nsw / secs, "seconds_per_sweep": secs / nsw,
                     "lockstep_steps_per_sweep": steps / nsw,
                     "mcmc_acceptance": mh_a / max(mh_p, 1), "gibbs_passes": n_gibbs,
                     "seconds_per_sweep_in": {"mcmc": parts[0] / nsw, "learned_move": parts[1] / nsw,
                                              "gibbs": parts[2] / nsw},
                     "ess": ess, "ess_per_s": {k: v / secs for k, v in ess.items()},
                     "mean_lnl_last": float(np.mean(traces["lnl"][-1])),
                     "mean_classes_last": float(np.mean(traces["classes"][-1]))})
        if acc:
            info["learned_acceptance"] = float(np.mean(acc))
        res[arm] = info
        finals[arm] = (eng.get_particles(), eng.lnl())
        eng.close()
    # FP64 re-evaluation of the chosen arm's final states.
    g, l32 = finals["fp32_graph_learned"]
    e64 = smccat.Engine(codes, cfg.R, n, max_classes=kmax, lg=cfg.lg, invar=cfg.invar, cat=cfg.cat,
                        device=local)
    e64.set_particles(0, g["parent"], g["branch"], g["base"], g["num_classes"], g["logits"],
                      g["assign"], g["pinv"], g["shape"])
    e64.refresh(full=True)
    res["fp32_graph_learned"]["max_abs_dlogl_vs_fp64"] = float(np.max(np.abs(l32 - e64.lnl())))
    e64.close()
    p, c = res["plain_fp64_gibbs"], res["fp32_graph_learned"]
    res["speedup_sweeps_per_s"] = c["sweeps_per_s"] / p["sweeps_per_s"]
    res["ess_per_s_ratio"] = {k: (c["ess_per_s"][k] / p["ess_per_s"][k])
                              if p["ess_per_s"][k] and np.isfinite(p["ess_per_s"][k]) else None
                              for k in p["ess_per_s"]}
    return res


def measure_smc(reps, n, local, torch, iterations=5, alg8=0.1):
    """Whole SMC analyses (main.cpp:147-336 through smccat.smc.run) from the
    same initial population, per arm and replicate seed (plain: FP64, host
    lockstep rejuvenation, Gibbs; chosen: FP32, the device sweep, the learned
    proposal with Gibbs every 4th round): log marginal
    likelihood, SMC steps, resampling rounds, wall seconds, final ESS per
    second. The initial population comes from the workload generator, not
    from the prior, so log Z is compared between arms, not to a truth."""
    import smccat
    from smccat import smc, workload
    cfg = workload.WorkloadConfig("cat_gtr_g4_16x500", T=16, S=500, R=4, particles=n,
                                  iterations=iterations, lg=False, invar=False, cat=True, alpha=0.8,
                                  dp_concentration=3.0, k_range=(1, 6), seed=9)
    codes, _ = workload.simulate_alignment(cfg, np.random.default_rng(cfg.seed))
    st = workload.make_particles(cfg, n, np.random.default_rng(99))
    kmax = st["logits"].shape[1] + 24
    logits = np.zeros((n, kmax, 20))
    logits[:, :st["logits"].shape[1]] = st["logits"]
    out = {"workload": cfg.name, "particles": n, "rejuvenation_iterations": cfg.iterations,
           "threshold": 0.6, "alg8_probability": alg8}
    for arm, prec, move, dev in (("plain_fp64_gibbs", smccat.PREC_FP64, "gibbs", False),
                                 ("fp32_learned", smccat.PREC_FP32, "learned", True)):
        runs = []
        for r in range(reps):
            eng = smccat.Engine(codes, cfg.R, n, max_classes=kmax, lg=cfg.lg, invar=cfg.invar,
                                cat=cfg.cat, device=local, precision=prec)
            eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                              logits, st["assign"], st["pinv"], st["shape"])
            eng.refresh(full=True)
            res = smc.run(eng, cat=True, iterations=cfg.iterations, reassign=move, seed=1000 + r,
                          alg8_probability=alg8, sync=torch.cuda.synchronize, device_sweep=dev)
            res.pop("temperatures")
            runs.append(res)
            eng.close()
        lz = np.array([x["log_z"] for x in runs])
        out[arm] = {"runs": runs, "log_z_mean": float(lz.mean()),
                    "log_z_sd": float(lz.std(ddof=1)) if reps > 1 else None,
                    "seconds_mean": float(np.mean([x["seconds"] for x in runs])),
                    "final_ess_per_s_mean": float(np.mean([x["final_ess_per_s"] for x in runs]))}
    out["speedup_wall"] = out["plain_fp64_gibbs"]["seconds_mean"] / out["fp32_learned"]["seconds_mean"]
    # Paired by replicate seed (the same initial population and SMC seed per pair).
    d = np.array([a["log_z"] - b["log_z"] for a, b in zip(out["fp32_learned"]["runs"],
                                                           out["plain_fp64_gibbs"]["runs"])])
    out["log_z_paired_difference"] = {
        "mean": float(d.mean()), "sd": float(d.std(ddof=1)) if reps > 1 else None,
        "standard_error": float(d.std(ddof=1) / np.sqrt(reps)) if reps > 1 else None}
    return out


def measure_config_waves(cid, steps, local, rank, particles=0, oracle_sample=2, gibbs_particles=0):
    """Full-refresh throughput of a configuration whose particles may not fit
    one context: particles stream through the device in waves (upload states,
    refreshLikelihood(true), read log-likelihoods), at FP64 and at FP32; the
    FP32 log-likelihoods are compared with FP64 per particle, and a few
    particles of both with the oracle."""
    import torch
    import oracle
    import smccat
    from smccat import discretize_gamma, workload
    cfg = workload.CONFIGS[cid]
    rng = np.random.default_rng(cfg.seed)
    codes, truth = workload.simulate_alignment(cfg, rng)
    n = particles or cfg.particles
    st = workload.make_particles(cfg, n, np.random.default_rng(cfg.seed * 1000 + rank))
    kmax = st["logits"].shape[1]
    res = {"workload": cfg.name, "taxa": cfg.T, "sites": cfg.S, "rates": cfg.R, "particles": n,
           "max_classes": kmax, "data_classes": int(truth["K"])}
    lnls = {}
    for prec, name in ((smccat.PREC_FP64, "fp64"), (smccat.PREC_FP32, "fp32")):
        esz = 4 if prec == smccat.PREC_FP32 else 8
        spad = (cfg.S + 31) // 32 * 32
        per = (cfg.T - 1) * 2 * (20 * esz + 8) * cfg.R * spad + \
            kmax * (2 * cfg.T - 1) * 2 * cfg.R * 440 * esz + 4 * cfg.S + 8 * cfg.S
        free = torch.cuda.mem_get_info(local)[0]
        W = max(1, min(n, int(0.8 * free / per)))
        eng = smccat.Engine(codes, cfg.R, W, max_classes=kmax, lg=cfg.lg, invar=cfg.invar,
                            cat=cfg.cat, device=local, precision=prec)
        stream = torch.cuda.ExternalStream(eng.stream_ptr, device=torch.device("cuda", local))

        def one_pass():
            out = []
            for w0 in range(0, n, W):
                c = min(W, n - w0)
                sl = slice(w0, w0 + c)
                eng.set_particles(0, st["parent"][sl], st["branch"][sl], st["base"][sl],
                                  st["num_classes"][sl], st["logits"][sl], st["assign"][sl],
                                  st["pinv"][sl], st["shape"][sl])
                eng.refresh(0, c, full=True)
                out.append(eng.lnl(0, c))
            return np.concatenate(out)

        lnls[name] = one_pass()
        eng.autotune(reps=1) if n <= W else None
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            one_pass()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / steps
        eng.set_profiling(True)
        one_pass()
        prof = eng.profile()
        eng.set_profiling(False)
        units = n * cfg.S * cfg.R
        b_unit, _, b_min = algorithmic_cost(cfg.T, cfg.R, w=esz)
        prune_s = prof["ms"]["prune"] * 1e-3
        peak = measured_peaks()[0]
        res[name] = {"value": units / (ms * 1e-3), "unit": UNIT, "ms_per_pass": ms,
                     "particles_per_wave": W, "waves": (n + W - 1) // W,
                     "device_gb": eng.device_bytes / 1e9,
                     "kernel_ms_per_pass": {k: round(v, 3) for k, v in prof["ms"].items()},
                     "prune_variant": eng.kernel_variants()[1],
                     "roofline": {"bound": "hbm", "unit": "GB/s", "peak": peak,
                                  "achieved": b_unit * units / prune_s / 1e9,
                                  "frac": b_unit * units / prune_s / 1e9 / peak,
                                  "min_bytes_frac": b_min * units / prune_s / 1e9 / peak,
                                  "what": "pruning kernels' summed CUDA-event time over the waves "
                                          "of one pass, algorithmic bytes (T-1)(60w+8) per unit"}}
        eng.close()
        if cfg.cat and name == "fp64" and gibbs_particles > 0:
            res["reassignment"] = measure_reassignment(codes, st, cfg, min(gibbs_particles, n),
                                                       local, torch)
    d = np.abs(lnls["fp32"] - lnls["fp64"])
    res["fp32_vs_fp64_abs_dlogl"] = {"max": float(d.max()), "mean": float(d.mean())}
    o = []
    for i in range(min(oracle_sample, n)):
        K = int(st["num_classes"][i])
        rates = discretize_gamma(st["shape"][i], cfg.R)
        ref = oracle.lnl(codes, st["parent"][i], st["branch"][i], st["base"][i],
                         st["logits"][i][:K], st["assign"][i], st["pinv"][i], rates)
        o.append({"fp64_rel": abs(lnls["fp64"][i] - ref) / abs(ref),
                  "fp32_abs": abs(lnls["fp32"][i] - ref)})
    res["vs_oracle"] = o
    return res


def cl_bytes(cfg, n, w=8):
    """Device bytes of the partial-likelihood buffers of n particles: T-1
    internal nodes x 2 workspaces x 20 states x R x sites padded to 32."""
    spad = (cfg.S + 31) // 32 * 32
    return (cfg.T - 1) * 2 * 20 * cfg.R * spad * w * n


MODEL_NAMES = {"lg_g4_16x500": "LG+G4", "gtr_g4_i_48x2000": "GTR+G4+I",
               "cat_gtr_g4_64x5000": "CAT-GTR+G4", "cat_uneven_100x10000": "CAT-GTR+G4, K ~ U{8..120}",
               "cat_gtr_g4_i_128x20000": "CAT-GTR+G4+I"}


def bench_config(cfg, n, world):
    """The workload description both arms print, identical between them."""
    return {"workload": cfg.name, "taxa": cfg.T, "sites": cfg.S, "rates": cfg.R,
            "particles_per_gpu": n,
            "model": MODEL_NAMES.get(cfg.name, cfg.name),
            "step": "full refresh of every particle (refreshLikelihood(true))",
            "l2": "inputs larger than L2 (partials %.1f GB per GPU at FP64)" % (cl_bytes(cfg, n) / 1e9),
            "parallelism": f"particles sharded, {world} GPU(s), no collective"}


def run_reference(args, rank, world):
    """Reference arm: the CPU implementation of the path on the host cores,
    over the same particles as the GPU arm's rank 0. The inputs are built with
    the oracle's gamma discretisation and LG table, so this process never
    loads the engine library."""
    if rank != 0:
        return
    import oracle
    from smccat import workload
    cfg = workload.CONFIGS[args.config]
    codes, _ = workload.simulate_alignment(cfg, np.random.default_rng(cfg.seed),
                                           gamma_fn=oracle.discretize_gamma, lg_fn=oracle.lg_base)
    n = args.particles or cfg.particles
    st = workload.make_particles(cfg, n, np.random.default_rng(cfg.seed * 1000),
                                 lg_fn=oracle.lg_base)
    rates = np.stack([oracle.discretize_gamma(s, cfg.R) for s in st["shape"]])
    a = (codes, st["parent"], st["branch"], st["base"], st["num_classes"], st["logits"],
         st["assign"], st["pinv"], rates)
    threads = oracle.max_threads()
    for _ in range(args.warmup):
        oracle.lnl_batch(*a, nthreads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.lnl_batch(*a, nthreads=threads)
    el = time.perf_counter() - t0
    value = args.steps * n * cfg.S * cfg.R / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(cfg, n, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"all {n} particles x {cfg.S} sites x {cfg.R} categories per "
                                   "step: the oracle's speed (an FP64 C++ restatement of the "
                                   "reference's refreshLikelihood(true) with its OpenMP loop over "
                                   "particles; the reference itself needs Eigen and Boost, absent "
                                   "here)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import smccat
    from smccat import workload

    torch.cuda.set_device(local)
    if args.reassign > 0:
        if rank == 0:
            print(json.dumps({"metric": "CAT reassignment pass seconds", "unit": "s",
                              "higher_is_better": False, "data": "synthetic",
                              "reassign": measure_reassign_only(args.sampler_config, args.reassign,
                                                                local, torch)}), flush=True)
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    cfg = workload.CONFIGS[args.config]
    rng = np.random.default_rng(cfg.seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    prng = np.random.default_rng(cfg.seed * 1000 + rank)
    n = args.particles or cfg.particles
    st = workload.make_particles(cfg, n, prng)
    eng = smccat.Engine(codes, cfg.R, n, max_classes=st["logits"].shape[1], lg=cfg.lg,
                        invar=cfg.invar, cat=cfg.cat, device=local)
    load = lambda: eng.set_particles(0, st["parent"], st["branch"], st["base"],  # noqa: E731
                                     st["num_classes"], st["logits"], st["assign"], st["pinv"],
                                     st["shape"])
    load()
    eng.refresh(full=True)
    if args.variant >= 0:
        eng.set_kernel_variant(args.variant)
        tuned = {"variant": args.variant, "ms": None}
    else:
        tuned = eng.autotune(reps=2)
    stream = torch.cuda.ExternalStream(eng.stream_ptr, device=torch.device("cuda", local))
    units_per_step = n * cfg.S * cfg.R

    # ---- device-resident value --------------------------------------------
    for _ in range(args.warmup):
        eng.refresh(full=True)
    barrier()
    eng.set_profiling(True)
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        eng.refresh(full=True)
    e1.record(stream)
    e1.synchronize()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    prof = eng.profile()
    eng.set_profiling(False)

    # ---- e2e through the C-ABI with host buffers ----------------------------
    lnl_host = eng.lnl()
    eng.set_profiling(False)
    for _ in range(0 if args.skip_e2e else 2):
        load()
        eng.refresh(full=True)
        lnl_host = eng.lnl()
    barrier()
    eng.set_profiling(False)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    f0.record(stream)
    for _ in range(0 if args.skip_e2e else args.steps):
        load()
        eng.refresh(full=True)
        lnl_host = eng.lnl()
    f1.record(stream)
    f1.synchronize()
    barrier()
    ms_e2e = f0.elapsed_time(f1)
    prof_e2e = eng.profile()
    assert np.all(np.isfinite(lnl_host))

    # ---- rejuvenation sweeps: Mcmc::operator() x iterations on every particle -----
    sweep_stats, ms_sweep = None, 0.0
    if args.sweeps > 0:
        load()
        eng.refresh(full=True)
        # Split posteriors of the population for adaptive NNI (main.cpp:203),
        # installed for this and the device sweep below.
        eng.compute_split_posteriors()
        eng.rejuvenate(iterations=cfg.iterations, temperature=args.sweep_temp, seed=999 + rank)
        barrier()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for k in range(args.sweeps):
            sweep_stats = eng.rejuvenate(iterations=cfg.iterations, temperature=args.sweep_temp,
                                         seed=1000 + k + 100 * rank)
        s1.record(stream)
        s1.synchronize()
        barrier()
        ms_sweep = s0.elapsed_time(s1)
    # ---- tree-move sweep with everything on the device (one CUDA graph) ----
    dev_sweep, ms_dev = None, 0.0
    if args.sweeps > 0 and args.branch_steps > 0:
        load()
        eng.refresh(full=True)
        eng.tree_sweep(steps=4, temperature=args.sweep_temp, seed=5 + rank)
        # Three sweeps from the same state; the median is reported (a single
        # call includes graph capture and instantiation, which can stall).
        reps = []
        for k in range(3):
            load()
            eng.refresh(full=True)
            barrier()
            d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            d0.record(stream)
            bst = eng.tree_sweep(steps=args.branch_steps, temperature=args.sweep_temp,
                                   seed=6 + rank)
            d1.record(stream)
            d1.synchronize()
            barrier()
            reps.append(d0.elapsed_time(d1))
        ms_dev = float(np.median(reps))
        dev_sweep = {"what": "treeMove MH steps (NNI, adaptive NNI, SPR, branch, subtree scale: 0.1 / 0.3 / 0.1 / 0.4 / 0.1) on every particle, proposals, plans "
                             "and accept/reject on the device, captured as one CUDA graph "
                             "(upload, capture and sync-back included); median of 3 sweeps",
                     "steps": args.branch_steps, "ms_per_sweep_each": reps, **bst}

    # ---- mixed precision (FP32 partials / matrices) on the same particles ----------
    mixed, ms_mixed = None, 0.0
    if args.mixed:
        load()
        eng.refresh(full=True)
        ref64 = eng.lnl()
        e32 = smccat.Engine(codes, cfg.R, n, max_classes=st["logits"].shape[1], lg=cfg.lg,
                            invar=cfg.invar, cat=cfg.cat, device=local,
                            precision=smccat.PREC_FP32)
        e32.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                          st["logits"], st["assign"], st["pinv"], st["shape"])
        e32.refresh(full=True)
        tuned32 = e32.autotune(reps=2)
        stream32 = torch.cuda.ExternalStream(e32.stream_ptr, device=torch.device("cuda", local))
        for _ in range(args.warmup):
            e32.refresh(full=True)
        e32.set_profiling(True)
        barrier()
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream32)
        for _ in range(args.steps):
            e32.refresh(full=True)
        m1.record(stream32)
        m1.synchronize()
        barrier()
        ms_mixed = m0.elapsed_time(m1)
        p32 = e32.profile()
        dl = np.abs(e32.lnl() - ref64)
        mixed = {"precision": "fp32 partials and matrices; fp64 eigensystems, log-scalers, sums",
                 "ms_per_step": ms_mixed / args.steps,
                 "prune_ms": p32["ms"]["prune"] / max(p32["launches"]["prune"], 1),
                 "max_abs_dlogl_vs_fp64": float(dl.max()), "mean_abs_dlogl_vs_fp64": float(dl.mean()),
                 "autotune": tuned32}
        e32.close()

    # ---- site-pattern compression (FP64) on the same particles -----------------
    pat, ms_pat = None, 0.0
    if args.patterns:
        load()
        eng.refresh(full=True)
        ref64 = eng.lnl()
        ep = smccat.Engine(codes, cfg.R, n, max_classes=st["logits"].shape[1], lg=cfg.lg,
                           invar=cfg.invar, cat=cfg.cat, device=local, patterns=True)
        ep.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                         st["logits"], st["assign"], st["pinv"], st["shape"])
        ep.set_kernel_variant(tuned["variant"])
        streamp = torch.cuda.ExternalStream(ep.stream_ptr, device=torch.device("cuda", local))
        for _ in range(args.warmup):
            ep.refresh(full=True)
        barrier()
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        q0.record(streamp)
        for _ in range(args.steps):
            ep.refresh(full=True)
        q1.record(streamp)
        q1.synchronize()
        barrier()
        ms_pat = q0.elapsed_time(q1)
        uniq = np.unique(codes.T, axis=0).shape[0]
        pat = {"what": "each distinct alignment column evaluated once per particle and class, "
                       "weighted by its site count (no counterpart in the reference)",
               "distinct_columns": int(uniq), "sites": int(cfg.S),
               "max_rel_dlogl_vs_uncompressed": float(np.max(np.abs(ep.lnl() - ref64) / np.abs(ref64)))}
        ep.close()

    times = torch.tensor([ms, ms_e2e, ms_sweep, ms_mixed, ms_pat, ms_dev], dtype=torch.float64,
                         device="cuda")
    if dist is not None:
        dist.all_reduce(times, op=dist.ReduceOp.MAX)
    ms, ms_e2e, ms_sweep, ms_mixed, ms_pat, ms_dev = times.tolist()
    if dev_sweep is not None:
        dev_sweep["ms_per_step"] = ms_dev / args.branch_steps
        if sweep_stats is not None and sweep_stats["lockstep_steps"]:
            dev_sweep["host_driven_ms_per_lockstep_step"] = ms_sweep / args.sweeps / sweep_stats["lockstep_steps"]
    if pat is not None:
        pat["value"] = units_per_step * args.steps * world / (ms_pat * 1e-3)
        pat["unit"] = UNIT + " (every site counted)"
        pat["ms_per_step"] = ms_pat / args.steps
    if mixed is not None:
        mixed["value"] = units_per_step * args.steps * world / (ms_mixed * 1e-3)
        mixed["unit"] = UNIT
        b32, _, b32_min = algorithmic_cost(cfg.T, cfg.R, w=4)
        mixed["roofline_hbm_frac"] = b32 * units_per_step / (mixed["prune_ms"] * 1e-3) / 1e9 / \
            measured_peaks()[0]
        mixed["min_bytes_hbm_frac"] = b32_min * units_per_step / (mixed["prune_ms"] * 1e-3) / \
            1e9 / measured_peaks()[0]
    total_units = units_per_step * args.steps * world
    value = total_units / (ms * 1e-3)
    e2e_value = None if args.skip_e2e else total_units / (ms_e2e * 1e-3)

    if rank == 0:
        b_unit, f_unit, b_min = algorithmic_cost(cfg.T, cfg.R)
        prune_ms = prof["ms"]["prune"] / max(prof["launches"]["prune"], 1)
        bytes_per_launch = b_unit * units_per_step
        achieved = bytes_per_launch / (prune_ms * 1e-3) / 1e9
        peak, peak_kind = measured_peaks()
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "prune_fp64_traffic.json")
        if os.path.exists(tpath):
            with open(tpath) as f:
                tj = json.load(f)
            if tj.get("workload") == cfg.name:
                # measured on a small case; DRAM bytes scale with the units processed
                traffic = tj["dram_bytes"] / tj["units"] * units_per_step
        try:
            fp64_peak = dgemm_peak_tflops()
        except Exception:
            fp64_peak = None
        fp64_achieved = f_unit * units_per_step / (prune_ms * 1e-3) / 1e12
        # Executed: a tip child costs a shared-memory gather, not a mat-vec, so
        # only the T-2 internal child edges run 20x20 mat-vecs.
        f_exec = (cfg.T - 2) * 800 + (cfg.T - 1) * 60
        fp64_executed = f_exec * units_per_step / (prune_ms * 1e-3) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": bench_config(cfg, n, world),
            "autotune": tuned,
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": prof_e2e["h2d_bytes"] // args.steps,
                    "d2h_bytes_per_step": prof_e2e["d2h_bytes"] // args.steps},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "prune_kernel<4>", "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": bytes_per_launch,
                         "algorithmic_bytes_per_unit": b_unit,
                         "min_bytes_per_unit": b_min,
                         "min_bytes_frac": b_min * units_per_step / (prune_ms * 1e-3) / 1e9 / peak,
                         "avg_launch_ms": prune_ms},
            "fp64": {"achieved_tflops": fp64_achieved, "dgemm_peak_tflops": fp64_peak,
                     "frac": (fp64_achieved / fp64_peak) if fp64_peak else None,
                     "flops_per_unit": f_unit,
                     "executed_flops_per_unit": f_exec, "executed_tflops": fp64_executed,
                     "executed_frac": (fp64_executed / fp64_peak) if fp64_peak else None},
            "kernel_ms_per_step": {k: v / args.steps for k, v in prof["ms"].items()},
            "gpu_launches": sum(prof["launches"].values()),
            "mixed_precision": mixed,
            "site_patterns": pat,
            "device_tree_sweep": dev_sweep,
            "sweeps_per_s": (args.sweeps / (ms_sweep * 1e-3)) if args.sweeps > 0 else None,
            "sweep": None if sweep_stats is None else {
                "definition": f"Mcmc::operator() with {cfg.iterations} iterations on all {n} "
                              f"particles per GPU at temperature {args.sweep_temp}, lockstep",
                "ms_per_sweep": ms_sweep / args.sweeps,
                "lockstep_steps": sweep_stats["lockstep_steps"],
                "proposed": sum(sweep_stats["proposed"]),
                "accepted": sum(sweep_stats["accepted"])},
            "clocks": clk,
        }
        if args.extra_configs:
            line["extra_configs"] = [
                measure_config_waves(int(c), max(1, args.steps // 5), local, rank,
                                     particles=args.extra_particles,
                                     gibbs_particles=args.gibbs_particles)
                for c in args.extra_configs.split(",") if c.strip()]
        if args.smc:
            line["smc"] = measure_smc(args.smc, args.smc_particles, local, torch,
                                      iterations=args.smc_iterations, alg8=args.smc_alg8)
        if args.sampler_config:
            line["sampler"] = measure_sampler(args.sampler_config, args.sampler_particles,
                                              args.sampler_sweeps, local, torch,
                                              chosen_sweeps=args.sampler_chosen_sweeps)
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(cfg, codes, st, args.cpu_sample)
        print(json.dumps(line), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""The reference-style C++ interface (include/smccat_particle.hpp): class
Particle / Mcmc with the reference's signatures (src/analysis/Particle.hpp:48-94,
Mcmc.hpp:15-26), compiled here with g++ against the C-ABI library.

* CPU: the header compiles warning-free, the driver links, and without a
  device the first Particle fails with SMCCAT_ENODEV through smccat::Error.
* GPU: tests/facade/facade_drive.cpp builds particles with the reference's
  constructor, runs Mcmc with the reference's move registry on each, a Gibbs
  reassignment, then copyFromSerialized into a shared batch and the batched
  sweep. Every state it prints must have the oracle's log-likelihood (1e-9
  relative) and log-prior, and reloading a state must reproduce its value.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from smccat import workload

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "facade", "facade_drive.cpp")
LIBDIR = os.path.join(ROOT, "smc-cat_b200", "lib")


def _build(tmp_path):
    exe = str(tmp_path / "facade_drive")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           SRC, "-L", LIBDIR, "-lsmccat", f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return exe


def _input(tmp_path, cfg, codes):
    path = str(tmp_path / "aln.bin")
    hdr = np.array([cfg.T, cfg.S, cfg.R, int(cfg.lg), int(cfg.invar), int(cfg.cat)], np.int32)
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(np.ascontiguousarray(codes, np.uint8).tobytes())
    return path


CFG = workload.WorkloadConfig("facade", T=8, S=120, R=4, particles=3, iterations=3, lg=False,
                              invar=True, cat=True, pinv=0.1, dp_concentration=2.0, seed=23)


def test_header_compiles_and_reports_no_device(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: the GPU test covers this path")
    exe = _build(tmp_path)
    codes, _ = workload.simulate_alignment(CFG, np.random.default_rng(CFG.seed))
    out = subprocess.run([exe, _input(tmp_path, CFG, codes), "1", "1", "1.0"], capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 3
    assert "smccat error 6" in out.stderr


@pytest.mark.gpu
def test_reference_interface_drives_the_engine(tmp_path):
    exe = _build(tmp_path)
    codes, _ = workload.simulate_alignment(CFG, np.random.default_rng(CFG.seed))
    out = subprocess.run([exe, _input(tmp_path, CFG, codes), str(CFG.particles),
                          str(CFG.iterations), "0.7"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-3000:]
    recs = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    n = CFG.particles
    expected = [ph for _ in range(n) for ph in ("init", "mcmc", "gibbs")] + ["loaded"] * n + ["batch"] * n
    assert [r["phase"] for r in recs] == expected
    final = {}
    for r in recs:
        K = r["num_classes"]
        logits = np.array(r["logits"]).reshape(K, 20)
        assign = np.array(r["assign"], np.int32)
        counts = np.bincount(assign, minlength=K)
        assert np.all(counts > 0) and counts.tolist() == r["category_size"]
        rates = oracle.discretize_gamma(r["shape"], CFG.R)
        ref = oracle.lnl(codes, np.array(r["parent"], np.int32), np.array(r["branch"]),
                         np.array(r["base"]), logits, assign, r["pinv"], rates)
        assert r["lnl"] == pytest.approx(ref, rel=1e-9), (r["phase"], r["index"])
        prior = oracle.ln_prior(CFG.T, CFG.S, CFG.R, CFG.lg, np.array(r["branch"]), r["shape"],
                                np.array(r["base"]), logits, counts)
        assert r["ln_prior"] == pytest.approx(prior, rel=1e-12, abs=1e-9), (r["phase"], r["index"])
        assert r["splits"] == 2 * CFG.T - 2 - 1  # distinct non-root clades, one pair merged at the root
        if r["phase"] == "mcmc":
            assert sum(r["move_count"]) > 0
            assert all(a <= m for a, m in zip(r["accept_count"], r["move_count"]))
        if r["phase"] == "gibbs":
            final[r["index"]] = r["lnl"]
        if r["phase"] == "loaded":
            assert r["lnl"] == pytest.approx(final[r["index"]], rel=1e-12)

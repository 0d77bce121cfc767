"""The allocation-free transition-matrix entry point, against the context path.

``smccat_transition_matrices_noalloc`` is for callers that cannot call
cudaMalloc -- hosts running inside another framework's memory budget or
allocator, or plugins that are only handed pre-allocated buffers. Here the
test plays that caller: it owns every device buffer (allocated through torch)
and compares the entry point's matrices with the FP64 oracle's P(t) and with
the ones the regular context path (``smccat_create`` / ``smccat_refresh``)
builds for the same particles, on two calls in a row, and once at the largest
class count the scratch array takes. This file is collected last so that a
run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import oracle
import smccat
from smccat import workload

pytestmark = pytest.mark.gpu

TOL = 1e-13  # the transition-matrix tolerance of tests/test_gpu_parity.py


def _entry():
    f = smccat.lib().smccat_transition_matrices_noalloc
    f.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _inputs(st, p, R):
    K = int(st["num_classes"][p])
    rates = smccat.discretize_gamma(st["shape"][p], R)
    root = int(np.where(st["parent"][p] < 0)[0][0])
    nodes = [n for n in range(st["parent"].shape[1]) if n != root]
    times = np.array([[st["branch"][p, n] * rates[r] for n in nodes for r in range(R)]] * K)
    base = np.tile(st["base"][p], (K, 1))
    logits = np.ascontiguousarray(st["logits"][p, :K])
    return K, nodes, base, logits, times


def test_noalloc_matches_context_path_on_two_calls():
    import torch
    cfg = workload.WorkloadConfig("noalloc", T=7, S=96, R=4, particles=3, iterations=1, lg=False,
                                  invar=True, cat=True, k_range=(2, 5), seed=21)
    rng = np.random.default_rng(cfg.seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng)
    eng = smccat.Engine(codes, cfg.R, cfg.particles, max_classes=st["logits"].shape[1],
                        invar=True, cat=True)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    f = _entry()
    stream = torch.cuda.current_stream()
    for p in (0, 1):  # two calls in a row, different inputs, same scratch array
        K, nodes, base, logits, times = _inputs(st, p, cfg.R)
        d_base = torch.tensor(base, dtype=torch.float64, device="cuda")
        d_logits = torch.tensor(logits, dtype=torch.float64, device="cuda")
        d_times = torch.tensor(times, dtype=torch.float64, device="cuda")
        d_out = torch.full((K, times.shape[1], 20, 20), float("nan"), dtype=torch.float64,
                           device="cuda")
        rc = f(K, d_base.data_ptr(), d_logits.data_ptr(), times.shape[1], d_times.data_ptr(),
               d_out.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
        assert rc == smccat.OK, smccat.lib().smccat_last_error().decode()
        stream.synchronize()
        out = d_out.cpu().numpy()
        worst, worst_oracle = 0.0, 0.0
        for k in range(K):
            pi = oracle.softmax20(logits[k])
            for i, n in enumerate(nodes):
                for r in range(cfg.R):
                    ref = eng.transition_matrix(p, k, n, r)
                    worst = max(worst, float(np.abs(out[k, i * cfg.R + r] - ref).max()))
                    orc = oracle.transition(base[k], pi, times[k, i * cfg.R + r])
                    worst_oracle = max(worst_oracle, float(np.abs(out[k, i * cfg.R + r] - orc).max()))
        assert worst < TOL, (p, worst)
        assert worst_oracle < TOL, (p, worst_oracle)
    eng.close()


def test_noalloc_at_its_largest_class_count():
    """512 classes, the most one call takes: every matrix against the oracle."""
    import torch
    K, nt = 512, 2
    rng = np.random.default_rng(5)
    base = rng.normal(size=(K, 190))
    logits = np.zeros((K, 20))
    logits[:, :19] = rng.normal(size=(K, 19))
    times = rng.exponential(0.2, size=(K, nt))
    d_base = torch.tensor(base, dtype=torch.float64, device="cuda")
    d_logits = torch.tensor(logits, dtype=torch.float64, device="cuda")
    d_times = torch.tensor(times, dtype=torch.float64, device="cuda")
    d_out = torch.full((K, nt, 20, 20), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = _entry()(K, d_base.data_ptr(), d_logits.data_ptr(), nt, d_times.data_ptr(),
                  d_out.data_ptr(), ctypes.c_void_p(stream.cuda_stream))
    assert rc == smccat.OK, smccat.lib().smccat_last_error().decode()
    stream.synchronize()
    out = d_out.cpu().numpy()
    worst = 0.0
    for k in range(K):
        pi = oracle.softmax20(logits[k])
        for t in range(nt):
            worst = max(worst, float(np.abs(out[k, t] - oracle.transition(base[k], pi, times[k, t])).max()))
    assert worst < TOL, worst


def test_noalloc_rejects_requests_beyond_its_scratch():
    import torch
    f = _entry()
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    rc = f(513, buf.data_ptr(), buf.data_ptr(), 1, buf.data_ptr(), buf.data_ptr(), None)
    assert rc == smccat.EINVAL
    assert "512" in smccat.lib().smccat_last_error().decode()

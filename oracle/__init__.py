"""Smc-CAT likelihood oracle -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``oracle/liboracle.so``, an FP64 CPU restatement of the
reference's likelihood path (see ``oracle/oracle.cpp`` for the per-function
reference citations). Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` may import this module, and only as a checker or as
the timed CPU baseline -- never as part of the product path.

Parity status: parity unpinned. The reference (C++23 on Eigen + Boost) has no
tests or golden vectors and cannot be compiled on this machine. The oracle is
checked instead against golden vectors produced by
``tests/golden/make_golden.py``, an independent numpy/scipy restatement that
follows the reference's own formulas (general eigendecomposition + inverse for
P(t), Boost-equivalent gamma quantiles) and parses the LG table out of the
reference source.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_up = ctypes.POINTER(ctypes.c_uint8)


def build() -> str:
    """Compile liboracle.so with the committed Makefile (no-op if current)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_lg_base.argtypes = [_dp]
        L.orc_gamma_p.argtypes = [ctypes.c_double, ctypes.c_double]
        L.orc_gamma_p.restype = ctypes.c_double
        L.orc_gamma_quantile.argtypes = [ctypes.c_double] * 3
        L.orc_gamma_quantile.restype = ctypes.c_double
        L.orc_discretize_gamma.argtypes = [ctypes.c_double, ctypes.c_int, _dp]
        L.orc_softmax20.argtypes = [_dp, _dp]
        L.orc_rate_matrix.argtypes = [_dp, _dp, _dp]
        L.orc_transition.argtypes = [_dp, _dp, ctypes.c_double, _dp]
        L.orc_eigenvalues.argtypes = [_dp, _dp, _dp]
        L.orc_tip_encode.argtypes = [_up, ctypes.c_int, ctypes.c_int, _dp, _ip]
        L.orc_postorder.argtypes = [ctypes.c_int, _ip, _ip]
        L.orc_postorder.restype = ctypes.c_int
        L.orc_lnl.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _up, _ip, _dp, _dp,
                              ctypes.c_int, _dp, _ip, ctypes.c_double, _dp, _dp]
        L.orc_lnl.restype = ctypes.c_double
        L.orc_lnl_batch.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _up,
                                    _ip, _dp, _dp, _ip, ctypes.c_int, _dp, _ip, _dp, _dp, _dp,
                                    ctypes.c_int]
        L.orc_max_threads.restype = ctypes.c_int
        L.orc_ln_prior.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                   ctypes.c_double, _dp, ctypes.c_int, _dp, _ip, ctypes.c_double]
        L.orc_ln_prior.restype = ctypes.c_double
        L.orc_next_step.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double, _dp,
                                    ctypes.c_double]
        L.orc_gibbs_weights.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _up, _ip, _dp,
                                        _dp, ctypes.c_int, _dp, _ip, ctypes.c_double, _dp,
                                        ctypes.c_int, ctypes.c_int, _dp, ctypes.c_double,
                                        ctypes.c_double, _dp]
        _lib = L
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def _u(a):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    return a, a.ctypes.data_as(_up)


def lg_base() -> np.ndarray:
    out = np.zeros(190)
    lib().orc_lg_base(out.ctypes.data_as(_dp))
    return out


def gamma_p(a: float, x: float) -> float:
    return lib().orc_gamma_p(a, x)


def gamma_quantile(shape: float, scale: float, p: float) -> float:
    return lib().orc_gamma_quantile(shape, scale, p)


def discretize_gamma(shape: float, R: int) -> np.ndarray:
    out = np.zeros(R)
    lib().orc_discretize_gamma(shape, R, out.ctypes.data_as(_dp))
    return out


def softmax20(logits) -> np.ndarray:
    lg, lp = _d(logits)
    out = np.zeros(20)
    lib().orc_softmax20(lp, out.ctypes.data_as(_dp))
    return out


def rate_matrix(base, pi) -> np.ndarray:
    b, bp = _d(base)
    p, pp = _d(pi)
    Q = np.zeros((20, 20))
    lib().orc_rate_matrix(bp, pp, Q.ctypes.data_as(_dp))
    return Q


def transition(base, pi, t: float) -> np.ndarray:
    b, bp = _d(base)
    p, pp = _d(pi)
    P = np.zeros((20, 20))
    lib().orc_transition(bp, pp, t, P.ctypes.data_as(_dp))
    return P


def eigenvalues(base, pi) -> np.ndarray:
    b, bp = _d(base)
    p, pp = _d(pi)
    lam = np.zeros(20)
    lib().orc_eigenvalues(bp, pp, lam.ctypes.data_as(_dp))
    return lam


def tip_encode(codes):
    c, cp = _u(codes)
    T, S = c.shape
    inv = np.zeros(S)
    ch = np.zeros(S, dtype=np.int32)
    lib().orc_tip_encode(cp, T, S, inv.ctypes.data_as(_dp), ch.ctypes.data_as(_ip))
    return inv, ch


def postorder(parent) -> np.ndarray:
    par, pp = _i(parent)
    T = (len(par) + 1) // 2
    out = np.zeros(len(par), dtype=np.int32)
    if lib().orc_postorder(T, pp, out.ctypes.data_as(_ip)) != 0:
        raise ValueError("not a rooted binary tree")
    return out


def lnl(codes, parent, branch, base, logits, assign, pinv, rates, site_out=False):
    """refreshLikelihood(true) of one particle state; returns lnL (and sites)."""
    c, cp = _u(codes)
    T, S = c.shape
    rates = np.atleast_1d(np.asarray(rates, dtype=np.float64))
    R = len(rates)
    logits = np.atleast_2d(np.asarray(logits, dtype=np.float64))
    K = logits.shape[0]
    par, pp = _i(parent)
    br, bp = _d(branch)
    ba, bap = _d(base)
    lg, lgp = _d(logits)
    asg, ap = _i(assign)
    rt, rp = _d(rates)
    sites = np.zeros(S) if site_out else None
    v = lib().orc_lnl(T, S, R, cp, pp, bp, bap, K, lgp, ap, float(pinv), rp,
                      sites.ctypes.data_as(_dp) if site_out else None)
    return (v, sites) if site_out else v


def lnl_batch(codes, parent, branch, base, K, logits, assign, pinv, rates, nthreads=0):
    """OpenMP-over-particles full refresh of a batch; arrays are [np, ...]."""
    c, cp = _u(codes)
    T, S = c.shape
    par, pp = _i(parent)
    npart = par.shape[0]
    br, bp = _d(branch)
    ba, bap = _d(base)
    kk, kp = _i(K)
    lg, lgp = _d(logits)
    kmax = lg.shape[1]
    asg, ap = _i(assign)
    pv, pvp = _d(pinv)
    rt, rp = _d(rates)
    R = rt.shape[1]
    out = np.zeros(npart)
    lib().orc_lnl_batch(npart, T, S, R, cp, pp, bp, bap, kp, kmax, lgp, ap, pvp, rp,
                        out.ctypes.data_as(_dp), int(nthreads))
    return out


def max_threads() -> int:
    return lib().orc_max_threads()


def ln_prior(T, S, R, lg, branch, shape, base, logits, counts, dpp_alpha=0.01):
    br, bp = _d(branch)
    ba, bap = _d(base)
    logits = np.atleast_2d(np.asarray(logits, dtype=np.float64))
    lgt, lgp = _d(logits)
    cn, cnp = _i(counts)
    return lib().orc_ln_prior(T, S, R, int(lg), bp, float(shape), bap, logits.shape[0], lgp,
                              cnp, float(dpp_alpha))


def next_step(raw_w, lnl_vals, target_ess, last_temp):
    """computeNextStep: returns (new raw weights, normalised weights, ESS, temp)."""
    rw = np.array(raw_w, dtype=np.float64, copy=True)
    ll, llp = _d(lnl_vals)
    nw = np.zeros_like(rw)
    ess = ctypes.c_double(0.0)
    temp = ctypes.c_double(0.0)
    lib().orc_next_step(len(rw), rw.ctypes.data_as(_dp), llp, nw.ctypes.data_as(_dp),
                        ctypes.byref(ess), float(target_ess), ctypes.byref(temp),
                        float(last_temp))
    return rw, nw, ess.value, temp.value


def gibbs_weights(codes, parent, branch, base, logits, counts, pinv, rates, site,
                  aux_logits, temp, dpp_alpha=0.01):
    c, cp = _u(codes)
    T, S = c.shape
    rates = np.atleast_1d(np.asarray(rates, dtype=np.float64))
    logits = np.atleast_2d(np.asarray(logits, dtype=np.float64))
    aux = np.atleast_2d(np.asarray(aux_logits, dtype=np.float64))
    K, m = logits.shape[0], aux.shape[0]
    par, pp = _i(parent)
    br, bp = _d(branch)
    ba, bap = _d(base)
    lg, lgp = _d(logits)
    cn, cnp = _i(counts)
    rt, rp = _d(rates)
    ax, axp = _d(aux)
    out = np.zeros(K + m)
    lib().orc_gibbs_weights(T, S, len(rates), cp, pp, bp, bap, K, lgp, cnp, float(pinv), rp,
                            int(site), m, axp, float(temp), float(dpp_alpha),
                            out.ctypes.data_as(_dp))
    return out

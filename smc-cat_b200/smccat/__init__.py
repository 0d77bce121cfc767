"""Python binding of the B200 Smc-CAT likelihood engine (ctypes over the C-ABI).

Everything here calls ``lib/libsmccat.so`` through the functions declared in
``include/smccat.h``; there is no Python or CPU fallback. Importing works
without a GPU (the library loads, host-only helpers run); creating an
:class:`Engine` needs a CUDA device and raises :class:`SmccatError` otherwise.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_DIR, "lib", "libsmccat.so")
HEADER_PATH = os.path.join(os.path.dirname(_PKG_DIR), "include", "smccat.h")

OK, EINVAL, ECUDA, ENOMEM, ESTATE, ENUMERIC, ENODEV, ETIMEOUT = range(8)
MODEL_LG, MODEL_INVAR, MODEL_CAT, MODEL_PATTERNS = 1, 2, 4, 8
PREC_FP64, PREC_FP32 = 0, 1
REFRESH_DIRTY, REFRESH_FULL = 0, 1

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_up = ctypes.POINTER(ctypes.c_uint8)
_i32 = ctypes.c_int32


class SmccatError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"smccat error {code}: {msg}")
        self.code = code


KERNEL_NAMES = ("spec", "pmat", "prune", "reduce", "accept")


class Profile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_uint64 * 5), ("ms", ctypes.c_double * 5),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64)]


class Tuning(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "adaptive_nni_epsilon", "shape_delta", "scale_delta", "subtree_scale_delta",
        "stationary_delta", "rate_matrix_delta", "invar_alpha", "dpp_alpha")]


class MoveStats(ctypes.Structure):
    _fields_ = [("proposed", ctypes.c_uint64 * 10), ("accepted", ctypes.c_uint64 * 10),
                ("lockstep_steps", ctypes.c_uint64)]


MOVE_NAMES = ("Adaptive NNI", "NNI", "SPR", "Branch Length", "Scale Subtree",
              "Proportion Invariant", "Rate Shape", "Stationary", "Rate Matrix Single",
              "Rate Matrix Full")
FAMILY_TREE, FAMILY_STATIONARY, FAMILY_SHAPE, FAMILY_INVAR, FAMILY_RATE_MATRIX = range(5)


class GibbsStats(ctypes.Structure):
    _fields_ = [("particles", ctypes.c_int64), ("classes_before", ctypes.c_int64),
                ("classes_after", ctypes.c_int64), ("created", ctypes.c_int64)]


class LearnedStats(ctypes.Structure):
    _fields_ = [("proposed", ctypes.c_int64), ("accepted", ctypes.c_int64)]


MLP_PARAMS, MLP_INPUTS = 22401, 44
_fp = ctypes.POINTER(ctypes.c_float)


class Config(ctypes.Structure):
    _fields_ = [("num_taxa", _i32), ("num_sites", _i32), ("num_rates", _i32),
                ("max_particles", _i32), ("max_classes", _i32), ("model_flags", _i32),
                ("precision", _i32), ("device", _i32)]


_lib = None


def build() -> str:
    """Compile libsmccat.so in-tree with the package Makefile."""
    subprocess.run(["make", "-s", "-C", _PKG_DIR], check=True)
    return LIB_PATH


def lib():
    """Load the engine library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {_PKG_DIR}`")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    sig = {
        "smccat_version": ([], ctypes.c_char_p),
        "smccat_last_error": ([], ctypes.c_char_p),
        "smccat_discretize_gamma": ([ctypes.c_double, _i32, _dp], ctypes.c_int),
        "smccat_lg_exchangeabilities": ([_dp], ctypes.c_int),
        "smccat_create": ([ctypes.POINTER(Config), _up, ctypes.POINTER(vp)], ctypes.c_int),
        "smccat_destroy": ([vp], ctypes.c_int),
        "smccat_device_bytes": ([vp, ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
        "smccat_set_particles": ([vp, _i32, _i32, _ip, _dp, _dp, _ip, _dp, _ip, _dp, _dp],
                                 ctypes.c_int),
        "smccat_get_particles": ([vp, _i32, _i32, _ip, _dp, _dp, _ip, _dp, _ip, _dp, _dp],
                                 ctypes.c_int),
        "smccat_refresh": ([vp, _i32, _i32, _i32], ctypes.c_int),
        "smccat_get_lnl": ([vp, _i32, _i32, _dp], ctypes.c_int),
        "smccat_get_site_lnl": ([vp, _i32, _dp], ctypes.c_int),
        "smccat_get_transition_matrix": ([vp, _i32, _i32, _i32, _i32, _dp], ctypes.c_int),
        "smccat_set_branch_lengths": ([vp, _i32, _i32, _ip, _dp], ctypes.c_int),
        "smccat_set_topology": ([vp, _i32, _ip, _dp], ctypes.c_int),
        "smccat_set_pinv": ([vp, _i32, ctypes.c_double], ctypes.c_int),
        "smccat_set_shape": ([vp, _i32, ctypes.c_double], ctypes.c_int),
        "smccat_set_base": ([vp, _i32, _dp], ctypes.c_int),
        "smccat_set_class_logits": ([vp, _i32, _i32, _dp], ctypes.c_int),
        "smccat_accept": ([vp, _i32, _i32, _up], ctypes.c_int),
        "smccat_sync": ([vp], ctypes.c_int),
        "smccat_get_stream": ([vp, ctypes.POINTER(vp)], ctypes.c_int),
        "smccat_set_profiling": ([vp, _i32], ctypes.c_int),
        "smccat_autotune": ([vp, _i32, _ip, _dp], ctypes.c_int),
        "smccat_kernel_variants": ([vp, _ip, _ip], ctypes.c_int),
        "smccat_set_kernel_variant": ([vp, _i32], ctypes.c_int),
        "smccat_set_wait_limit": ([vp, _i32], ctypes.c_int),
        "smccat_set_reassign_group": ([vp, _i32], ctypes.c_int),
        "smccat_set_tuning": ([vp, ctypes.POINTER(Tuning)], ctypes.c_int),
        "smccat_get_tuning": ([vp, ctypes.POINTER(Tuning)], ctypes.c_int),
        "smccat_set_rate_cholesky": ([vp, _dp], ctypes.c_int),
        "smccat_set_split_posteriors": ([vp, _i32, ctypes.POINTER(ctypes.c_uint64), _dp],
                                        ctypes.c_int),
        "smccat_compute_split_posteriors": ([vp, _i32, _i32, _dp, _i32, _ip,
                                             ctypes.POINTER(ctypes.c_uint64), _dp], ctypes.c_int),
        "smccat_ln_prior": ([vp, _i32, _i32, _dp], ctypes.c_int),
        "smccat_resample_tune": ([vp, _i32, _i32, _dp, ctypes.c_double, _i32, _ip], ctypes.c_int),
        "smccat_get_rate_cholesky": ([vp, _dp], ctypes.c_int),
        "smccat_tree_sweep": ([vp, _i32, _i32, _i32, ctypes.c_double, ctypes.c_uint64, _i32,
                                 ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
        "smccat_propose": ([vp, _i32, _i32, ctypes.c_uint64, _ip, _dp], ctypes.c_int),
        "smccat_rejuvenate": ([vp, _i32, _i32, _i32, ctypes.c_double, ctypes.c_uint64,
                               ctypes.POINTER(MoveStats)], ctypes.c_int),
        "smccat_mcmc_sweep": ([vp, _i32, _i32, _i32, ctypes.c_double, ctypes.c_uint64, _i32,
                               ctypes.POINTER(MoveStats)], ctypes.c_int),
        "smccat_smc_step": ([vp, _i32, _i32, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp,
                             _dp], ctypes.c_int),
        "smccat_gibbs": ([vp, _i32, _i32, _up, ctypes.c_double, ctypes.c_uint64,
                          ctypes.POINTER(GibbsStats)], ctypes.c_int),
        "smccat_gibbs_weights": ([vp, _i32, _i32, _dp, ctypes.c_double, _dp], ctypes.c_int),
        "smccat_learned_train": ([vp, _i32, _i32, _i32, _i32, ctypes.c_double, ctypes.c_uint64,
                                  _dp], ctypes.c_int),
        "smccat_learned_gradients": ([vp, _i32, _ip, _fp, _ip, _fp, _dp], ctypes.c_int),
        "smccat_learned_params": ([vp, _fp, _fp], ctypes.c_int),
        "smccat_learned_move": ([vp, _i32, _i32, _up, _i32, ctypes.c_double, ctypes.c_uint64,
                                 ctypes.POINTER(LearnedStats)], ctypes.c_int),
        "smccat_learned_scores": ([vp, _i32, _i32, _dp], ctypes.c_int),
        "smccat_get_profile": ([vp, ctypes.POINTER(Profile)], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _check(rc: int):
    if rc != OK:
        raise SmccatError(rc, lib().smccat_last_error().decode())


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def version() -> str:
    return lib().smccat_version().decode()


def discretize_gamma(shape: float, num_rates: int) -> np.ndarray:
    out = np.zeros(num_rates)
    _check(lib().smccat_discretize_gamma(float(shape), int(num_rates), out.ctypes.data_as(_dp)))
    return out


def lg_exchangeabilities() -> np.ndarray:
    out = np.zeros(190)
    _check(lib().smccat_lg_exchangeabilities(out.ctypes.data_as(_dp)))
    return out


class Engine:
    """One device context over a fixed alignment and a batch of particles.

    Mirrors the reference's per-particle likelihood interface
    (``class Particle``, src/analysis/Particle.hpp:48-125) as batched calls.
    """

    def __init__(self, codes, num_rates: int, max_particles: int, max_classes: int = 1,
                 lg: bool = False, invar: bool = False, cat: bool = False, device: int = 0,
                 precision: int = PREC_FP64, patterns: bool = False):
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        self.T, self.S = codes.shape
        self.R = int(num_rates)
        self.N = 2 * self.T - 1
        self.P = int(max_particles)
        self.Kmax = int(max_classes)
        flags = (MODEL_LG if lg else 0) | (MODEL_INVAR if invar else 0) | (MODEL_CAT if cat else 0)
        flags |= MODEL_PATTERNS if patterns else 0
        self.precision = int(precision)
        cfg = Config(self.T, self.S, self.R, self.P, self.Kmax, flags, self.precision, device)
        h = ctypes.c_void_p()
        _check(lib().smccat_create(ctypes.byref(cfg), codes.ctypes.data_as(_up), ctypes.byref(h)))
        self._h = h
        self._codes = codes

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().smccat_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        v = ctypes.c_uint64(0)
        _check(lib().smccat_device_bytes(self._h, ctypes.byref(v)))
        return v.value

    # -- particle state ---------------------------------------------------
    def set_particles(self, first, parent, branch, base, num_classes, logits, assign, pinv, shape):
        par, pp = _i(parent)
        n = par.shape[0]
        br, bp = _d(branch)
        ba, bap = _d(base)
        nk, nkp = _i(num_classes)
        lg = np.zeros((n, self.Kmax, 20))
        lgs = np.asarray(logits, dtype=np.float64).reshape(n, -1, 20)
        lg[:, :lgs.shape[1], :] = lgs
        lg, lgp = _d(lg)
        asg, ap = _i(assign)
        pv, pvp = _d(pinv)
        sh, shp = _d(shape)
        _check(lib().smccat_set_particles(self._h, int(first), n, pp, bp, bap, nkp, lgp, ap, pvp, shp))

    def get_particles(self, first=0, count=None):
        count = self.P - first if count is None else count
        out = dict(parent=np.zeros((count, self.N), np.int32), branch=np.zeros((count, self.N)),
                   base=np.zeros((count, 190)), num_classes=np.zeros(count, np.int32),
                   logits=np.zeros((count, self.Kmax, 20)),
                   assign=np.zeros((count, self.S), np.int32), pinv=np.zeros(count),
                   shape=np.zeros(count))
        _check(lib().smccat_get_particles(
            self._h, int(first), int(count), out["parent"].ctypes.data_as(_ip),
            out["branch"].ctypes.data_as(_dp), out["base"].ctypes.data_as(_dp),
            out["num_classes"].ctypes.data_as(_ip), out["logits"].ctypes.data_as(_dp),
            out["assign"].ctypes.data_as(_ip), out["pinv"].ctypes.data_as(_dp),
            out["shape"].ctypes.data_as(_dp)))
        return out

    def refresh(self, first=0, count=None, full=False):
        count = self.P - first if count is None else count
        _check(lib().smccat_refresh(self._h, int(first), int(count),
                                    REFRESH_FULL if full else REFRESH_DIRTY))

    def lnl(self, first=0, count=None) -> np.ndarray:
        count = self.P - first if count is None else count
        out = np.zeros(count)
        _check(lib().smccat_get_lnl(self._h, int(first), int(count), out.ctypes.data_as(_dp)))
        return out

    def site_lnl(self, p) -> np.ndarray:
        out = np.zeros(self.S)
        _check(lib().smccat_get_site_lnl(self._h, int(p), out.ctypes.data_as(_dp)))
        return out

    def transition_matrix(self, p, k, node, r) -> np.ndarray:
        """P(t r) (row-major 20x20) of particle p, class k, edge above node."""
        out = np.zeros((20, 20))
        _check(lib().smccat_get_transition_matrix(self._h, int(p), int(k), int(node), int(r),
                                                  out.ctypes.data_as(_dp)))
        return out

    # -- edits --------------------------------------------------------------
    def set_branch_lengths(self, p, nodes, lengths):
        nd, ndp = _i(nodes)
        ln, lnp = _d(lengths)
        _check(lib().smccat_set_branch_lengths(self._h, int(p), len(nd), ndp, lnp))

    def set_topology(self, p, parent, branch):
        par, pp = _i(parent)
        br, bp = _d(branch)
        _check(lib().smccat_set_topology(self._h, int(p), pp, bp))

    def set_pinv(self, p, v):
        _check(lib().smccat_set_pinv(self._h, int(p), float(v)))

    def set_shape(self, p, v):
        _check(lib().smccat_set_shape(self._h, int(p), float(v)))

    def set_base(self, p, base):
        b, bp = _d(base)
        _check(lib().smccat_set_base(self._h, int(p), bp))

    def set_class_logits(self, p, k, logits):
        lg, lgp = _d(logits)
        _check(lib().smccat_set_class_logits(self._h, int(p), int(k), lgp))

    def accept(self, mask, first=0):
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        _check(lib().smccat_accept(self._h, int(first), len(m), m.ctypes.data_as(_up)))

    def sync(self):
        _check(lib().smccat_sync(self._h))

    # -- MCMC / SMC ---------------------------------------------------------
    def tuning(self) -> dict:
        t = Tuning()
        _check(lib().smccat_get_tuning(self._h, ctypes.byref(t)))
        return {n: getattr(t, n) for n, _ in Tuning._fields_}

    def set_tuning(self, **kw):
        cur = self.tuning()
        cur.update(kw)
        t = Tuning(**cur)
        _check(lib().smccat_set_tuning(self._h, ctypes.byref(t)))

    def set_rate_cholesky(self, L):
        a, ap = _d(np.tril(np.asarray(L, dtype=np.float64)))
        _check(lib().smccat_set_rate_cholesky(self._h, ap))

    def set_split_posteriors(self, bits, probs):
        b = np.ascontiguousarray(bits, dtype=np.uint64).reshape(-1, 2)
        pr, prp = _d(probs)
        _check(lib().smccat_set_split_posteriors(
            self._h, len(pr), b.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), prp))

    def compute_split_posteriors(self, weights=None, first=0, count=None, cap=None):
        """computeSplitPosteriors over the particles' trees; also installs the
        result for the adaptive NNI move. Returns (bits [n, 2] uint64, prob [n])."""
        count = self.P - first if count is None else count
        wp = None
        if weights is not None:
            w, wp = _d(weights)
        n = ctypes.c_int32(0)
        _check(lib().smccat_compute_split_posteriors(self._h, int(first), int(count), wp, 0,
                                                     ctypes.byref(n), None, None))
        cap = n.value if cap is None else int(cap)
        bits = np.zeros((max(cap, 1), 2), dtype=np.uint64)
        prob = np.zeros(max(cap, 1))
        _check(lib().smccat_compute_split_posteriors(
            self._h, int(first), int(count), wp, cap, ctypes.byref(n),
            bits.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), prob.ctypes.data_as(_dp)))
        m = min(cap, n.value)
        return bits[:m], prob[:m]

    def tree_sweep(self, steps, temperature, seed, use_graph=True, first=0, count=None) -> dict:
        """Tree-move MCMC steps (the reference's treeMove mixture) entirely on
        the device, one CUDA graph; returns proposed / accepted per move kind."""
        count = self.P - first if count is None else count
        st = np.zeros(10, dtype=np.int64)
        _check(lib().smccat_tree_sweep(self._h, int(first), int(count), int(steps),
                                       float(temperature), int(seed), 1 if use_graph else 0,
                                       st.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        out = {}
        for k, name in enumerate(("adaptive_nni", "nni", "spr", "branch", "subtree")):
            out[name + "_proposed"] = int(st[2 * k])
            out[name + "_accepted"] = int(st[2 * k + 1])
        return out

    def rate_cholesky(self) -> np.ndarray:
        out = np.zeros((190, 190))
        _check(lib().smccat_get_rate_cholesky(self._h, out.ctypes.data_as(_dp)))
        return out

    def resample_tune(self, norm_weights, u, copy=True, first=0) -> np.ndarray:
        """Systematic resampling + the reference's proposal tuning; returns the
        ancestor of every slot of [first, first + len(norm_weights))."""
        w, wp = _d(norm_weights)
        anc = np.zeros(len(w), dtype=np.int32)
        _check(lib().smccat_resample_tune(self._h, int(first), len(w), wp, float(u),
                                          1 if copy else 0, anc.ctypes.data_as(_ip)))
        return anc

    def ln_prior(self, first=0, count=None) -> np.ndarray:
        count = self.P - first if count is None else count
        out = np.zeros(count)
        _check(lib().smccat_ln_prior(self._h, int(first), int(count), out.ctypes.data_as(_dp)))
        return out

    def propose(self, p, family, seed):
        k = ctypes.c_int32(-1)
        h = ctypes.c_double(0.0)
        _check(lib().smccat_propose(self._h, int(p), int(family), int(seed), ctypes.byref(k),
                                    ctypes.byref(h)))
        return int(k.value), float(h.value)

    def rejuvenate(self, iterations, temperature, seed, first=0, count=None) -> dict:
        count = self.P - first if count is None else count
        st = MoveStats()
        _check(lib().smccat_rejuvenate(self._h, int(first), int(count), int(iterations),
                                       float(temperature), int(seed), ctypes.byref(st)))
        return {"proposed": list(st.proposed), "accepted": list(st.accepted),
                "lockstep_steps": int(st.lockstep_steps)}

    def mcmc_sweep(self, iterations, temperature, seed, use_graph=True, first=0,
                   count=None) -> dict:
        """Mcmc::operator() on every particle with everything on the device
        (smccat_mcmc_sweep); the whole sweep is one CUDA graph by default."""
        count = self.P - first if count is None else count
        st = MoveStats()
        _check(lib().smccat_mcmc_sweep(self._h, int(first), int(count), int(iterations),
                                       float(temperature), int(seed), 1 if use_graph else 0,
                                       ctypes.byref(st)))
        return {"proposed": list(st.proposed), "accepted": list(st.accepted),
                "lockstep_steps": int(st.lockstep_steps)}

    def gibbs(self, temperature, seed, mask=None, first=0, count=None) -> dict:
        count = self.P - first if count is None else count
        st = GibbsStats()
        mp = None
        if mask is not None:
            m = np.ascontiguousarray(mask, dtype=np.uint8)
            mp = m.ctypes.data_as(_up)
        _check(lib().smccat_gibbs(self._h, int(first), int(count), mp, float(temperature),
                                  int(seed), ctypes.byref(st)))
        return {n: int(getattr(st, n)) for n, _ in GibbsStats._fields_}

    def gibbs_weights(self, p, site, aux_logits, temperature, num_classes) -> np.ndarray:
        aux, ap = _d(np.asarray(aux_logits, dtype=np.float64).reshape(5, 20))
        out = np.zeros(int(num_classes) + 5)
        _check(lib().smccat_gibbs_weights(self._h, int(p), int(site), ap, float(temperature),
                                          out.ctypes.data_as(_dp)))
        return out

    # -- learned CAT proposal ------------------------------------------------
    def learned_train(self, epochs, batch_sites=512, lr=1e-3, seed=0, first=0, count=None):
        count = self.P - first if count is None else count
        loss = ctypes.c_double(0.0)
        _check(lib().smccat_learned_train(self._h, int(first), int(count), int(epochs),
                                          int(batch_sites), float(lr), int(seed), ctypes.byref(loss)))
        return loss.value

    def learned_params(self, set_to=None) -> np.ndarray:
        out = np.zeros(MLP_PARAMS, dtype=np.float32)
        src = None
        if set_to is not None:
            src = np.ascontiguousarray(set_to, dtype=np.float32)
        _check(lib().smccat_learned_params(self._h, out.ctypes.data_as(_fp),
                                           src.ctypes.data_as(_fp) if src is not None else None))
        return out

    def learned_gradients(self, x, group_off, labels):
        xx = np.ascontiguousarray(x, dtype=np.float32)
        off, offp = _i(group_off)
        lab, labp = _i(labels)
        g = np.zeros(MLP_PARAMS, dtype=np.float32)
        loss = ctypes.c_double(0.0)
        _check(lib().smccat_learned_gradients(self._h, len(lab), offp, xx.ctypes.data_as(_fp), labp,
                                              g.ctypes.data_as(_fp), ctypes.byref(loss)))
        return loss.value, g

    def learned_move(self, updates, temperature, seed, mask=None, first=0, count=None) -> dict:
        count = self.P - first if count is None else count
        st = LearnedStats()
        mp = None
        if mask is not None:
            m = np.ascontiguousarray(mask, dtype=np.uint8)
            mp = m.ctypes.data_as(_up)
        _check(lib().smccat_learned_move(self._h, int(first), int(count), mp, int(updates),
                                         float(temperature), int(seed), ctypes.byref(st)))
        return {"proposed": int(st.proposed), "accepted": int(st.accepted)}

    def learned_scores(self, p, site, num_classes) -> np.ndarray:
        """The learned proposal's score of every class of particle p at `site`."""
        out = np.zeros(int(num_classes))
        _check(lib().smccat_learned_scores(self._h, int(p), int(site), out.ctypes.data_as(_dp)))
        return out

    def smc_step(self, raw_weights, target_ess, last_temp, first=0):
        w = np.array(raw_weights, dtype=np.float64, copy=True)
        nw = np.zeros_like(w)
        t = ctypes.c_double(0.0)
        e = ctypes.c_double(0.0)
        _check(lib().smccat_smc_step(self._h, int(first), len(w), w.ctypes.data_as(_dp),
                                     float(target_ess), float(last_temp), ctypes.byref(t),
                                     ctypes.byref(e), nw.ctypes.data_as(_dp)))
        return w, nw, e.value, t.value

    # -- measurement --------------------------------------------------------
    @property
    def stream_ptr(self) -> int:
        """The cudaStream_t the engine launches on (for caller-side events)."""
        v = ctypes.c_void_p()
        _check(lib().smccat_get_stream(self._h, ctypes.byref(v)))
        return v.value or 0

    def autotune(self, reps: int = 3) -> dict:
        """Pick the fastest pruning-kernel variant on the loaded particles."""
        v = ctypes.c_int32(0)
        ms = np.full(self.kernel_variants()[0], np.nan)
        _check(lib().smccat_autotune(self._h, int(reps), ctypes.byref(v), ms.ctypes.data_as(_dp)))
        return {"variant": int(v.value), "ms": [float(x) for x in ms if not np.isnan(x)]}

    def kernel_variants(self):
        """(number of pruning-kernel variants, the one in use)."""
        n, cur = ctypes.c_int32(0), ctypes.c_int32(0)
        _check(lib().smccat_kernel_variants(self._h, ctypes.byref(n), ctypes.byref(cur)))
        return int(n.value), int(cur.value)

    def set_kernel_variant(self, v: int):
        _check(lib().smccat_set_kernel_variant(self._h, int(v)))

    def set_wait_limit(self, polls: int):
        """Polls per bounded device wait; a negative value restores the default."""
        _check(lib().smccat_set_wait_limit(self._h, int(polls)))

    def set_reassign_group(self, n: int):
        """Particles per device pass of Gibbs / the learned move (0: from free memory)."""
        _check(lib().smccat_set_reassign_group(self._h, int(n)))

    def set_profiling(self, enable: bool):
        _check(lib().smccat_set_profiling(self._h, 1 if enable else 0))

    def profile(self) -> dict:
        pr = Profile()
        _check(lib().smccat_get_profile(self._h, ctypes.byref(pr)))
        return dict(launches={n: int(pr.launches[i]) for i, n in enumerate(KERNEL_NAMES)},
                    ms={n: float(pr.ms[i]) for i, n in enumerate(KERNEL_NAMES)},
                    h2d_bytes=int(pr.h2d_bytes), d2h_bytes=int(pr.d2h_bytes))

"""Pruning under reduced-precision arithmetic -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference's likelihood (refreshLikelihood(true),
Particle.cpp:530-675: tips as one-hot / all-ones vectors, pN = prod over the
two children of P(child, r) . pChild, per-(site, r) rescaling by the maximum,
root reduction without a 1/R weight, pinv mixing) in which the matrix-vector
products run in a chosen arithmetic, so that the log-likelihood error of each
arithmetic can be measured against FP64 on the same state:

  "fp64"    FP64 partials and products (equals oracle.lnl to rounding);
  "fp32"    FP32 partials and matrices, the engine's FP32 summation order;
  "bf16x3"  FP32 partials and matrices split into BF16 hi + lo parts, each
            product as hi.hi + hi.lo + lo.hi with FP32 accumulation -- the
            split-operand form a BF16 tensor-core kernel would compute;
  "tf32x3"  the same split with TF32 parts: hi = x rounded to TF32,
            lo = x - hi read truncated as a tensor core reads an FP32 operand;
  "tf32x3raw" the FP32 operand itself as hi (read truncated), lo likewise:
            both parts cut toward zero;
  "bf16"    BF16 operands, one product, FP32 accumulation;
  "fp16x3"  the split with FP16 parts (hi = x rounded to FP16, lo = the
            rounded remainder; FP16's 5-bit exponent flushes small entries
            and remainders to subnormals or zero) -- the kind::f16 form,
            twice the TF32 MMA rate;
  "fp16"    FP16 operands, one product, FP32 accumulation.

Rescaling is by exact powers of two and the log-scalers and root sums are
FP64 in every mode, as in the engine's kernels; only the node products and the
stored partials change precision. Transition matrices come from the FP64
oracle (oracle.transition). Only tests and the design study at the bottom of
this file use it.
"""
from __future__ import annotations

import numpy as np

import oracle

MODES = ("fp64", "fp32", "tf32x3", "tf32x3raw", "bf16x3", "bf16", "fp16x3", "fp16")


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to the nearest BF16 (ties to even), kept as FP32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def tf32_round(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to TF32 (10 stored mantissa bits; ties away from zero,
    as cvt.rna.tf32.f32), kept as FP32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x1000) & 0xFFFFE000
    return u.astype(np.uint32).view(np.float32)


def tf32_trunc(x: np.ndarray) -> np.ndarray:
    """The TF32 value a tensor core reads from an FP32 operand: the low 13
    mantissa bits dropped."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    return (u & np.uint32(0xFFFFE000)).view(np.float32)


def _split_tf32(x: np.ndarray, raw: bool = False):
    """hi = x rounded to TF32 and lo = x - hi (exact in FP32, read truncated
    by the tensor core). raw: the FP32 operand itself as hi, read truncated,
    so both parts are cut toward zero."""
    x = x.astype(np.float32)
    hi = tf32_trunc(x) if raw else tf32_round(x)
    lo = tf32_trunc(x - hi)
    return hi, lo


def fp16_round(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to the nearest FP16 (ties to even, subnormals kept,
    no overflow for the [0, 1] values of partials and matrices), as FP32."""
    return np.asarray(x, dtype=np.float32).astype(np.float16).astype(np.float32)


def _split(x: np.ndarray, rnd=bf16_round):
    x = x.astype(np.float32)
    hi = rnd(x)
    lo = rnd(x - hi)
    return hi, lo


def _parts(x: np.ndarray, mode: str):
    """hi, lo operand parts of a split mode (lo unused by the one-product modes)."""
    if mode.startswith("tf32"):
        return _split_tf32(x, mode == "tf32x3raw")
    return _split(x, fp16_round if mode.startswith("fp16") else bf16_round)


def _fma32(a, b, c):
    """FP32 fused multiply-add: the product of two FP32 values is exact in
    FP64; the sum is rounded once to FP64 and once to FP32."""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def _product(P: np.ndarray, X: np.ndarray, mode: str) -> np.ndarray:
    """P [20, 20] (FP64 values) times partials X [20, n] in `mode`.

    fp32 follows the engine's FP32 mat-vec exactly in order: two FMA chains
    over the even and the odd off-diagonal columns, then the diagonal term
    fused onto their sum. The BF16 forms are what a tensor-core kernel would
    compute: the off-diagonal part of P as one accumulation per split
    product (hi.hi, then hi.lo, then lo.hi, each over the columns in order,
    products exact, FP32 sums), the diagonal term fused on in the epilogue
    from the FP32 values."""
    if mode == "fp64":
        return P @ X
    P32 = P.astype(np.float32)
    X32 = X.astype(np.float32)
    diag = np.diagonal(P32)[:, None]
    off = P32.copy()
    np.fill_diagonal(off, 0.0)
    acc = np.zeros_like(X32)
    if mode == "fp32":
        s0 = np.zeros_like(X32)
        s1 = np.zeros_like(X32)
        for j in range(0, 20, 2):
            s0 = _fma32(off[:, j:j + 1], X32[j][None, :], s0)
            s1 = _fma32(off[:, j + 1:j + 2], X32[j + 1][None, :], s1)
        acc = (s0.astype(np.float64) + s1).astype(np.float32)
    else:
        Oh, Ol = _parts(off, mode)
        Xh, Xl = _parts(X32, mode)
        terms = [(Oh, Xh)] if mode in ("bf16", "fp16") else [(Oh, Xh), (Oh, Xl), (Ol, Xh)]
        for A, B in terms:
            for j in range(20):
                acc = _fma32(A[:, j:j + 1], B[j][None, :], acc)
    return _fma32(diag, X32, acc)


def _column(P: np.ndarray, codes: np.ndarray, mode: str) -> np.ndarray:
    """P times the tip vectors of `codes` (one-hot, all ones for 20-22)."""
    if mode == "fp64":
        Pc = P
    else:
        P32 = P.astype(np.float32)
        if mode == "fp32":
            Pc = P32
        else:
            Ph, Pl = _parts(P32, mode)
            Pc = Ph if mode in ("bf16", "fp16") else Ph + Pl
    full = np.concatenate([Pc, Pc.sum(axis=1, keepdims=True)], axis=1)  # col 20 = row sums
    return full[:, np.minimum(codes, 20)]


def lnl(codes, parent, branch, base, logits, assign, pinv, rates, mode: str = "fp64") -> float:
    """lnL of one particle state with the node products in `mode`."""
    codes = np.asarray(codes, dtype=np.uint8)
    T, S = codes.shape
    N = 2 * T - 1
    parent = np.asarray(parent)
    branch = np.asarray(branch, dtype=np.float64)
    logits = np.atleast_2d(np.asarray(logits, dtype=np.float64))
    assign = np.asarray(assign)
    rates = np.atleast_1d(np.asarray(rates, dtype=np.float64))
    R = len(rates)
    K = logits.shape[0]
    post = oracle.postorder(parent)
    kids = {}
    for n in range(N):
        if parent[n] >= 0:
            kids.setdefault(int(parent[n]), []).append(n)
    root = int(np.flatnonzero(parent < 0)[0])
    isinv, invchar = oracle.tip_encode(codes)
    store = np.float64 if mode == "fp64" else np.float32
    site_l = np.zeros(S)
    for k in range(K):
        idx = np.flatnonzero(assign == k)
        if idx.size == 0:
            continue
        pi = oracle.softmax20(logits[k])
        P = {(n, r): oracle.transition(base, pi, branch[n] * rates[r])
             for n in range(N) if n != root for r in range(R)}
        cl = {}
        lsc = {}
        for n in post:
            n = int(n)
            if n < T:
                continue
            for r in range(R):
                acc = None
                ls = np.zeros(idx.size)
                for c in kids[n]:
                    if c < T:
                        v = _column(P[c, r], codes[c, idx], mode)
                    else:
                        v = _product(P[c, r], cl[c, r], mode)
                        ls = ls + lsc[c, r]
                    acc = v if acc is None else (acc * v).astype(v.dtype)
                m = acc.max(axis=0)
                e = np.frexp(m.astype(np.float64))[1]
                acc = (acc * np.ldexp(1.0, -e).astype(acc.dtype)).astype(store)
                cl[n, r] = acc
                lsc[n, r] = ls + e * np.log(2.0)
        lr = np.stack([np.log(pi @ cl[root, r].astype(np.float64)) + lsc[root, r] for r in range(R)])
        mx = lr.max(axis=0)
        L = np.exp(mx + np.log(np.exp(lr - mx).sum(axis=0)))  # no 1/R weight (Particle.cpp:660-668)
        inv = pinv * pi[invchar[idx]] * isinv[idx]
        site_l[idx] = L * (1.0 - pinv) + inv
    return float(np.sum(np.log(site_l)))


def study(T: int, S: int, K: int, seed: int = 0) -> dict:
    """|lnL(mode) - lnL(fp64)| for one simulated CAT-GTR+G4 state."""
    import sys, os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "smc-cat_b200"))
    from smccat import workload
    cfg = workload.WorkloadConfig("study", T=T, S=S, R=4, particles=1, iterations=1, lg=False,
                                  invar=True, cat=K > 1, alpha=0.5, pinv=0.1,
                                  k_range=(K, K), seed=seed)
    rng = np.random.default_rng(seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, 1, rng)
    Kp = int(st["num_classes"][0])
    args = (codes, st["parent"][0], st["branch"][0], st["base"][0], st["logits"][0][:Kp],
            st["assign"][0], float(st["pinv"][0]), oracle.discretize_gamma(st["shape"][0], 4))
    ref = lnl(*args, mode="fp64")
    out = {"lnl_fp64": ref, "lnl_oracle": oracle.lnl(*args), "classes": Kp}
    for m in MODES[1:]:
        out[m] = abs(lnl(*args, mode=m) - ref)
    return out


if __name__ == "__main__":
    import json
    import sys
    T, S, K = (int(v) for v in sys.argv[1:4]) if len(sys.argv) >= 4 else (100, 10000, 64)
    print(json.dumps(study(T, S, K)))

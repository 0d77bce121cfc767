"""Site-pattern compression (SMCCAT_MODEL_PATTERNS) against the uncompressed
engine and the oracle.

With compression each particle evaluates every distinct (alignment column,
class) pair once and weights it by its number of sites; the reference
evaluates every site. Log-likelihoods must agree to 1e-12 relative with the
uncompressed engine (only the summation order differs) and to 1e-9 with the
oracle; per-site values must be given for every site.
"""
import numpy as np
import pytest

import oracle
import smccat
from smccat import workload

from test_gpu_parity import SMALL, oracle_lnl

pytestmark = pytest.mark.gpu

REL = 1e-12


def pair(cfg, n, seed, kmax=None):
    rng = np.random.default_rng(seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, n, rng, kmax=kmax)
    engs = []
    for patterns in (False, True):
        e = smccat.Engine(codes, cfg.R, n, max_classes=st["logits"].shape[1], lg=cfg.lg,
                          invar=cfg.invar, cat=cfg.cat, patterns=patterns)
        e.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                        st["logits"], st["assign"], st["pinv"], st["shape"])
        e.refresh(full=True)
        engs.append(e)
    return engs[0], engs[1], codes, st


def assert_same(plain, comp, n):
    a, b = plain.lnl(), comp.lnl()
    np.testing.assert_allclose(b, a, rtol=REL, atol=0)
    for i in range(n):
        np.testing.assert_allclose(comp.site_lnl(i), plain.site_lnl(i), rtol=1e-11, atol=1e-11)


def duplicate_fraction(codes):
    return 1.0 - np.unique(codes.T, axis=0).shape[0] / codes.shape[1]


@pytest.mark.parametrize("cfg", SMALL + [workload.CONFIGS[1]], ids=lambda c: c.name)
def test_compressed_matches_uncompressed_and_oracle(cfg):
    n = min(cfg.particles, 8)
    plain, comp, codes, st = pair(cfg, n, cfg.seed)
    assert duplicate_fraction(codes) > 0.05  # the case exercises compression
    assert_same(plain, comp, n)
    got = comp.lnl()
    for i in range(n):
        ref, ref_site = oracle_lnl(codes, st, i, cfg.R)
        assert got[i] == pytest.approx(ref, rel=1e-9)
        np.testing.assert_allclose(comp.site_lnl(i), ref_site, rtol=1e-9, atol=1e-9)
    plain.close()
    comp.close()


def test_every_kernel_variant_with_compression():
    cfg = SMALL[2]  # CAT, R = 4, +I
    plain, comp, codes, st = pair(cfg, cfg.particles, cfg.seed)
    ref = plain.lnl()
    nv, _ = comp.kernel_variants()
    for v in range(nv):
        comp.set_kernel_variant(v)
        comp.refresh(full=True)
        np.testing.assert_allclose(comp.lnl(), ref, rtol=1e-11, atol=0, err_msg=f"variant {v}")
    plain.close()
    comp.close()


def test_dirty_edits_with_compression():
    cfg = SMALL[1]  # GTR + G4 + I
    n = cfg.particles
    plain, comp, codes, st = pair(cfg, n, cfg.seed)
    rng = np.random.default_rng(5)
    for step in range(6):
        p = int(rng.integers(n))
        node = int(rng.integers(2 * cfg.T - 1))
        if node == int(np.where(st["parent"][p] < 0)[0][0]):
            node = 0
        length = float(rng.exponential(0.1))
        pinv = float(rng.uniform(0.01, 0.3)) if step % 2 else float(st["pinv"][p])
        for e in (plain, comp):
            e.set_branch_lengths(p, [node], [length])
            e.set_pinv(p, pinv)
        mask = np.ones(n, np.uint8) if step % 3 else np.zeros(n, np.uint8)
        for e in (plain, comp):
            e.refresh()
        assert_same(plain, comp, n)
        for e in (plain, comp):
            e.accept(mask)
        assert_same(plain, comp, n)
    plain.close()
    comp.close()


def test_gibbs_reassignment_with_compression():
    """Gibbs changes the class sets; the next upload recompresses per class."""
    cfg = SMALL[2]
    n = cfg.particles
    plain, comp, codes, st = pair(cfg, n, cfg.seed, kmax=16)
    comp.gibbs(temperature=1.0, seed=3)
    fin = comp.get_particles()
    got = comp.lnl()
    for i in range(n):
        K = int(fin["num_classes"][i])
        rates = oracle.discretize_gamma(fin["shape"][i], cfg.R)
        ref = oracle.lnl(codes, fin["parent"][i], fin["branch"][i], fin["base"][i],
                         fin["logits"][i][:K], fin["assign"][i], fin["pinv"][i], rates)
        assert got[i] == pytest.approx(ref, rel=1e-9)
    plain.close()
    comp.close()

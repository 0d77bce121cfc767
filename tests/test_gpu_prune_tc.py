"""The tcgen05 3xTF32 pruning kernel (the last FP32 variant): full and dirty
refreshes against the FP64 oracle within the FP32 tolerance, and against the
SIMT FP32 kernel, on GTR, LG and CAT particles (partial 128-slot tiles
included), with and without site-pattern compression."""
import numpy as np
import pytest

import oracle
import smccat
from smccat import workload

pytestmark = pytest.mark.gpu

FP32_ATOL = 3e-4

CFGS = [
    workload.WorkloadConfig("tc_gtr", T=20, S=300, R=4, particles=12, iterations=1, lg=False,
                            invar=True, cat=False, alpha=0.5, pinv=0.1, seed=33),
    workload.WorkloadConfig("tc_lg", T=16, S=500, R=4, particles=6, iterations=1, lg=True,
                            invar=False, cat=False, alpha=0.8, pinv=0.0, seed=7),
    workload.WorkloadConfig("tc_cat", T=12, S=400, R=4, particles=6, iterations=1, lg=False,
                            invar=True, cat=True, alpha=0.6, pinv=0.1, k_range=(2, 9), seed=19),
    workload.WorkloadConfig("tc_r2", T=10, S=260, R=2, particles=5, iterations=1, lg=False,
                            invar=True, cat=False, alpha=0.4, pinv=0.2, seed=3),
]


def engine(cfg, patterns=False):
    rng = np.random.default_rng(cfg.seed)
    codes, _ = workload.simulate_alignment(cfg, rng)
    st = workload.make_particles(cfg, cfg.particles, rng)
    eng = smccat.Engine(codes, cfg.R, cfg.particles, max_classes=st["logits"].shape[1], lg=cfg.lg,
                        invar=cfg.invar, cat=cfg.cat, precision=smccat.PREC_FP32, patterns=patterns)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"],
                      st["logits"], st["assign"], st["pinv"], st["shape"])
    return eng, codes, st


def oracle_lnl(codes, cfg, s, i, sites=False):
    K = int(s["num_classes"][i])
    rates = oracle.discretize_gamma(s["shape"][i], cfg.R)
    return oracle.lnl(codes, s["parent"][i], s["branch"][i], s["base"][i], s["logits"][i][:K],
                      s["assign"][i], s["pinv"][i], rates, site_out=sites)


def tc_variant(eng):
    return eng.kernel_variants()[0] - 1


@pytest.mark.parametrize("cfg", CFGS, ids=lambda c: c.name)
def test_tc_full_refresh_matches_oracle_and_simt(cfg):
    eng, codes, st = engine(cfg)
    eng.refresh(full=True)
    simt = eng.lnl()
    eng.set_kernel_variant(tc_variant(eng))
    eng.refresh(full=True)
    got = eng.lnl()
    for i in range(cfg.particles):
        ref, sites = oracle_lnl(codes, cfg, st, i, sites=True)
        assert abs(got[i] - ref) < FP32_ATOL
        np.testing.assert_allclose(eng.site_lnl(i), sites, rtol=0, atol=2e-5)
    np.testing.assert_allclose(got, simt, rtol=0, atol=FP32_ATOL)
    eng.close()


def test_tc_dirty_refresh_after_moves():
    cfg = CFGS[0]
    eng, codes, st = engine(cfg)
    eng.set_kernel_variant(tc_variant(eng))
    eng.refresh(full=True)
    st2 = {k: np.array(v, copy=True) for k, v in st.items()}
    for i in range(cfg.particles):
        x = (3 * i + 1) % (2 * cfg.T - 1)
        if st2["parent"][i][x] < 0:
            x = (x + 1) % (2 * cfg.T - 1)
        st2["branch"][i][x] *= 1.7
        eng.set_branch_lengths(i, [x], [st2["branch"][i][x]])
    eng.refresh()
    got = eng.lnl()
    for i in range(cfg.particles):
        assert abs(got[i] - oracle_lnl(codes, cfg, st2, i)) < FP32_ATOL
    eng.accept(np.ones(cfg.particles, np.uint8))
    # rejuvenation on the tensor-core kernel keeps exact bookkeeping
    eng.rejuvenate(iterations=1, temperature=0.8, seed=4)
    fin = eng.get_particles()
    got = eng.lnl()
    for i in range(cfg.particles):
        assert abs(got[i] - oracle_lnl(codes, cfg, fin, i)) < FP32_ATOL
    eng.close()


def test_tc_with_site_patterns():
    cfg = CFGS[1]
    eng, codes, st = engine(cfg, patterns=True)
    eng.set_kernel_variant(tc_variant(eng))
    eng.refresh(full=True)
    got = eng.lnl()
    for i in range(cfg.particles):
        assert abs(got[i] - oracle_lnl(codes, cfg, st, i)) < FP32_ATOL
    eng.close()


def test_tc_variant_is_in_the_autotuner():
    cfg = CFGS[0]
    eng, codes, st = engine(cfg)
    eng.refresh(full=True)
    n, _ = eng.kernel_variants()
    res = eng.autotune(reps=1)
    assert len(res["ms"]) == n
    assert all(np.isfinite(res["ms"]))
    eng.refresh(full=True)
    got = eng.lnl()
    for i in range(cfg.particles):
        assert abs(got[i] - oracle_lnl(codes, cfg, st, i)) < FP32_ATOL
    eng.close()


def test_tc_kernel_inside_the_device_tree_sweep():
    cfg = CFGS[0]
    eng, codes, st = engine(cfg)
    eng.set_kernel_variant(tc_variant(eng))
    eng.refresh(full=True)
    stats = eng.tree_sweep(steps=12, temperature=0.9, seed=8)
    assert sum(v for k, v in stats.items() if k.endswith("_proposed")) == 12 * cfg.particles
    fin = eng.get_particles()
    got = eng.lnl()
    for i in range(cfg.particles):
        assert abs(got[i] - oracle_lnl(codes, cfg, fin, i)) < FP32_ATOL
    eng.close()

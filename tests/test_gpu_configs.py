"""Parity at the shapes of the CAT workloads the engine is measured on, a few
particles each, against the FP64 oracle:

* 64 taxa x 5,000 sites, CAT-GTR+G4 (DP concentration 5);
* 100 taxa x 10,000 sites, uneven CAT: per-particle trees and K ~ U{8..120};
* 128 taxa x 20,000 sites, CAT-GTR+G4+I.

FP64 partials must match to 1e-9 relative per particle; FP32 partials (the
mixed-precision path) to 1e-3 nats per particle, the accuracy budget of the
mixed-precision sampler.
"""
import numpy as np
import pytest

import oracle
import smccat
from smccat import workload

pytestmark = pytest.mark.gpu

PARTICLES = 2


@pytest.fixture(scope="module", params=[3, 4, 5], ids=lambda c: workload.CONFIGS[c].name)
def case(request):
    cfg = workload.CONFIGS[request.param]
    codes, _ = workload.simulate_alignment(cfg, np.random.default_rng(cfg.seed))
    st = workload.make_particles(cfg, PARTICLES, np.random.default_rng(cfg.seed * 1000))
    rates = np.stack([oracle.discretize_gamma(s, cfg.R) for s in st["shape"]])
    ref = oracle.lnl_batch(codes, st["parent"], st["branch"], st["base"], st["num_classes"],
                           st["logits"], st["assign"], st["pinv"], rates,
                           nthreads=oracle.max_threads())
    return cfg, codes, st, ref


@pytest.mark.parametrize("precision", [smccat.PREC_FP64, smccat.PREC_FP32], ids=["fp64", "fp32"])
def test_config_shape_matches_oracle(case, precision):
    cfg, codes, st, ref = case
    eng = smccat.Engine(codes, cfg.R, PARTICLES, max_classes=st["logits"].shape[1], lg=cfg.lg,
                        invar=cfg.invar, cat=cfg.cat, precision=precision)
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"], st["logits"],
                      st["assign"], st["pinv"], st["shape"])
    eng.refresh(full=True)
    got = eng.lnl()
    eng.close()
    assert np.all(np.isfinite(ref))
    if precision == smccat.PREC_FP64:
        np.testing.assert_allclose(got, ref, rtol=1e-9, atol=0)
    else:
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-3)

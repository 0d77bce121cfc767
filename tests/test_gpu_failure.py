"""Failure detection on the device, exercised without faulting it.

* Bounded waits: a test knob (``smccat_set_wait_limit``) makes every pruning
  kernel's wait for its staged transition matrices (and, in the tensor-core
  kernel, its products) give up at once. The refresh must come back with
  SMCCAT_ETIMEOUT -- the kernels drain the copies they still have in flight
  and return -- and, with the default limit restored, the next refresh must
  match the oracle again. Nothing waits on a flag that is never set: the
  copies really complete; only the poll budget is zero. The learned move's
  tensor-core product waits go through the same knob.
* Non-finite state: a NaN in one particle's exchangeabilities, made on the
  host before upload, must surface as SMCCAT_ENUMERIC (the reference aborts on
  a NaN ESS instead, main.cpp:158-174), with that particle's log-likelihood NaN
  and every other particle still exact.
"""
import numpy as np
import pytest

import oracle
import smccat
from smccat import workload

pytestmark = pytest.mark.gpu

CFG = workload.WorkloadConfig("fail_cat_i", T=9, S=300, R=4, particles=6, iterations=1, lg=False,
                              invar=True, cat=True, pinv=0.1, k_range=(1, 4), seed=41)


def _setup(precision=smccat.PREC_FP64):
    rng = np.random.default_rng(CFG.seed)
    codes, _ = workload.simulate_alignment(CFG, rng)
    st = workload.make_particles(CFG, CFG.particles, rng)
    eng = smccat.Engine(codes, CFG.R, CFG.particles, max_classes=st["logits"].shape[1],
                        invar=True, cat=True, precision=precision)
    return eng, codes, st


def _load(eng, st):
    eng.set_particles(0, st["parent"], st["branch"], st["base"], st["num_classes"], st["logits"],
                      st["assign"], st["pinv"], st["shape"])


def _oracle(codes, st):
    rates = np.stack([oracle.discretize_gamma(s, CFG.R) for s in st["shape"]])
    return oracle.lnl_batch(codes, st["parent"], st["branch"], st["base"], st["num_classes"],
                            st["logits"], st["assign"], st["pinv"], rates)


# Every pruning-kernel variant at four rate categories (the engine has 13 FP64
# and 14 FP32 ones: SIMT, persistent, FP64 tensor-path and tcgen05 kernels);
# indices past a context's count are skipped.
@pytest.mark.parametrize("precision", [smccat.PREC_FP64, smccat.PREC_FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("variant", range(14))
def test_wait_timeout_reports_and_recovers(precision, variant):
    eng, codes, st = _setup(precision)
    if variant >= eng.kernel_variants()[0]:
        eng.close()
        pytest.skip("no such variant")
    ref = _oracle(codes, st)
    _load(eng, st)
    eng.set_kernel_variant(variant)
    eng.set_wait_limit(0)
    with pytest.raises(smccat.SmccatError) as err:
        eng.refresh(full=True)
    assert err.value.code == smccat.ETIMEOUT
    assert np.isnan(eng.lnl()).any()
    eng.set_wait_limit(-1)
    eng.refresh(full=True)
    got = eng.lnl()
    if precision == smccat.PREC_FP64:
        np.testing.assert_allclose(got, ref, rtol=1e-9, atol=0)
    else:
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-3)
    eng.close()


def test_nan_state_reports_enumeric():
    eng, codes, st = _setup()
    bad = {k: v.copy() for k, v in st.items()}
    bad["base"][2, 17] = np.nan
    _load(eng, bad)
    with pytest.raises(smccat.SmccatError) as err:
        eng.refresh(full=True)
    assert err.value.code == smccat.ENUMERIC
    got = eng.lnl()
    assert np.isnan(got[2])
    ok = np.arange(CFG.particles) != 2
    np.testing.assert_allclose(got[ok], _oracle(codes, st)[ok], rtol=1e-9, atol=0)
    # The state is usable again once the particle is repaired.
    _load(eng, st)
    eng.refresh(full=True)
    np.testing.assert_allclose(eng.lnl(), _oracle(codes, st), rtol=1e-9, atol=0)
    eng.close()


def test_learned_move_wait_timeout_reports_and_recovers():
    """The learned move's tcgen05 products are waited on with the same bounded
    polls: with a zero budget the move stops at its first product, drains it,
    releases its tensor memory and reports SMCCAT_ETIMEOUT with the particles'
    assignments untouched; with the default budget the next move runs and the
    likelihoods stay exact."""
    eng, codes, st = _setup()
    _load(eng, st)
    eng.refresh(full=True)
    eng.learned_params(set_to=(np.random.default_rng(2).normal(size=smccat.MLP_PARAMS) * 0.1)
                       .astype(np.float32))
    before = eng.get_particles()["assign"].copy()
    eng.set_wait_limit(0)
    with pytest.raises(smccat.SmccatError) as err:
        eng.learned_move(updates=20, temperature=1.0, seed=3)
    assert err.value.code == smccat.ETIMEOUT
    np.testing.assert_array_equal(eng.get_particles()["assign"], before)
    eng.set_wait_limit(-1)
    eng.refresh(full=True)
    eng.learned_move(updates=50, temperature=1.0, seed=4)
    fin = eng.get_particles()
    rates = np.stack([oracle.discretize_gamma(s, CFG.R) for s in fin["shape"]])
    ref = oracle.lnl_batch(codes, fin["parent"], fin["branch"], fin["base"], fin["num_classes"],
                           fin["logits"], fin["assign"], fin["pinv"], rates)
    np.testing.assert_allclose(eng.lnl(), ref, rtol=1e-9, atol=0)
    eng.close()

"""CPU-side checks of the C-ABI library: it loads, exports every symbol the
header declares, and its host-only numerics match the golden fixtures."""
import json
import os
import re

import numpy as np
import pytest

import oracle
import smccat
from smccat import workload

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def declared_symbols():
    txt = open(smccat.HEADER_PATH).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(smccat_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    names = declared_symbols()
    assert len(names) >= 20
    L = smccat.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version():
    assert smccat.version().startswith("smccat-b200")


@pytest.mark.parametrize("case", GOLD["discretize_gamma"], ids=lambda c: f"shape{c['shape']}-R{c['R']}")
def test_discretize_gamma_matches_golden(case):
    r = smccat.discretize_gamma(case["shape"], case["R"])
    np.testing.assert_allclose(r, case["rates"], rtol=1e-11, atol=0)


def test_discretize_gamma_agrees_with_oracle():
    for shape in np.geomspace(0.02, 200.0, 37):
        for R in (2, 3, 4, 6, 8):
            np.testing.assert_allclose(smccat.discretize_gamma(shape, R),
                                       oracle.discretize_gamma(shape, R), rtol=1e-11)


def test_lg_table_matches_reference_source():
    np.testing.assert_array_equal(smccat.lg_exchangeabilities(), np.array(GOLD["lg_base"]))


def test_bad_arguments_raise():
    with pytest.raises(smccat.SmccatError):
        smccat.discretize_gamma(-1.0, 4)


def test_create_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    codes = np.zeros((4, 10), np.uint8)
    with pytest.raises(smccat.SmccatError) as e:
        smccat.Engine(codes, num_rates=4, max_particles=2)
    assert e.value.code == smccat.ENODEV


def test_workload_trees_are_valid():
    rng = np.random.default_rng(0)
    for T in (3, 4, 16, 48):
        parent, branch = workload.random_tree(rng, T)
        post = oracle.postorder(parent)
        assert sorted(post) == list(range(2 * T - 1))
        assert branch[T] == 0.0 and parent[T] == -1


def test_simulated_alignment_shapes():
    cfg = workload.CONFIGS[1]
    codes, truth = workload.simulate_alignment(cfg)
    assert codes.shape == (cfg.T, cfg.S)
    assert codes.max() <= 20
    frac_gap = (codes == 20).mean()
    assert 0.005 < frac_gap < 0.05
    parts = workload.make_particles(cfg, 3, np.random.default_rng(1))
    assert parts["parent"].shape == (3, 2 * cfg.T - 1)


def test_transition_batch_matches_oracle():
    rng = np.random.default_rng(2)
    base = rng.normal(size=190)
    lg = np.zeros(20)
    lg[:19] = rng.normal(size=19)
    pi = oracle.softmax20(lg)
    P = workload.transition_batch(base, pi, [0.0, 0.1, 1.0])
    for i, t in enumerate([0.0, 0.1, 1.0]):
        np.testing.assert_allclose(P[i], oracle.transition(base, pi, t), atol=1e-12)

"""Precision tiers and the tier network on the GPU: the network's kernels
against the numpy oracle (forward, gradient, Adam training), reproducibility,
every tier's refined factor, and what the trained network gains over the
fixed policies on the held-out part of the labelled corpus."""
import ctypes as C

import numpy as np
import pytest

from oracle import tier_mlp as O
from oracle.oracle import backward_error
from rslab_b200 import LdltSymbolic, MixedLdltSolver, SolverSettings, matgen
from rslab_b200 import _native as N
from rslab_b200.tiers import (DATA, NFEAT, TierModel, policy_costs, run_tier, solve_learned, split, tier_features,
                              tier_settings)

pytestmark = pytest.mark.gpu

F = C.POINTER(C.c_float)


def _fp(a):
    return a.ctypes.data_as(F)


def _data(m, seed=21):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(m, NFEAT)).astype(np.float32)
    y = rng.integers(0, 3, size=m).astype(np.int32)
    w = rng.uniform(0.1, 2.0, size=m).astype(np.float32)
    return x, y, w


def _grad(p, x, y, w):
    g = np.zeros(N.TIER_MLP_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    rc = N.lib.rslab_tier_mlp_grad(_fp(p), _fp(x), y.ctypes.data_as(C.POINTER(C.c_int32)),
                                   None if w is None else _fp(w), len(y), _fp(g), _fp(loss), 0)
    assert rc == 0, N.last_error()
    return float(loss[0]), g


def test_forward_matches_oracle():
    p = TierModel.init(9).params
    x, _, _ = _data(333)
    probs = np.zeros((333, 3), np.float32)
    assert N.lib.rslab_tier_mlp_forward(_fp(p), _fp(x), 333, _fp(probs), 0) == 0, N.last_error()
    ref, _ = O.forward(p, x)
    assert np.abs(probs - ref).max() <= 2e-6


@pytest.mark.parametrize("weighted", [False, True])
def test_gradient_matches_oracle(weighted):
    p = TierModel.init(9).params
    x, y, w = _data(517)
    w = w if weighted else None
    loss, g = _grad(p, x, y, w)
    lref, gref = O.loss_and_grad(p, x, y, w)
    assert abs(loss - lref) <= 1e-5 * abs(lref)
    # FP32 accumulation against the float64 oracle: normwise and per entry
    assert np.linalg.norm(g - gref) <= 1e-5 * np.linalg.norm(gref)
    assert np.abs(g - gref).max() <= 1e-5 * np.abs(gref).max()


def test_gradient_is_reproducible():
    p = TierModel.init(4).params
    x, y, w = _data(300)
    assert np.array_equal(_grad(p, x, y, w)[1], _grad(p, x, y, w)[1])


def test_training_matches_oracle_adam():
    p0 = TierModel.init(2).params
    x, y, w = _data(400, 5)
    p = p0.copy()
    curve = np.zeros(60, np.float32)
    rc = N.lib.rslab_tier_mlp_train(_fp(p), _fp(x), y.ctypes.data_as(C.POINTER(C.c_int32)), _fp(w), 400, 60,
                                    C.c_float(3e-3), _fp(curve), 0)
    assert rc == 0, N.last_error()
    pref, cref = O.train(p0, x, y, w, epochs=60, lr=3e-3)
    assert np.abs(curve - cref).max() <= 1e-4 * cref[0]
    assert curve[-1] < curve[0]
    assert np.linalg.norm(p - pref) <= 1e-3 * np.linalg.norm(pref)


def test_bad_labels_are_rejected():
    p = TierModel.init(1).params
    x, y, w = _data(10)
    y[3] = 7
    g = np.zeros(N.TIER_MLP_PARAMS, np.float32)
    loss = np.zeros(1, np.float32)
    rc = N.lib.rslab_tier_mlp_grad(_fp(p), _fp(x), y.ctypes.data_as(C.POINTER(C.c_int32)), _fp(w), 10, _fp(g),
                                   _fp(loss), 0)
    assert rc == 2  # RSLAB_INVALID_INPUT
    assert "labels" in N.last_error()


@pytest.mark.parametrize("tier", [0, 1, 2])
def test_every_tier_certifies(tier):
    a = matgen.c2_matrix(12)
    b = matgen.uniform_rhs(a.n, 3, 1, complex_=True)
    sym = LdltSymbolic.analyze_with(a, tier_settings())
    t, cert, be, x = run_tier(a, b, tier, sym)
    assert cert and be <= 1e-14 and t > 0
    assert backward_error(a, x, b) <= 1e-14


def test_fp32_tier_is_the_fma_mixed_factor():
    a = matgen.c3_matrix(14)
    b = matgen.uniform_rhs(a.n, 2, 3)
    st = SolverSettings()
    st.schur_engine = "fma"
    x1, i1 = MixedLdltSolver.factor_with(a, st).solve_to(a, b, 1e-14)
    x2, i2 = MixedLdltSolver.factor_tier(a, N.TIER_FP32, SolverSettings()).solve_to(a, b, 1e-14)
    assert np.array_equal(x1, x2) and i1.ir_iters == i2.ir_iters


def test_fp64_tier_needs_at_most_one_correction():
    a = matgen.c2_matrix(12)
    b = matgen.uniform_rhs(a.n, 2, 1, complex_=True)
    x, info = MixedLdltSolver.factor_tier(a, N.TIER_FP64).solve_to(a, b, 1e-14)
    assert info.certified and info.ir_iters <= 1 and info.gmres_iters == 0


def _corpus():
    path = DATA / "tier_corpus.npz"
    if not path.exists():
        pytest.skip("no labelled corpus in the package")
    z = np.load(path)
    return {k: z[k] for k in z.files}


def test_trained_network_beats_fixed_policies_on_held_out_corpus():
    c = _corpus()
    model = TierModel.load()
    _, te = split(len(c["labels"]))
    pred = model.predict(c["features"][te])
    r = policy_costs(pred, c["times"][te], c["certified"][te])
    assert r["network"] < r["always_fp64"]
    assert r["network"] < r["always_tf32x3"]
    assert r["network"] < r["always_fp32"]


def test_solve_learned_certifies_corpus_samples():
    model = TierModel.load() if (DATA / "tier_mlp.npz").exists() else TierModel.init(1)
    for i, (fam, a) in enumerate(matgen.c5_corpus(12, 5)):
        if a.n > 20000:
            continue
        b = matgen.uniform_rhs(a.n, 2, 9 + i, complex_=np.iscomplexobj(a.values))
        x, info, tier, fell_back = solve_learned(a, b, model)
        assert info.certified and backward_error(a, x, b) <= 1e-14, (fam, tier, fell_back)


def test_features_feed_the_network():
    a = matgen.c5_heldout(8, 6)
    sym = LdltSymbolic.analyze_with(a, tier_settings())
    p = TierModel.init(1).predict_proba(tier_features(a, sym))
    assert p.shape == (1, 3) and abs(float(p.sum()) - 1.0) < 1e-5

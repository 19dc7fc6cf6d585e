"""Precision-tier network and corpus, host side (no GPU): the oracle's
gradient against finite differences, the corpus and held-out generators,
features, labels and policy costs."""
import math

import numpy as np
import pytest

from oracle import tier_mlp as O
from rslab_b200 import LdltSymbolic, matgen
from rslab_b200 import _native as N
from rslab_b200.solver import CscMatrix
from rslab_b200.tiers import (NFEAT, TIERS, TierModel, cheapest_certified, effective_cost, policy_costs,
                              sample_weight, split, tier_features, tier_settings)


def _data(m=40, seed=11):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(m, NFEAT))
    y = rng.integers(0, 3, size=m)
    w = rng.uniform(0.1, 2.0, size=m)
    return x, y, w


def test_oracle_parameter_count_matches_abi():
    assert O.NPARAM == N.TIER_MLP_PARAMS == 4931


def test_oracle_gradient_matches_finite_differences():
    p = TierModel.init(3).params.astype(np.float64)
    x, y, w = _data()
    _, g = O.loss_and_grad(p, x, y, w)
    rng = np.random.default_rng(0)
    for i in rng.choice(len(p), 40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (O.loss_and_grad(pp, x, y, w)[0] - O.loss_and_grad(pm, x, y, w)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_oracle_training_reduces_loss():
    p = TierModel.init(3).params
    x, y, w = _data(200)
    _, curve = O.train(p, x, y, w, epochs=200, lr=1e-2)
    assert curve[-1] < 0.5 * curve[0]


def test_init_is_seeded_he_uniform():
    a, b = TierModel.init(5), TierModel.init(5)
    assert np.array_equal(a.params, b.params)
    P = O.unpack(a.params)
    assert np.abs(P["W1"]).max() <= math.sqrt(6 / 8) and np.abs(P["W2"]).max() <= math.sqrt(6 / 64)
    assert not P["b1"].any() and not P["b3"].any()


def test_stencil27_lambda_max_formula():
    side = 4
    n = side ** 3
    diag, rows, cols, w = matgen.stencil27(side, matgen.Rng(1))
    a = np.zeros((n, n))
    a[rows, cols] = w
    a[cols, rows] = w
    a[np.arange(n), np.arange(n)] = 26.0
    lam = np.linalg.eigvalsh(a).max()
    assert abs(lam - matgen.stencil27_lambda_max(side)) < 1e-10


def test_corpus_is_seeded_and_covers_every_family():
    a = list(matgen.c5_corpus(30, 5))
    b = list(matgen.c5_corpus(30, 5))
    assert [f for f, _ in a] == [f for f, _ in b]
    for (_, x), (_, y) in zip(a, b):
        assert np.array_equal(x.values, y.values) and np.array_equal(x.row_idx, y.row_idx)
    fams = {f for f, _ in matgen.c5_corpus(200, 5)}
    assert fams == set(matgen.C5_FAMILIES)
    for f, m in a:
        assert np.iscomplexobj(m.values) == f.startswith("helmholtz")


def test_random_sparse_symmetric_row_counts():
    a = matgen.random_sparse_symmetric(300, matgen.Rng(2), 0.5)
    assert a.n == 300
    full = np.zeros((300, 300))
    cp = np.asarray(a.col_ptr)
    for j in range(300):
        for k in range(cp[j], cp[j + 1]):
            full[a.row_idx[k], j] = a.values[k]
    assert np.all(np.diag(full) != 0)
    offd = (full != 0).sum(axis=0) - 1
    assert offd.mean() > 5  # lower triangle holds about half of each row's 8-30 partners


def test_heldout_matrix_definition():
    a = matgen.c5_heldout(6, 6)
    diag, rows, cols, w = matgen.stencil27(6, matgen.Rng(6))
    k2 = 0.15 * matgen.stencil27_lambda_max(6)
    cp = np.asarray(a.col_ptr)
    d = np.asarray(a.values)[cp[:-1]]
    assert np.allclose(d, diag - k2 * (1 + 0.02j), rtol=0, atol=1e-14)


def test_features_of_a_diagonal_matrix():
    n = 50
    a = CscMatrix.from_triplets(n, np.arange(n), np.arange(n), np.full(n, 2.0))
    sym = LdltSymbolic.analyze_with(a, tier_settings())
    f = tier_features(a, sym)
    assert f.shape == (NFEAT,)
    assert abs(f[0] - math.log10(n)) < 1e-12
    assert f[3] == 0.0 and f[4] == 0.0 and f[5] == 0.0 and f[6] == 0.0
    assert abs(f[7] - 0.0) < 1e-12  # ||A||_inf / min |a_ii| = 1


def test_features_of_an_indefinite_complex_matrix():
    a = matgen.c5_heldout(5, 6)
    sym = LdltSymbolic.analyze_with(a, tier_settings())
    f = tier_features(a, sym)
    # |26 + U - k2 (1 + 0.02i)| < 26: exactly the interior rows (26 neighbours) are not dominant
    assert f[3] == 1.0 and f[6] == 0.0 and f[5] == pytest.approx(3 ** 3 / 5 ** 3)


def test_labels_costs_and_weights():
    t = np.array([1.0, 0.5, 0.2])
    assert cheapest_certified(t, np.array([True, True, True])) == 2
    assert cheapest_certified(t, np.array([True, True, False])) == 1
    assert cheapest_certified(t, np.array([False, False, False])) == 0
    c = np.array([True, True, False])
    assert effective_cost(t, c, 2) == pytest.approx(1.2)
    assert effective_cost(t, c, 0) == 1.0
    assert sample_weight(t, c) == pytest.approx(1.2 - 0.5 + 1e-4)
    times = np.array([[1.0, 0.5, 0.2], [0.1, 0.3, 0.4]])
    cert = np.array([[True, True, True], [True, True, True]])
    r = policy_costs(np.array([2, 0]), times, cert)
    assert r["network"] == pytest.approx(0.3) and r["always_fp64"] == pytest.approx(1.1)
    assert r["best_possible"] == pytest.approx(0.3)


def test_split_is_deterministic_and_disjoint():
    tr, te = split(100)
    assert len(te) == 20 and not set(tr) & set(te)
    assert len(TIERS) == 3


def _corpus():
    from rslab_b200.tiers import DATA
    z = np.load(DATA / "tier_corpus.npz")
    return {k: z[k] for k in z.files}


def test_committed_corpus_is_consistent():
    c = _corpus()
    m = len(c["labels"])
    assert m >= 1000 and c["features"].shape == (m, NFEAT) and c["times"].shape == (m, 3)
    assert all(cheapest_certified(c["times"][i], c["certified"][i]) == c["labels"][i] for i in range(m))
    assert set(np.unique(c["family"])) == set(range(len(matgen.C5_FAMILIES)))
    # the features recorded on the GPU box are the host features of the same seeded matrices
    for i, (_, a) in enumerate(matgen.c5_corpus(5, int(c["seed"]))):
        f = tier_features(a, LdltSymbolic.analyze_with(a, tier_settings()))
        assert np.allclose(f, c["features"][i], rtol=1e-12, atol=1e-12)


def test_training_recipe_beats_fixed_policies_with_the_oracle_trainer():
    """The recipe (regret weights, 200 Adam epochs) run by the oracle: the
    network's choices cost less on the held-out matrices than any fixed tier."""
    c = _corpus()
    m = len(c["labels"])
    tr, te = split(m)
    w = np.array([sample_weight(c["times"][i], c["certified"][i]) for i in range(m)])
    f = c["features"]
    mu, sd = f[tr].mean(0), np.maximum(f[tr].std(0), 1e-6)
    p, curve = O.train(TierModel.init(7).params, (f[tr] - mu) / sd, c["labels"][tr], w[tr], 200, 3e-3)
    pred = O.forward(p, (f[te] - mu) / sd)[0].argmax(1)
    r = policy_costs(pred, c["times"][te], c["certified"][te])
    assert curve[-1] < curve[0]
    assert r["network"] < min(r["always_fp64"], r["always_fp32"], r["always_tf32x3"])

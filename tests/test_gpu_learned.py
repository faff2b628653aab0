"""Learned solver settings: the GPU MLP kernels against the FP64 numpy
oracle (forward logits, loss and every gradient), training that lowers the
loss, and, for both matrix families (banded: partitions, coupled or
decoupled, LU_UL or LU_only; sparse with reordering: partitions, coupled or
decoupled, drop-off fraction), the chooser's time-to-solution against the
default setting on held-out matrices of a measured settings sweep."""
import numpy as np
import pytest

from oracle import mlp_oracle
from saplibrary_b200 import learned

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SHAPE = (learned.NUM_FEATURES, 64, 64, len(learned.SETTINGS))


def test_forward_and_gradients_match_oracle():
    net = learned.SettingsNet(seed=3)
    rng = np.random.default_rng(0)
    X = rng.standard_normal((97, learned.NUM_FEATURES)).astype(np.float32)
    y = rng.integers(0, len(learned.SETTINGS), 97).astype(np.int32)
    p = net.params()
    z_gpu = net.logits(X, normalise=False)
    _, _, z = mlp_oracle.forward(p, SHAPE, X)
    assert np.allclose(z_gpu, z, rtol=1e-4, atol=1e-5)
    g_gpu, loss_gpu = net.gradients(X, y)
    loss, g = mlp_oracle.loss_and_grad(p, SHAPE, X, y)
    assert abs(loss_gpu - loss) <= 1e-5 * max(1.0, abs(loss))
    assert np.linalg.norm(g_gpu - g) <= 1e-4 * np.linalg.norm(g)
    # the oracle's gradient itself against central differences on a few weights
    for k in (0, 100, 1500, len(p) - 3):
        e = np.zeros_like(p, dtype=np.float64)
        e[k] = 1e-5
        lp, _ = mlp_oracle.loss_and_grad(p + e, SHAPE, X, y)
        lm, _ = mlp_oracle.loss_and_grad(p - e, SHAPE, X, y)
        assert abs((lp - lm) / 2e-5 - g[k]) <= 1e-5 + 1e-4 * abs(g[k])


def test_training_lowers_loss_and_is_deterministic():
    rng = np.random.default_rng(1)
    X = rng.standard_normal((200, learned.NUM_FEATURES)).astype(np.float32)
    y = (X[:, 0] > 0).astype(np.int32) + 2 * (X[:, 1] > 0).astype(np.int32)
    a, b = learned.SettingsNet(seed=5), learned.SettingsNet(seed=5)
    l0 = a.gradients(X, y, normalise=False)[1]
    la = a.train(X, y, epochs=300)
    lb = b.train(X, y, epochs=300)
    assert la < 0.5 * l0
    assert la == lb and np.array_equal(a.params(), b.params())
    assert (a.choose(X, min_confidence=0.0) == y).mean() > 0.9


def test_chooser_against_default_on_held_out_sweep():
    X, T = learned.sweep(48, seed=11, n_range=(20000, 80000), k_range=(8, 96))
    train, held = slice(0, 36), slice(36, 48)
    net = learned.SettingsNet(seed=9)
    net.train(X[train], learned.labels_from_times(T[train]), epochs=500)
    picks = net.choose(X[held])
    g = learned.gain(T[held], picks)
    print("held-out", g)
    print("held-out times [matrix, setting] (s):\n", np.array2string(T[held], precision=4))
    print("picks", picks, "confidence", np.round(net.probabilities(X[held]).max(axis=1), 2))
    assert g["failed_chosen"] <= g["failed_default"]
    # the trained chooser is at least as fast as the default heuristic in
    # total over the held-out matrices
    assert g["total_chosen_s"] <= g["total_default_s"]


def test_sparse_chooser_against_default_on_held_out_sweep():
    fam = learned.SPARSE
    X, T = learned.sweep(fam, 40, seed=13, m_range=(60, 140))
    train, held = slice(0, 30), slice(30, 40)
    net = learned.SettingsNet(fam, seed=9)
    net.train(X[train], learned.labels_from_times(T[train]), epochs=500)
    picks = net.choose(X[held])
    g = learned.gain(fam, T[held], picks)
    print("sparse held-out", g)
    print("picks", [fam.settings[p] for p in picks])
    assert g["failed_chosen"] <= g["failed_default"]
    assert g["total_chosen_s"] <= g["total_default_s"]

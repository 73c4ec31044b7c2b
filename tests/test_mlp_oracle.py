"""CPU checks of the learned pruner's host logic and of its numpy oracle:
the oracle's analytic gradient against central differences, the parameter
layout shared with the C ABI, and the label/threshold helpers."""
import numpy as np

from oracle import mlp_oracle as mo


def test_param_count_matches_abi():
    from tsr_b200 import core
    assert mo.NPARAM == core.MLP_PARAMS == 4994


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    theta = mo.init(1) * 0.5
    x = rng.normal(size=(12, mo.NF))
    y = (rng.uniform(size=(12, mo.NO)) < 0.3).astype(np.float64)
    _, g = mo.loss_and_grad(theta, x, y, pos_weight=(3.0, 2.0))
    idx = rng.choice(mo.NPARAM, 60, replace=False)
    h = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        num = (mo.loss_and_grad(tp, x, y, (3.0, 2.0))[0] - mo.loss_and_grad(tm, x, y, (3.0, 2.0))[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-5 * max(1.0, abs(num)), (i, num, g[i])


def test_labels_mark_both_sides_of_a_sign_change():
    from tsr_b200.pruner import labels

    class L:
        neighbors_offsets = np.array([0, 1, 2, 2, 2])
        neighbors = np.array([1, 2])
    occ = np.array([-1e-6, -1e-6, 0.3, -1e-6])
    y = labels(occ, L)
    assert y[:, 0].tolist() == [0, 0, 1, 0]
    assert y[:, 1].tolist() == [0, 1, 1, 0]


def test_thresholds_bound_the_missed_fractions():
    from tsr_b200.pruner import choose_thresholds
    rng = np.random.default_rng(0)
    y = (rng.uniform(size=(20000, 2)) < 0.3).astype(np.float32)
    z = rng.normal(size=(20000, 2)) + 4.0 * (y - 0.5)
    ts, tb = choose_thresholds(z, y, miss=0.01)
    p = 1 / (1 + np.exp(-z))
    band = y[:, 1] > 0.5
    assert (band & (p[:, 1] < tb)).sum() <= 0.01 * band.sum() + 1
    rest = ~band
    wrong = ((p[rest, 0] >= 1 - ts) & (y[rest, 0] < 0.5)) | ((p[rest, 0] <= ts) & (y[rest, 0] > 0.5))
    assert wrong.mean() <= 0.01
    assert 0 < ts < 0.5 and 0 < tb < 1


def test_he_init_layout():
    from tsr_b200.pruner import he_init
    th = he_init(0)
    assert th.shape == (mo.NPARAM,) and th.dtype == np.float32
    p = mo.unpack(th)
    assert np.all(p["b1"] == 0) and np.all(p["b3"] == 0)


def test_committed_pruner_weights_load():
    import json
    from tsr_b200 import core
    p = core.Pruner.load()
    assert p.weights.shape == (core.MLP_PARAMS,) and np.isfinite(p.weights).all()
    assert 0 < p.sign_threshold < 0.5 and 0 < p.band_threshold < 1 and p.dilation >= 0
    z = np.load(core.Path(core.__file__).resolve().parent / "pruner_weights.npz")
    meta = json.loads(str(z["meta"]))
    assert meta["validation_band_missed_fraction"] <= 2e-3

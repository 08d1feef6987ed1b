"""The learned far-field correction: MLP kernels against the NumPy oracle,
GPU training, and what the trained network gains over the monopole."""
import numpy as np
import pytest

from conftest import rel_err


def _data(seed, n=4096):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 12)).astype(np.float32)
    X[:, 2] = rng.uniform(0.5, 1.0, n)
    return X


def test_oracle_backward_matches_finite_differences():
    from oracle import mlp_oracle as mo

    p = mo.init(3)
    X = _data(1, 64)
    T = np.random.default_rng(2).normal(size=(64, 2))
    _, g = mo.loss_grad(p, X, T, exact=True)
    rng = np.random.default_rng(5)
    for k in rng.choice(mo.YS, 40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (mo.loss_grad(pp, X, T, exact=True)[0] - mo.loss_grad(pm, X, T, exact=True)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


@pytest.mark.gpu
def test_forward_matches_oracle(nbp):
    from oracle import mlp_oracle as mo

    p = mo.init(7)
    # 2^17 + 5 rows: 1025 tiles of 128 for the tcgen05 kernel, the last one ragged
    X = _data(8, (1 << 17) + 5)
    y = nbp.mlp_forward(p.astype(np.float32), X)
    y_o, _ = mo.forward(p.astype(np.float32), X)
    assert np.abs(y - y_o).max() < 2e-2 * max(1.0, np.abs(y_o).max())
    assert np.corrcoef(y.ravel(), y_o.ravel())[0, 1] > 0.9999


@pytest.mark.gpu
def test_forward_bulk_many_tiles_per_cta(nbp):
    """2^21 + 77 rows: 16,385 tiles of 128, about 22 per CTA, so each CTA's
    next feature tile is copied in while the current one runs; the last tile
    is ragged."""
    from oracle import mlp_oracle as mo

    p = mo.init(7).astype(np.float32)
    X = _data(9, (1 << 21) + 77)
    y = nbp.mlp_forward(p, X)
    assert y.shape == (X.shape[0], 2) and np.isfinite(y).all()
    rows = np.concatenate([np.random.default_rng(3).choice(X.shape[0] - 77, 65536, replace=False),
                           np.arange(X.shape[0] - 77, X.shape[0])])
    y_o, _ = mo.forward(p, X[rows])
    assert np.abs(y[rows] - y_o).max() < 2e-2 * max(1.0, np.abs(y_o).max())
    # a row's output depends on its own features only
    assert np.array_equal(nbp.mlp_forward(p, X[:1000]), y[:1000])


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 5, 127, 128, 129, 255])
def test_forward_ragged_tiles(nbp, n):
    """Tiles of 128 rows with empty rows: each row's output depends on its
    own features only, so any n gives the rows of a larger batch."""
    from oracle import mlp_oracle as mo

    p = mo.init(3).astype(np.float32)
    X = _data(4, 256)
    y_all = nbp.mlp_forward(p, X)
    y = nbp.mlp_forward(p, X[:n])
    assert y.shape == (n, 2) and np.isfinite(y).all()
    assert np.array_equal(y, y_all[:n])
    y_o, _ = mo.forward(p, X[:n])
    assert np.abs(y - y_o).max() < 2e-2 * max(1.0, np.abs(y_o).max())


@pytest.mark.gpu
def test_gradients_match_oracle(nbp):
    from oracle import mlp_oracle as mo

    p = mo.init(11).astype(np.float32)
    X = _data(12, 3000)
    T = np.random.default_rng(13).normal(size=(3000, 2)).astype(np.float32)
    loss, g = nbp.mlp_loss_grad(p, X, T)
    loss_o, g_o = mo.loss_grad(p, X, T)
    assert loss == pytest.approx(loss_o, rel=1e-2)
    g, g_o = g[:mo.YS].astype(np.float64), g_o[:mo.YS]
    assert np.linalg.norm(g - g_o) < 2e-2 * np.linalg.norm(g_o)
    assert g @ g_o / (np.linalg.norm(g) * np.linalg.norm(g_o)) > 0.999
    for name, a, b in (("W1", mo.W1, mo.B1), ("W2", mo.W2, mo.B2), ("W3", mo.W3, mo.B3),
                       ("b1", mo.B1, mo.W2), ("b2", mo.B2, mo.W3), ("b3", mo.B3, mo.YS)):
        assert np.linalg.norm(g[a:b] - g_o[a:b]) < 3e-2 * np.linalg.norm(g_o[a:b]), name


@pytest.mark.gpu
def test_training_fits_a_smooth_target(nbp):
    X = _data(21, 1 << 15)
    Y = np.stack([np.sin(X[:, 0]) * X[:, 2], X[:, 1] * X[:, 3] * 0.5], axis=1).astype(np.float32)
    p, losses = nbp.mlp_train(X, Y, epochs=30, batch=1024, lr=3e-3, seed=1)
    assert (np.diff(losses[:5]) < 0).all()
    assert losses[-1] < 0.02 * losses[0]
    pred = nbp.mlp_forward(p, X) * p[-1]
    assert np.sqrt(((pred - Y) ** 2).mean()) < 0.15 * np.sqrt((Y ** 2).mean())


@pytest.mark.gpu
def test_learned_correction_beats_the_monopole_at_theta_one(nbp):
    eps2 = 1e-4
    # training data from snapshots of other seeds
    Xs, Ys = [], []
    for seed in (1, 2, 3):
        m, p, v = nbp.universes.colliding_discs(65536, seed)
        cfg = nbp.SimConfig(theta=1.0, epsilon_squared=eps2, mode=nbp.NB_MODE_SPLIT, learned=True)
        with nbp.NbContext(cfg, m, p, v) as ctx:
            X, Y = ctx.mlp_samples(4096, seed=seed)
        Xs.append(X)
        Ys.append(Y)
    X, Y = np.concatenate(Xs), np.concatenate(Ys)
    assert X.shape[0] > 100000 and np.isfinite(X).all() and np.isfinite(Y).all()
    assert (X[:, 2] > 0).all() and ((X[:, 0] ** 2 + X[:, 1] ** 2 - 1) ** 2 < 1e-6).all()
    params, losses = nbp.mlp_train(X, Y, epochs=30, batch=1024, lr=2e-3, seed=0)
    assert losses[-1] < 0.5 * losses[0]
    # evaluation on an unseen seed
    m, p, v = nbp.universes.colliding_discs(65536, 9)
    tgt = np.arange(0, 65536, 4)
    exact = nbp.allpairs_accelerations(m, p, tgt, eps2)
    cfg = nbp.SimConfig(theta=1.0, epsilon_squared=eps2, mode=nbp.NB_MODE_SPLIT)
    with nbp.NbContext(cfg, m, p, v) as ctx:
        a_mono = ctx.accelerations()
    cfg.learned = True
    with nbp.NbContext(cfg, m, p, v) as ctx:
        ctx.set_mlp_weights(params)
        a_learned = ctx.accelerations()
    e_mono = np.percentile(rel_err(a_mono[tgt], exact), [50, 99])
    e_learned = np.percentile(rel_err(a_learned[tgt], exact), [50, 99])
    # the correction is evaluated once per 64-body group at its centre, so it
    # removes only part of the monopole error.  Over four training seeds with
    # this data the learned/monopole ratio measured 0.68-0.81 at p50 but
    # 0.86-1.00 at p99 (0.86-1.09 with half the samples and 20 epochs): the
    # median gain is reliable, the tail's is not, so the tail is only held to
    # not getting worse beyond that scatter
    assert e_learned[0] < 0.9 * e_mono[0], (e_learned, e_mono)
    assert e_learned[1] < 1.05 * e_mono[1], (e_learned, e_mono)


@pytest.mark.gpu
def test_shipped_weights_run_with_zero_softening(nbp):
    """The committed correction on an eps^2 = 0 context: the eps^2 = 0 walk
    variant with band lists, then the correction, stays finite."""
    import json
    import pathlib

    wdir = pathlib.Path(nbp.__file__).resolve().parent / "weights"
    params = np.load(wdir / "correction_theta1.npy")
    bmax = json.loads((wdir / "correction_theta1.json").read_text())["bmax_ratio"]
    m, p, v = nbp.universes.colliding_discs(32768, 6)
    cfg = nbp.SimConfig(theta=1.0, epsilon_squared=0.0, mode=nbp.NB_MODE_SPLIT, learned=True,
                        bmax_ratio=bmax)
    with nbp.NbContext(cfg, m, p, v) as ctx:
        ctx.set_mlp_weights(params)
        a = ctx.accelerations()
        ctx.step(2)
        pos, _ = ctx.download()
    assert np.isfinite(a).all() and np.isfinite(pos).all()

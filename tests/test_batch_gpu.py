"""GPU tests of batched universes (nb_batch_create) and the SPLIT autotuner.

A batch advances many independent universes in one sort, one tree and one
traversal launch.  The tests check isolation (universes laid over the same
coordinates feel nothing of each other), agreement with one context per
universe, the edge cases of tiny and degenerate universes, and that the
autotuner leaves the bodies as it found them."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
EPS2 = 1e-4


def _concat(universes):
    m = np.concatenate([u[0] for u in universes])
    p = np.concatenate([u[1] for u in universes])
    v = np.concatenate([u[2] for u in universes])
    return m, p, v, np.array([u[0].shape[0] for u in universes], dtype=np.uint64)


def _overlapping(nbp, sizes, seed):
    """Discs centred on the same point, so a leak between universes shows."""
    out = []
    for k, n in enumerate(sizes):
        if n >= 2:
            out.append(nbp.universes.exponential_disc(int(n), seed + k))
        else:
            out.append((np.ones(1), np.full((1, 2), 0.25), np.zeros((1, 2))))
    return out


def _split_cfg(nbp, theta, leaf=0, quad=False):
    return nbp.SimConfig(theta=theta, epsilon_squared=EPS2, mode=nbp.NB_MODE_SPLIT,
                         leaf_size=leaf, quadrupole=quad)


def test_batch_theta_zero_is_allpairs_per_universe(nbp, orc):
    sizes = [1, 2, 3, 33, 1000, 4096, 70]
    unis = _overlapping(nbp, sizes, 11)
    m, p, v, counts = _concat(unis)
    with nbp.NbContext(_split_cfg(nbp, 0.0, leaf=1), m, p, v, counts=counts) as ctx:
        a = ctx.accelerations()
    off = 0
    for mu, pu, _ in unis:
        n = mu.shape[0]
        au = a[off:off + n]
        off += n
        if n == 1:
            assert np.array_equal(au, np.zeros((1, 2)))
            continue
        exact = orc.allpairs_plummer(mu, pu, eps2=EPS2)
        box = orc.bbox_squared(pu)
        center = (0.5 * (box[0] + box[1]), 0.5 * (box[2] + box[3]))
        bound = orc.allpairs_fp32_bound(mu, pu, center, eps2=EPS2)
        assert (np.linalg.norm(au - exact, axis=1) <= bound).all()


@pytest.mark.parametrize("theta,quad", [(0.5, False), (0.8, True)])
def test_batch_matches_one_context_per_universe(nbp, theta, quad):
    unis = nbp.universes.ensemble(12, 5, nmin=512, nmax=40000)
    m, p, v, counts = _concat(unis)
    with nbp.NbContext(_split_cfg(nbp, theta, quad=quad), m, p, v, counts=counts) as ctx:
        a = ctx.accelerations()
        ctx.step(2)
        pb, vb = ctx.download()
    off = 0
    for mu, pu, vu in unis:
        n = mu.shape[0]
        with nbp.NbContext(_split_cfg(nbp, theta, quad=quad), mu, pu, vu) as one:
            a1 = one.accelerations()
            one.step(2)
            p1, v1 = one.download()
        exact = nbp.allpairs_accelerations(mu, pu, np.arange(n), EPS2)
        eb, e1 = rel_err(a[off:off + n], exact), rel_err(a1, exact)
        # the same tree below the universe's root: the same accuracy
        assert np.percentile(eb, 99) <= 1.02 * np.percentile(e1, 99) + 1e-6
        assert np.percentile(eb, 50) <= 1.02 * np.percentile(e1, 50) + 1e-6
        scale = np.abs(a1).max()
        assert np.abs(a[off:off + n] - a1).max() <= 2e-2 * scale
        dv = np.abs(vb[off:off + n] - v1).max()
        assert dv <= 2 * 2e-2 * scale * 1e-4 + 1e-12
        off += n


def test_batch_degenerate_universes(nbp, orc):
    rng = np.random.default_rng(9)
    same = (np.full(40, 0.5), np.tile([[3.0, -1.0]], (40, 1)), np.zeros((40, 2)))
    pair = (np.array([1.0, 2.0]), np.array([[0.0, 0.0], [1e-9, 0.0]]), np.zeros((2, 2)))
    cloud = (rng.random(500) + 0.5, rng.random((500, 2)), np.zeros((500, 2)))
    unis = [same, pair, cloud, same]
    m, p, v, counts = _concat(unis)
    with nbp.NbContext(_split_cfg(nbp, 0.0, leaf=1), m, p, v, counts=counts) as ctx:
        a = ctx.accelerations()
        ctx.step(3)
        pb, _ = ctx.download()
    assert np.isfinite(a).all() and np.isfinite(pb).all()
    # coincident bodies pull each other with zero force (Plummer, d = 0)
    assert np.abs(a[:40]).max() == 0.0 and np.abs(a[-40:]).max() == 0.0
    off = 40
    for mu, pu, _ in unis[1:3]:
        n = mu.shape[0]
        exact = orc.allpairs_plummer(mu, pu, eps2=EPS2)
        box = orc.bbox_squared(pu)
        center = (0.5 * (box[0] + box[1]), 0.5 * (box[2] + box[3]))
        bound = orc.allpairs_fp32_bound(mu, pu, center, eps2=EPS2)
        assert (np.linalg.norm(a[off:off + n] - exact, axis=1) <= bound).all()
        off += n


def test_batch_rejects_unsupported_modes(nbp):
    m, p, v = nbp.universes.exponential_disc(64, 0)
    counts = np.array([32, 32], dtype=np.uint64)
    with pytest.raises(nbp.NbError):
        nbp.NbContext(nbp.SimConfig(mode=nbp.NB_MODE_FP64), m, p, v, counts=counts)
    with pytest.raises(nbp.NbError):
        nbp.NbContext(_split_cfg(nbp, 0.5), m, p, v, counts=np.array([64, 0], dtype=np.uint64))
    m2, p2, v2 = nbp.universes.exponential_disc(1025, 0)
    with pytest.raises(nbp.NbError):
        nbp.NbContext(_split_cfg(nbp, 0.5), m2, p2, v2, counts=np.ones(1025, dtype=np.uint64))


def test_autotune_restores_bodies(nbp):
    m, p, v = nbp.universes.colliding_discs(65536, 3)
    with nbp.NbContext(_split_cfg(nbp, 0.5), m, p, v) as ctx:
        ctx.step(1)
        p0, v0 = ctx.download()
        a0 = ctx.accelerations()
        leaf, bpl = ctx.autotune(2)
        assert leaf in (4, 8, 16, 32) and bpl in (1, 2, 4)
        p1, v1 = ctx.download()
        assert np.array_equal(p0, p1) and np.array_equal(v0, v1)
        assert ctx.stats().steps == 1
        a1 = ctx.accelerations()
    # a different leaf size or group size changes the cell set, not the law
    exact = nbp.allpairs_accelerations(m, p0, np.arange(0, 65536, 7), EPS2)
    assert np.percentile(rel_err(a1[::7], exact), 99) <= 1.5 * np.percentile(
        rel_err(a0[::7], exact), 99) + 1e-4


def test_batch_autotune(nbp):
    unis = nbp.universes.ensemble(16, 2, nmin=1024, nmax=20000)
    m, p, v, counts = _concat(unis)
    with nbp.NbContext(_split_cfg(nbp, 0.5), m, p, v, counts=counts) as ctx:
        leaf, bpl = ctx.autotune(2)
        ctx.step(2)
        pb, _ = ctx.download()
    assert leaf in (4, 8, 16, 32) and bpl in (1, 2, 4)
    assert np.isfinite(pb).all()

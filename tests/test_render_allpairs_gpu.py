"""GPU tests: the headless renderer against its CPU restatement (bit for bit)
and the all-pairs backend (the reference's AllPairsSim) against the FP64
oracle, in both pair laws."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("diam", [1.0, 2.5, 3.0, 7.0])
def test_render_matches_oracle(nbp, orc_render, diam):
    m, p, v = nbp.universes.colliding_discs(4000, 2)
    vp = nbp.render.ViewPort(256, 192, 0.25)
    with nbp.NbContext(nbp.SimConfig(mode=nbp.NB_MODE_SPLIT), m, p, v) as ctx:
        ctx.step(2)
        img = ctx.render(vp, point_diameter=diam)
        pos, _ = ctx.download()
    ref = orc_render.render(pos, vp.x, vp.y, vp.width, vp.height, vp.res_x, vp.res_y, diam)
    assert img.shape == (192, 256, 4)
    assert np.array_equal(img, ref)
    assert (img[..., 0] > 0).sum() > 100


def test_render_zoomed_and_clipped(nbp, orc_render):
    m, p, v = nbp.universes.exponential_disc(20000, 4)
    vp = nbp.render.ViewPort(300, 200, 0.02)
    vp.zoom(True, 30.0, 170.0)
    vp.pan(-40.0, 25.0)
    with nbp.NbContext(nbp.SimConfig(), m, p, v) as ctx:
        img = ctx.render(vp, point_diameter=4.0)
    ref = orc_render.render(p, vp.x, vp.y, vp.width, vp.height, vp.res_x, vp.res_y, 4.0)
    assert np.array_equal(img, ref)


def test_render_rejects_bad_views(nbp):
    m, p, v = nbp.universes.exponential_disc(100, 0)
    with nbp.NbContext(nbp.SimConfig(), m, p, v) as ctx:
        for bad in (nbp.NbView(0, 0, 1, 1, 0, 10, 1.0, 0), nbp.NbView(0, 0, 0, 1, 10, 10, 1.0, 0),
                    nbp.NbView(0, 0, 1, 1, 10, 10, 0.5, 0), nbp.NbView(0, 0, 1, 1, 10, 10, 51.0, 0)):
            with pytest.raises(nbp.NbError):
                ctx.render(bad)


@pytest.mark.parametrize("cpu_law", [False, True])
def test_allpairs_backend_accelerations(nbp, orc, cpu_law):
    m, p, v = nbp.universes.exponential_disc(3000, 7)
    cfg = nbp.SimConfig(mode=nbp.NB_MODE_ALLPAIRS, cpu_law=cpu_law, epsilon_squared=1e-4)
    with nbp.NbContext(cfg, m, p, v) as ctx:
        a = ctx.accelerations()
        st = ctx.stats()
    exact = (orc.allpairs_cpulaw(m, p, eps2=1e-4) if cpu_law
             else orc.allpairs_plummer(m, p, eps2=1e-4))
    assert rel_err(a, exact).max() < 1e-12
    assert st.body_interactions == 3000 * 2999


@pytest.mark.parametrize("cpu_law", [False, True])
def test_allpairs_backend_step_is_drift_then_kick(nbp, orc, cpu_law):
    """AllPairsSim::simulate (AllPairs.cpp:24-29): positions move with the old
    velocities, then the velocities take the forces at the new positions."""
    m, p, v = nbp.universes.colliding_discs(2000, 5)
    dt, G = 1e-3, 0.7
    cfg = nbp.SimConfig(mode=nbp.NB_MODE_ALLPAIRS, cpu_law=cpu_law, epsilon_squared=1e-4,
                        timestep=dt, G=G)
    with nbp.NbContext(cfg, m, p, v) as ctx:
        ctx.step(1)
        p1, v1 = ctx.download()
    p_ref = p + v * dt
    acc = (orc.allpairs_cpulaw(m, p_ref, eps2=1e-4) if cpu_law
           else orc.allpairs_plummer(m, p_ref, eps2=1e-4))
    v_ref = v + acc * G * dt
    assert np.array_equal(p1, p_ref)
    assert np.abs(v1 - v_ref).max() <= 1e-12 * np.abs(v_ref).max()


def test_allpairs_single_body_and_pair(nbp):
    cfg = nbp.SimConfig(mode=nbp.NB_MODE_ALLPAIRS, epsilon_squared=1e-4)
    with nbp.NbContext(cfg, np.ones(1), np.zeros((1, 2)), np.zeros((1, 2))) as ctx:
        assert np.array_equal(ctx.accelerations(), np.zeros((1, 2)))
    m = np.array([1.0, 3.0])
    p = np.array([[0.0, 0.0], [2.0, 0.0]])
    with nbp.NbContext(cfg, m, p, np.zeros((2, 2))) as ctx:
        a = ctx.accelerations()
    r3 = (4.0 + 1e-4) ** 1.5
    assert a[0, 0] == pytest.approx(3.0 * 2.0 / r3, rel=1e-14)
    assert a[1, 0] == pytest.approx(-1.0 * 2.0 / r3, rel=1e-14)

"""GPU tests of SPLIT mode (warp-cooperative FP32 group traversal).

SPLIT decides acceptance once per 32-body group, so its cell set differs from
the reference's per-body walk; it is judged against the FP64 all-pairs sum and
against the FP64 parity mode's own error."""
import pathlib

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
EPS2 = 1e-4


def accel(nbp, m, p, v, mode, theta, quad=False, leaf=0, eps2=EPS2):
    cfg = nbp.SimConfig(theta=theta, epsilon_squared=eps2, mode=mode, quadrupole=quad,
                        leaf_size=leaf)
    with nbp.NbContext(cfg, m, p, v) as ctx:
        a = ctx.accelerations()
        st = ctx.stats()
    return a, st


@pytest.mark.parametrize("n", [1, 2, 33, 1000, 16384])
def test_theta_zero_is_allpairs_in_fp32(nbp, orc, n):
    m, p, v = nbp.universes.exponential_disc(max(n, 2), 3)
    m, p, v = m[:n], p[:n], v[:n]
    a, _ = accel(nbp, m, p, v, nbp.NB_MODE_SPLIT, 0.0, leaf=1)
    exact = orc.allpairs_plummer(m, p, eps2=EPS2)
    if n == 1:
        assert np.array_equal(a, np.zeros((1, 2)))
        return
    # FP32: coordinates are rounded relative to the box centre, so the bound
    # grows with |x - centre| / |d| for close pairs
    box = orc.bbox_squared(p)
    center = (0.5 * (box[0] + box[1]), 0.5 * (box[2] + box[3]))
    bound = orc.allpairs_fp32_bound(m, p, center, eps2=EPS2)
    assert (np.linalg.norm(a - exact, axis=1) <= bound).all()


def test_monopole_error_not_worse_than_reference_walk(nbp):
    m, p, v = nbp.universes.exponential_disc(16384, 0)
    exact = nbp.allpairs_accelerations(m, p, np.arange(16384), EPS2)
    a64, _ = accel(nbp, m, p, v, nbp.NB_MODE_FP64, 0.5)
    a32, st = accel(nbp, m, p, v, nbp.NB_MODE_SPLIT, 0.5)
    e64, e32 = rel_err(a64, exact), rel_err(a32, exact)
    assert np.percentile(e32, 99) <= np.percentile(e64, 99) * 1.02
    assert np.percentile(e32, 50) <= np.percentile(e64, 50) * 1.02
    assert st.cell_interactions > 0 and st.body_interactions > 0


@pytest.mark.parametrize("theta", [0.5, 0.8])
def test_quadrupole_reduces_error(nbp, theta):
    m, p, v = nbp.universes.colliding_discs(32768, 1)
    tgt = np.arange(0, 32768, 3)
    exact = nbp.allpairs_accelerations(m, p, tgt, EPS2)
    a1, _ = accel(nbp, m, p, v, nbp.NB_MODE_SPLIT, theta)
    a2, _ = accel(nbp, m, p, v, nbp.NB_MODE_SPLIT, theta, quad=True)
    e1, e2 = rel_err(a1[tgt], exact), rel_err(a2[tgt], exact)
    assert np.percentile(e2, 99) < 0.5 * np.percentile(e1, 99)
    if theta == 0.5:
        assert np.percentile(e2, 99) < 1e-3


def test_split_step_matches_fp64_step(nbp):
    m, p, v = nbp.universes.colliding_discs(8192, 2)
    out = {}
    for mode in (nbp.NB_MODE_FP64, nbp.NB_MODE_SPLIT):
        cfg = nbp.SimConfig(theta=0.0, epsilon_squared=EPS2, mode=mode, leaf_size=1)
        with nbp.NbContext(cfg, m, p, v) as ctx:
            a0 = ctx.accelerations()
            ctx.step(1)
            out[mode] = (a0, *ctx.download())
    a64, p64, v64 = out[nbp.NB_MODE_FP64]
    a32, p32, v32 = out[nbp.NB_MODE_SPLIT]
    dv = 1e-4 * np.abs(a64 - a32).max()
    assert np.abs(v64 - v32).max() <= dv * 1.01 + 1e-15
    assert np.abs(p64 - p32).max() <= 1e-4 * dv * 1.01 + 1e-13


def test_split_coincident_and_ragged(nbp, orc):
    rng = np.random.default_rng(4)
    n = 1000
    p = rng.random((n, 2))
    p[10:40] = p[5]  # 31 coincident bodies (a multi-body leaf)
    m = rng.random(n) + 0.5
    a, _ = accel(nbp, m, p, np.zeros((n, 2)), nbp.NB_MODE_SPLIT, 0.0, leaf=1)
    exact = orc.allpairs_plummer(m, p, eps2=EPS2)
    box = orc.bbox_squared(p)
    center = (0.5 * (box[0] + box[1]), 0.5 * (box[2] + box[3]))
    bound = orc.allpairs_fp32_bound(m, p, center, eps2=EPS2)
    assert (np.linalg.norm(a - exact, axis=1) <= bound).all()


def test_split_zero_softening_coincident_bodies_add_nothing(nbp):
    """eps^2 = 0: bodies that share FP32 coordinates (here: exactly coincident
    pairs) add nothing to each other instead of 0 * inf; every other pair
    follows the unsoftened law."""
    rng = np.random.default_rng(6)
    n = 2000
    p = rng.random((n, 2))
    p[1000:1010] = p[:10]
    m = rng.random(n) + 0.5
    a, _ = accel(nbp, m, p, np.zeros((n, 2)), nbp.NB_MODE_SPLIT, 0.0, leaf=1, eps2=0.0)
    assert np.isfinite(a).all()
    d = p[None, :, :] - p[:, None, :]
    r2 = (d * d).sum(-1)
    w = np.where(r2 > 0, m[None, :] / np.where(r2 > 0, r2, 1.0) ** 1.5, 0.0)
    exact = (w[:, :, None] * d).sum(1)
    assert np.percentile(rel_err(a, exact), 99) < 1e-3


@pytest.mark.parametrize("quad", [False, True])
def test_bmax_guard_tightens_the_walk(nbp, quad):
    """Barnes' b_max test on top of the width test: a cell whose centre of
    mass sits near a corner is opened unless d > b_max / ratio.  At theta = 1
    that removes the slowly converging cells that set the p99 error."""
    m, p, v = nbp.universes.colliding_discs(65536, 4)
    tgt = np.arange(0, 65536, 5)
    exact = nbp.allpairs_accelerations(m, p, tgt, EPS2)
    out = {}
    for ratio in (0.0, 0.75):
        cfg = nbp.SimConfig(theta=1.0, epsilon_squared=EPS2, mode=nbp.NB_MODE_SPLIT,
                            quadrupole=quad, bmax_ratio=ratio)
        with nbp.NbContext(cfg, m, p, v) as ctx:
            a = ctx.accelerations()
            st = ctx.stats()
        out[ratio] = (np.percentile(rel_err(a[tgt], exact), 99), st.cell_interactions)
    assert out[0.75][1] >= out[0.0][1]  # only ever opens more cells
    assert out[0.75][0] < 0.7 * out[0.0][0]


@pytest.mark.parametrize("bpl", [1, 2, 4])
def test_group_sizes_theta_zero_and_errors(nbp, orc, bpl):
    # target groups of 32, 64 and 128 bodies: at theta = 0 every group sums
    # every body (the FP32 bound of the all-pairs sum holds), and at theta =
    # 0.5 (monopole and quadrupole) the error stays that of the default groups
    m, p, v = nbp.universes.colliding_discs(20000, 6)
    cfg = nbp.SimConfig(theta=0.0, epsilon_squared=EPS2, mode=nbp.NB_MODE_SPLIT, leaf_size=1,
                        bodies_per_lane=bpl)
    with nbp.NbContext(cfg, m, p, v) as ctx:
        a0 = ctx.accelerations()
    tgt = np.arange(0, 20000, 7)
    box = orc.bbox_squared(p)
    center = (0.5 * (box[0] + box[1]), 0.5 * (box[2] + box[3]))
    bound = orc.allpairs_fp32_bound(m, p, center, targets=tgt, eps2=EPS2)
    exact = orc.allpairs_plummer(m, p, tgt, eps2=EPS2)
    assert (np.linalg.norm(a0[tgt] - exact, axis=1) <= bound).all()
    for quad in (False, True):
        errs = {}
        for b in (2, bpl):
            cfg = nbp.SimConfig(theta=0.5, epsilon_squared=EPS2, mode=nbp.NB_MODE_SPLIT,
                                quadrupole=quad, bodies_per_lane=b)
            with nbp.NbContext(cfg, m, p, v) as ctx:
                ctx.step(1)  # a step first: groups are built by the step's graph too
                errs[b] = np.percentile(rel_err(ctx.accelerations()[tgt],
                                                nbp.allpairs_accelerations(
                                                    m, ctx.download()[0], tgt, EPS2)), 99)
        # larger groups accept fewer cells (a looser box), smaller ones more
        assert errs[bpl] <= errs[2] * (1.3 if bpl == 1 else 1.02), (quad, errs)


def _bodies_in_group_boxes(pos, groups, chunk=64):
    """For each group [first, last] (device order), how many bodies of pos lie
    inside the bounding box of the group's own bodies."""
    lo = np.array([pos[a:b + 1].min(axis=0) for a, b in groups])
    hi = np.array([pos[a:b + 1].max(axis=0) for a, b in groups])
    out = np.empty(len(groups), dtype=np.int64)
    for s in range(0, len(groups), chunk):
        l, h = lo[s:s + chunk, None, :], hi[s:s + chunk, None, :]
        inside = ((pos[None] >= l) & (pos[None] <= h)).all(axis=2)
        out[s:s + chunk] = inside.sum(axis=1)
    return out


@pytest.mark.parametrize("kind", ["disc", "plummer"])
@pytest.mark.parametrize("bpl", [1, 2, 4])
@pytest.mark.parametrize("learned", [False, True])
def test_group_boxes_hold_few_foreign_bodies(nbp, kind, bpl, learned):
    # A group's walk opens every cell inside its bounding box down to the
    # bodies, so the box must not cover a dense region.  Runs of sibling
    # children stay inside one half of their parent when a sibling is large,
    # which bounds the bodies inside any group's box by 4 group sizes (the
    # parent of a run without large siblings holds at most 4).  Merged runs
    # across both halves once put the core of a sparse 65,536-body universe
    # inside one group's box (a 2-5 ms step instead of 0.3 ms).
    n = 65536
    m, p, v = nbp.universes.make(kind, n, 0)
    cfg = nbp.SimConfig(theta=0.5, epsilon_squared=EPS2, mode=nbp.NB_MODE_SPLIT,
                        bodies_per_lane=bpl, learned=learned)
    with nbp.NbContext(cfg, m, p, v) as ctx:
        if learned:
            wdir = pathlib.Path(nbp.__file__).resolve().parent / "weights"
            ctx.set_mlp_weights(np.load(wdir / "correction_theta1.npy"))
        ctx.accelerations()
        g = ctx.debug_groups()
        _, pos, _, _ = ctx.debug_state()
    gsize = 64 if learned else 32 * bpl      # the learned correction keeps groups of 64
    assert (g[:, 1] - g[:, 0] + 1).max() <= gsize
    inside = _bodies_in_group_boxes(pos, g)
    assert inside.max() <= 4 * gsize, (inside.max(), int((inside > 4 * gsize).sum()))

"""CPU tests of the oracle itself (the checker), against known answers,
independent restatements and the reference's own invariants."""
import numpy as np
import pytest

from conftest import rel_err


def _interleave(v: int) -> int:
    out = 0
    for b in range(32):
        out |= ((v >> b) & 1) << (2 * b)
    return out


def test_morton_known_answers(orc):
    # Box [0, 1) x [0, 1) after squaring; codes by hand from CU:54-69:
    # x bits on odd positions, y bits on even positions, 32 bits per axis.
    pos = np.array([[0.0, 0.0], [1.0, 1.0], [0.5, 0.0], [0.0, 0.5], [0.25, 0.75]])
    box = orc.bbox_squared(pos)
    assert box.tolist() == [0.0, 1.0, 0.0, 1.0]
    codes = orc.morton(pos, box)
    assert codes[0] == 0
    assert codes[1] == 0xFFFFFFFFFFFFFFFF  # clamped to 2^32 - 1 on both axes
    assert codes[2] == 1 << 63             # x = 2^31 -> top x bit
    assert codes[3] == 1 << 62             # y = 2^31 -> top y bit
    ix, iy = 1 << 30, 3 << 30
    assert codes[4] == (_interleave(ix) << 1) | _interleave(iy)


def test_morton_matches_python_restatement(orc):
    rng = np.random.default_rng(3)
    pos = rng.normal(size=(5000, 2)) * np.array([3.0, 0.5]) + 7.0
    box = orc.bbox_squared(pos)
    # squaring: the shorter (y) side grows about its midpoint
    assert box[1] - box[0] == pytest.approx(box[3] - box[2], rel=1e-15)
    codes = orc.morton(pos, box)
    inv_w = 1.0 / (box[1] - box[0])
    inv_h = 1.0 / (box[3] - box[2])
    for k in range(0, 5000, 97):
        nx = (pos[k, 0] - box[0]) * inv_w
        ny = (pos[k, 1] - box[2]) * inv_h
        qx = int(np.floor(min(max(nx * 4294967296.0, 0.0), 4294967295.0)))
        qy = int(np.floor(min(max(ny * 4294967296.0, 0.0), 4294967295.0)))
        assert int(codes[k]) == (_interleave(qx) << 1) | _interleave(qy)


def test_stable_sort_matches_numpy(orc):
    rng = np.random.default_rng(5)
    keys = rng.integers(0, 50, size=20000).astype(np.uint64) << np.uint64(40)
    keys |= rng.integers(0, 4, size=20000).astype(np.uint64)  # many ties
    out, order = orc.stable_sort(keys)
    ref = np.argsort(keys, kind="stable")
    assert np.array_equal(order, ref)
    assert np.array_equal(out, keys[ref])


def test_theta_zero_equals_allpairs(nbp, orc):
    # With theta = 0 no internal cell is ever accepted, so the reference
    # traversal (CU:382-486) degenerates to the exact pair sum.
    m, p, v = nbp.universes.exponential_disc(4096, 11)
    st = orc.RefState(m, p, v)
    r = st.step(theta=0.0, integrate=False, want_acc=True)
    acc_bh = st.in_original_order(r["acc"])
    acc_ap = orc.allpairs_plummer(m, p, eps2=1e-4)
    assert rel_err(acc_bh, acc_ap).max() < 1e-12
    assert r["stats"]["cell_interactions"] == 0
    assert r["stats"]["body_interactions"] == 4096 * 4095


def test_tree_counts_small_case(orc):
    # Four bodies, one per quadrant of the unit box: root + 4 children.
    p = np.array([[0.1, 0.1], [0.1, 0.9], [0.9, 0.1], [0.9, 0.9]])
    m = np.ones(4)
    st = orc.RefState(m, p, np.zeros((4, 2)))
    r = st.step(theta=0.5, integrate=False, want_acc=True)
    s = r["stats"]
    assert s["nodes_allocated"] == 5 and s["nodes_nonempty"] == 5 and s["levels"] == 2
    # order by Morton quadrant digit (x<<1)|y: q0=(lo,lo) q1=(lo,hi) q2=(hi,lo) q3=(hi,hi)
    assert st.orig.tolist() == [0, 1, 2, 3]


def test_kick_then_drift(orc):
    # CU:484-495: v += a G dt first, then x += v dt with the new velocity.
    p = np.array([[0.0, 0.0], [1.0, 0.0]])
    m = np.array([1.0, 2.0])
    st = orc.RefState(m, p, np.zeros((2, 2)))
    G, dt, eps2 = 0.5, 0.1, 0.0
    st.step(G=G, dt=dt, eps2=eps2, theta=0.5)
    vel = st.in_original_order(st.vel)
    pos = st.in_original_order(st.pos)
    assert vel[0, 0] == pytest.approx(2.0 * G * dt)
    assert vel[1, 0] == pytest.approx(-1.0 * G * dt)
    assert pos[0, 0] == pytest.approx(vel[0, 0] * dt)


def test_duplicate_positions_make_level30_leaf(orc):
    # Bodies closer than width / 2^30 share a 60-bit prefix and end in one
    # multi-body leaf at level 30 (CU:182); a body outside sees its COM.
    rng = np.random.default_rng(2)
    p = np.concatenate([rng.random((60, 2)), [[0.5, 0.5], [0.5, 0.5]]])
    m = rng.random(62) + 0.5
    st = orc.RefState(m, p, np.zeros((62, 2)))
    r = st.step(theta=0.0, integrate=False, want_acc=True)
    assert r["stats"]["multi_leaves"] == 1
    assert r["stats"]["max_level"] == 30
    # at theta = 0 only the coincident pair is summed through its COM, which
    # sits exactly on both bodies, so the result is the exact pair sum
    acc = st.in_original_order(r["acc"])
    ap = orc.allpairs_plummer(m, p, eps2=1e-4)
    assert rel_err(acc, ap).max() < 1e-12


def test_node_pool_truncation_quirk(orc):
    # The reference's node pool holds 5n cells (BarnesHutCuda.cpp:9); when a
    # split would overflow it, the cell silently stays a multi-body leaf
    # (CU:212-214).  Four bodies with one duplicate pair overflow at level 4.
    p = np.array([[0.0, 0.0], [1.0, 1.0], [1.0, 1.0], [0.3, 0.6]])
    m = np.array([1.0, 1.0, 2.0, 1.0])
    st = orc.RefState(m, p, np.zeros((4, 2)))
    r = st.step(theta=0.5, integrate=False, want_acc=True)
    assert r["stats"]["multi_leaves"] == 1
    assert r["stats"]["max_level"] == 4
    assert r["stats"]["nodes_allocated"] > 5 * 4


def test_cpu_law_allpairs(orc):
    # Simulation::force (Simulation.cpp:74-80): |a| = G M / (d^2 + eps^2).
    p = np.array([[0.0, 0.0], [3.0, 4.0]])
    m = np.array([1.0, 2.0])
    a = orc.allpairs_cpulaw(m, p, G=1.5, eps2=1.0)
    assert np.allclose(a[0], 1.5 * 2.0 / 26.0 * np.array([0.6, 0.8]))


def test_walk_targets_equals_the_full_step(orc, nbp):
    # the targets-only walk sorts and builds exactly as the full step does and
    # walks the chosen bodies with the same DFS: same accelerations (bit for
    # bit), and per-target counts that add up to the step's totals
    m, p, v = nbp.universes.colliding_discs(6000, 4)
    full = orc.RefState(m, p, v)
    r = full.step(theta=0.7, eps2=1e-4, integrate=False, want_acc=True)
    acc_full = full.in_original_order(r["acc"])
    tgt = np.random.default_rng(1).permutation(6000)
    part = orc.RefState(m, p, v)
    w = part.walk_targets(tgt, eps2=1e-4, theta=0.7)
    assert np.array_equal(w["acc"], acc_full[tgt])
    assert np.array_equal(part.orig, full.orig)
    assert w["cells"].sum() == r["stats"]["cell_interactions"]
    assert w["pairs"].sum() == r["stats"]["body_interactions"]
    assert w["stack"].max() == r["stats"]["max_stack"]
    few = orc.RefState(m, p, v).walk_targets(tgt[:17], eps2=1e-4, theta=0.7)
    assert np.array_equal(few["acc"], acc_full[tgt[:17]])
    with pytest.raises(IndexError):
        orc.RefState(m, p, v).walk_targets(np.array([6000]))

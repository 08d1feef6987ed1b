"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Bit-exact for Morton codes, the squared box and the sort permutation;
accelerations within 1e-5 relative (FP64 mode) of the oracle's restatement
of the reference traversal, with the same accepted-cell counts."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

EPS2 = 1e-4
TOL = 1e-5  # FP64 mode: relative acceleration tolerance vs the oracle


def ctx_for(nbp, m, p, v, theta=0.5, dt=1e-4, G=1.0, mode=0):
    cfg = nbp.SimConfig(timestep=dt, theta=theta, epsilon_squared=EPS2, G=G, mode=mode)
    return nbp.NbContext(cfg, m, p, v)


def universes(nbp):
    u = nbp.universes
    rng = np.random.default_rng(7)
    yield "disc16k", u.exponential_disc(16384, 0)
    yield "collision8k", u.colliding_discs(8192, 1)
    yield "plummer5k", u.plummer_disc(5000, 2)
    m = rng.random(3001) + 0.1
    yield "uniform3001", (m, rng.random((3001, 2)) * 100 - 50, rng.normal(size=(3001, 2)))


@pytest.mark.parametrize("n", [1, 2, 3, 31, 2047, 2048, 2049, 65537])
def test_morton_sort_bitexact_ragged(nbp, orc, n):
    rng = np.random.default_rng(n)
    p = rng.normal(size=(n, 2)) * [4.0, 1.0]
    if n > 8:
        p[5] = p[3]  # exact ties keep their slot order
        p[7] = p[3]
    m = np.ones(n)
    with ctx_for(nbp, m, p, np.zeros((n, 2))) as ctx:
        codes, order, box = ctx.debug_morton()
    box_o = orc.bbox_squared(p)
    assert np.array_equal(box, box_o)
    codes_o, order_o = orc.stable_sort(orc.morton(p, box_o))
    assert np.array_equal(codes, codes_o)
    assert np.array_equal(order, order_o)


def test_morton_sort_bitexact_workloads(nbp, orc):
    for name, (m, p, v) in universes(nbp):
        with ctx_for(nbp, m, p, v) as ctx:
            codes, order, box = ctx.debug_morton()
        codes_o, order_o = orc.stable_sort(orc.morton(p))
        assert np.array_equal(codes, codes_o), name
        assert np.array_equal(order, order_o), name


@pytest.mark.parametrize("theta", [0.0, 0.3, 0.5, 1.0])
def test_accelerations_fp64(nbp, orc, theta):
    for name, (m, p, v) in universes(nbp):
        with ctx_for(nbp, m, p, v, theta=theta) as ctx:
            acc = ctx.accelerations()
            st = ctx.stats()
        ref = orc.RefState(m, p, v)
        r = ref.step(theta=theta, eps2=EPS2, integrate=False, want_acc=True)
        acc_o = ref.in_original_order(r["acc"])
        err = rel_err(acc, acc_o)
        assert err.max() < TOL, (name, theta, err.max())
        s = r["stats"]
        total_o = s["cell_interactions"] + s["body_interactions"]
        total = st.cell_interactions + st.body_interactions
        assert abs(total - total_o) <= 1e-6 * total_o + 2, (name, theta, total, total_o)


def test_steps_track_oracle(nbp, orc):
    # Each GPU step is checked against one oracle step taken from the GPU's own
    # device-order state, so chaos cannot amplify earlier rounding.
    m, p, v = nbp.universes.exponential_disc(16384, 0)
    dt = 1e-4
    with ctx_for(nbp, m, p, v, dt=dt) as ctx:
        for _ in range(5):
            mass, pos, vel, orig = ctx.debug_state()
            v_pre = np.empty_like(vel)
            v_pre[orig] = vel
            ref = orc.RefState(mass, pos, vel, orig)
            ref.step(theta=0.5, eps2=EPS2, dt=dt, G=1.0)
            ctx.step(1)
            mass2, pos2, vel2, orig2 = ctx.debug_state()
            assert np.array_equal(orig2, ref.orig)
            assert np.array_equal(mass2, ref.mass)
            kick = vel2 - v_pre[orig2]
            kick_o = ref.vel - v_pre[ref.orig]
            assert rel_err(kick, kick_o).max() < TOL
            bound = 1e-15 * np.abs(ref.pos).max() + dt * np.abs(vel2 - ref.vel).max() * 1.01
            assert np.abs(pos2 - ref.pos).max() <= bound + 1e-300


def test_download_original_order(nbp, orc):
    m, p, v = nbp.universes.colliding_discs(4096, 3)
    with ctx_for(nbp, m, p, v) as ctx:
        pos0, vel0 = ctx.download()
        assert np.array_equal(pos0, p) and np.array_equal(vel0, v)
        ctx.step(3)
        pos, vel = ctx.download()
    ref = orc.RefState(m, p, v)
    for _ in range(3):
        ref.step(theta=0.5, eps2=EPS2)
    assert np.abs(ref.in_original_order(ref.pos) - pos).max() < 1e-10
    assert np.abs(ref.in_original_order(ref.vel) - vel).max() < 1e-8


def test_tree_invariants(nbp):
    m, p, v = nbp.universes.exponential_disc(20000, 4)
    with ctx_for(nbp, m, p, v) as ctx:
        ctx.accelerations()
        t = ctx.debug_tree()
        mass, pos, _, _ = ctx.debug_state()
    root = t["root"]
    assert root >= 0
    assert t["first"][root] == 0 and t["last"][root] == len(m) - 1
    assert t["mass"][root] == pytest.approx(m.sum(), rel=1e-12)
    # every cell's mass and centre of mass equal the direct sums over its range
    for cid in range(0, len(t["mass"]), 37):
        a, b = t["first"][cid], t["last"][cid]
        mm = mass[a:b + 1]
        assert t["mass"][cid] == pytest.approx(mm.sum(), rel=1e-12)
        com = (mm[:, None] * pos[a:b + 1]).sum(0) / mm.sum()
        assert np.allclose(t["com"][cid], com, rtol=1e-12, atol=1e-12)
    assert (t["level"] >= 0).all() and (t["level"] < 30).all()


def _cells_from_codes(codes):
    """The compressed quadtree's cells from sorted codes, built on the host
    with a plain stack: boundary i (bodies i, i + 1) has level c_i = shared
    leading 2-bit digits (capped at 30); the cell a boundary below 30
    separates spans the bodies between the nearest smaller levels on either
    side, and its first separator creates it.  Returns {(first, last, level)}."""
    codes = codes.astype(np.uint64)
    x = codes[:-1] ^ codes[1:]
    bitlen = np.zeros(x.shape, dtype=np.int64)
    for k in range(64):
        bitlen += ((x >> np.uint64(k)) > 0).astype(np.int64)
    c = np.minimum((64 - bitlen) // 2, 30)
    n, m = len(codes), len(c)
    left_lt, left_le, right_lt = np.full(m, -1), np.full(m, -1), np.full(m, n - 1)
    stack = []
    for i in range(m):  # nearest smaller (and smaller-or-equal) on the left
        while stack and c[stack[-1]] > c[i]:
            stack.pop()
        left_le[i] = stack[-1] if stack else -1
        j = len(stack) - 1
        while j >= 0 and c[stack[j]] >= c[i]:
            j -= 1
        left_lt[i] = stack[j] if j >= 0 else -1
        stack.append(i)
    stack = []
    for i in range(m - 1, -1, -1):  # nearest smaller on the right
        while stack and c[stack[-1]] >= c[i]:
            stack.pop()
        right_lt[i] = stack[-1] if stack else n - 1
        stack.append(i)
    return {(int(left_lt[i] + 1), int(right_lt[i]), int(c[i])) for i in range(m)
            if c[i] < 30 and left_le[i] == left_lt[i]}


@pytest.mark.parametrize("n", [2047, 2048, 2049, 6145, 40000])
def test_tree_cells_across_tiles(nbp, n):
    """The device build works on tiles of 2,048 boundaries with per-tile
    tables for what lies beyond a tile; its cells (body range and level)
    must equal a plain host construction, including at tile edges and with
    level-30 leaves (coincident bodies)."""
    m, p, v = nbp.universes.colliding_discs(n + (n & 1), 2)
    m, p, v = m[:n], p[:n].copy(), v[:n]
    p[100:140] = p[100]          # a multi-body leaf
    p[n // 2:n // 2 + 5] = p[n // 2]
    with ctx_for(nbp, m, p, v) as ctx:
        ctx.accelerations()
        t = ctx.debug_tree()
        codes, order, _ = ctx.debug_morton()
    assert np.array_equal(order, np.arange(n))   # the state is already in code order
    got = set(zip(t["first"].tolist(), t["last"].tolist(), t["level"].tolist()))
    assert len(got) == len(t["first"])
    assert got == _cells_from_codes(codes)


def test_single_body_and_coincident_bodies(nbp, orc):
    with ctx_for(nbp, np.ones(1), np.zeros((1, 2)), np.ones((1, 2))) as ctx:
        assert np.array_equal(ctx.accelerations(), np.zeros((1, 2)))
        ctx.step(2)
        pos, vel = ctx.download()
        assert np.allclose(pos, 2e-4) and np.allclose(vel, 1.0)
    # all bodies on one point: one level-30 leaf holds everything
    n = 64
    p = np.full((n, 2), 3.25)
    m = np.linspace(1.0, 2.0, n)
    for theta in (0.5, 1.0, 2.0):
        with ctx_for(nbp, m, p, np.zeros((n, 2)), theta=theta) as ctx:
            acc = ctx.accelerations()
        ref = orc.RefState(m, p, np.zeros((n, 2)))
        r = ref.step(theta=theta, eps2=EPS2, integrate=False, want_acc=True)
        assert np.allclose(acc, ref.in_original_order(r["acc"]), atol=1e-12)


def test_coincident_pairs_inside_disc(nbp, orc):
    m, p, v = nbp.universes.exponential_disc(8192, 9)
    p[100:110] = p[50]       # a 11-body multi-body leaf
    p[200] = p[201]          # and a pair
    for theta in (0.5, 1.0):
        with ctx_for(nbp, m, p, v, theta=theta) as ctx:
            acc = ctx.accelerations()
        ref = orc.RefState(m, p, v)
        r = ref.step(theta=theta, eps2=EPS2, integrate=False, want_acc=True)
        assert r["stats"]["multi_leaves"] == 2
        err = rel_err(acc, ref.in_original_order(r["acc"]))
        assert err.max() < TOL, (theta, err.max())


def test_rejects_nonfinite_and_nonpositive(nbp):
    p = np.zeros((4, 2))
    p[2, 1] = np.nan
    with pytest.raises(nbp.NbError):
        ctx_for(nbp, np.ones(4), p, np.zeros((4, 2)))
    with pytest.raises(nbp.NbError):
        ctx_for(nbp, np.array([1.0, 0.0]), np.zeros((2, 2)), np.zeros((2, 2)))


def test_timestep_hot_swap(nbp, orc):
    m, p, v = nbp.universes.exponential_disc(2048, 6)
    with ctx_for(nbp, m, p, v, dt=1e-4) as ctx:
        ctx.step(1)
        ctx.set_timestep(2e-4)
        ctx.step(1)
        pos, vel = ctx.download()
    ref = orc.RefState(m, p, v)
    ref.step(dt=1e-4, eps2=EPS2)
    ref.step(dt=2e-4, eps2=EPS2)
    assert np.abs(ref.in_original_order(ref.pos) - pos).max() < 1e-10


def test_allpairs_kernel_matches_oracle(nbp, orc):
    m, p, _ = nbp.universes.colliding_discs(10000, 5)
    tgt = np.arange(0, 10000, 7)
    acc = nbp.allpairs_accelerations(m, p, tgt, EPS2)
    acc_o = orc.allpairs_plummer(m, p, tgt, eps2=EPS2)
    assert rel_err(acc, acc_o).max() < 1e-12


def test_upload_rejects_non_finite_and_non_positive_masses(nbp):
    m, p, v = nbp.universes.exponential_disc(5000, 1)
    with nbp.NbContext(nbp.SimConfig(mode=nbp.NB_MODE_SPLIT), m, p, v) as ctx:
        bad = p.copy()
        bad[1234, 1] = np.nan
        with pytest.raises(nbp.NbError, match="non-finite"):
            ctx.upload(m, bad, v)
        badv = v.copy()
        badv[17, 0] = np.inf
        with pytest.raises(nbp.NbError, match="non-finite"):
            ctx.upload(m, p, badv)
        badm = m.copy()
        badm[4999] = 0.0
        with pytest.raises(nbp.NbError, match="positive"):
            ctx.upload(badm, p, v)
        ctx.upload(m, p, v)
        ctx.step(1)
        p1, _ = ctx.download()
        assert np.isfinite(p1).all()
    with pytest.raises(nbp.NbError):
        nbp.NbContext(nbp.SimConfig(), -m, p, v)


def test_download_async_matches_download(nbp):
    torch = pytest.importorskip("torch")
    m, p, v = nbp.universes.colliding_discs(20000, 3)
    pin = lambda: torch.empty((20000, 2), dtype=torch.float64, pin_memory=True).numpy()
    with nbp.NbContext(nbp.SimConfig(mode=nbp.NB_MODE_SPLIT), m, p, v) as ctx:
        outs = []
        for k in range(3):
            ctx.upload(m, p, v)
            ctx.step(k + 1, sync=False)
            po, vo = pin(), pin()
            ctx.download_async(po, vo)
            outs.append((po, vo))
        ctx.download_wait()
        ps, vs = ctx.download()
    with nbp.NbContext(nbp.SimConfig(mode=nbp.NB_MODE_SPLIT), m, p, v) as ref:
        for k in range(3):
            ref.upload(m, p, v)
            ref.step(k + 1)
            pr, vr = ref.download()
            assert np.array_equal(outs[k][0], pr) and np.array_equal(outs[k][1], vr)
    assert np.array_equal(ps, outs[2][0]) and np.array_equal(vs, outs[2][1])


def test_upload_async_matches_upload(nbp):
    """Pipelined uploads give the steps the same bodies as synchronous ones;
    work enqueued before an asynchronous upload still sees the old state."""
    torch = pytest.importorskip("torch")
    n = 20000
    m, p, v = nbp.universes.colliding_discs(n, 4)
    pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    hm, hp, hv = pin((n,)), pin((n, 2)), pin((n, 2))
    hm[:], hp[:], hv[:] = m, p, v
    hp2 = pin((n, 2))
    hp2[:] = p + 0.5
    cfg = nbp.SimConfig(mode=nbp.NB_MODE_SPLIT)
    with nbp.NbContext(cfg, m, p, v) as ctx:
        outs = []
        for k in range(3):
            ctx.step(1, sync=False)  # after a step the state sits in the second buffer
            po0, vo0 = pin((n, 2)), pin((n, 2))
            ctx.download_async(po0, vo0)  # enqueued before the upload: old state
            ctx.upload_async(hm, hp2 if k == 1 else hp, hv)
            ctx.step(k + 1, sync=False)
            po, vo = pin((n, 2)), pin((n, 2))
            ctx.download_async(po, vo)
            outs.append((po0, vo0, po, vo))
        ctx.download_wait()
        ctx.sync()
    with nbp.NbContext(cfg, m, p, v) as ref:
        for k in range(3):
            ref.step(1)
            p0, v0 = ref.download()
            assert np.array_equal(outs[k][0], p0) and np.array_equal(outs[k][1], v0)
            ref.upload(m, p + 0.5 if k == 1 else p, v)
            ref.step(k + 1)
            pr, vr = ref.download()
            assert np.array_equal(outs[k][2], pr) and np.array_equal(outs[k][3], vr)


@pytest.mark.parametrize("steps_before", [0, 1])
def test_upload_async_rejects_and_keeps_state(nbp, steps_before):
    """A rejected asynchronous upload is reported at the next sync and leaves
    the state as it was, from either state buffer."""
    torch = pytest.importorskip("torch")
    n = 5000
    m, p, v = nbp.universes.exponential_disc(n, 2)
    pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    hm, hp, hv = pin((n,)), pin((n, 2)), pin((n, 2))
    hm[:], hp[:], hv[:] = m, p, v
    hp[100, 0] = np.nan
    with nbp.NbContext(nbp.SimConfig(mode=nbp.NB_MODE_SPLIT), m, p, v) as ctx:
        if steps_before:
            ctx.step(steps_before)
        p0, v0 = ctx.download()
        ctx.upload_async(hm, hp, hv)
        with pytest.raises(nbp.NbError, match="asynchronous upload rejected"):
            ctx.sync()
        p1, v1 = ctx.download()
        assert np.array_equal(p0, p1) and np.array_equal(v0, v1)
        hp[100, 0] = p[100, 0]
        hm[7] = -1.0
        ctx.upload_async(hm, hp, hv)
        with pytest.raises(nbp.NbError, match="asynchronous upload rejected"):
            ctx.sync()
        hm[7] = m[7]
        ctx.upload_async(hm, hp, hv)
        ctx.step(1)
        p2, _ = ctx.download()
    with nbp.NbContext(nbp.SimConfig(mode=nbp.NB_MODE_SPLIT), m, p, v) as ref:
        ref.step(1)
        pr, _ = ref.download()
    assert np.array_equal(p2, pr)


def test_bounded_wait_times_out_without_hanging(nbp):
    """The radix sort's look-back waits on a predecessor tile; with one that
    never publishes, the wait gives up after its iteration bound, the kernel
    raises the timeout flag and returns, and the GPU stays usable."""
    import time

    lib = nbp.load()
    t0 = time.perf_counter()
    assert lib.nb_debug_wait_timeout(0) == 4  # NB_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 60
    m, p, v = nbp.universes.exponential_disc(1000, 2)
    with nbp.NbContext(nbp.SimConfig(mode=nbp.NB_MODE_SPLIT), m, p, v) as ctx:
        ctx.step(2)
        assert np.isfinite(ctx.download()[0]).all()


def test_fp64_mode_ignores_the_bmax_ratio(nbp):
    m, p, v = nbp.universes.exponential_disc(3000, 4)
    out = []
    for ratio in (0.0, 0.75):
        cfg = nbp.SimConfig(mode=nbp.NB_MODE_FP64, theta=0.8, bmax_ratio=ratio)
        with nbp.NbContext(cfg, m, p, v) as ctx:
            out.append(ctx.accelerations())
    assert np.array_equal(out[0], out[1])


def _sort_cases(rng):
    yield "random", rng.normal(size=(100_003, 2)) * [4.0, 1.0]
    # half the bodies inside a square 1e-7 wide: groups tied in any number of
    # top bytes, of every size up to 50,000 (the one-warp radix path)
    p = rng.random((100_000, 2)) * 10.0
    p[:50_000] = 3.0 + rng.random((50_000, 2)) * 1e-7
    yield "cluster", p
    # exact copies: equal keys keep their input order
    p = rng.random((15_001, 2))
    p[:15_000] = np.repeat(rng.random((5, 2)), 3000, axis=0)
    yield "coincident", rng.permutation(p)


@pytest.mark.parametrize("passes", [1, 2, 3, 4, 5, 6, 7, 8])
def test_sort_with_any_pass_count_is_the_full_stable_sort(nbp, orc, passes):
    # the radix passes order only the top `passes` bytes; the tie pass must
    # turn that into the stable sort of all 64 bits
    rng = np.random.default_rng(100 + passes)
    for name, p in _sort_cases(rng):
        n = p.shape[0]
        with ctx_for(nbp, np.ones(n), p, np.zeros((n, 2))) as ctx:
            ctx.debug_sort_passes(passes)
            codes, order, box = ctx.debug_morton()
            assert ctx.debug_sort_passes() == passes
        codes_o, order_o = orc.stable_sort(orc.morton(p))
        assert np.array_equal(codes, codes_o), name
        assert np.array_equal(order, order_o), name


def test_automatic_pass_count_follows_the_tree(nbp, orc):
    # the first sort has no tree to learn from and takes all 8 passes; later
    # sorts take fewer on a smooth disc, and stay exact
    m, p, v = nbp.universes.colliding_discs(262_144, 9)
    with ctx_for(nbp, m, p, v, mode=nbp.NB_MODE_SPLIT) as ctx:
        ctx.debug_morton()
        assert ctx.debug_sort_passes() == 8
        ctx.step(2)
        codes, order, _ = ctx.debug_morton()
        auto = ctx.debug_sort_passes()
        mass, pos, vel, orig = ctx.debug_state()
    assert 1 <= auto < 8
    codes_o, order_o = orc.stable_sort(orc.morton(pos))
    assert np.array_equal(codes, codes_o)
    assert np.array_equal(order, order_o)

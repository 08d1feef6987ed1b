"""Golden vectors from the reference's own CUDA kernels.

tests/golden/*.npz were produced by tests/golden/make_golden.py, which runs
src/Simulation/src/BarnesHutCuda.cu's kernels (compiled unmodified into
oracle/_ref/ref_gpu_harness) on a B200.  They pin the CPU oracle (CPU tests)
and the CUDA path (GPU tests): squared box, Morton codes, sort permutation,
node-pool size and level count bit-exact; first-step accelerations and the
state after a few steps to tight tolerances."""
import pathlib

import numpy as np
import pytest

from conftest import rel_err

GOLDEN = sorted((pathlib.Path(__file__).parent / "golden").glob("*.npz"))


def load(path):
    g = dict(np.load(path))
    for k in ("theta", "eps2", "dt", "G"):
        g[k] = float(g[k])
    g["steps"] = int(g["steps"])
    return g


def test_goldens_present():
    assert len(GOLDEN) >= 8


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_reference_kernels(orc, path):
    g = load(path)
    assert np.array_equal(orc.bbox_squared(g["pos0"]), g["box"])
    st = orc.RefState(g["mass"], g["pos0"], g["vel0"])
    r = st.step(theta=g["theta"], eps2=g["eps2"], dt=g["dt"], G=g["G"], want_acc=True,
                want_codes=True)
    assert np.array_equal(r["codes"], g["codes"])
    assert np.array_equal(r["order"], g["perm"])
    assert np.array_equal(st.orig, g["orig"])
    assert r["stats"]["nodes_allocated"] == g["nodes_allocated"]
    assert r["stats"]["levels"] == g["levels"]
    # FP64 on both sides; the GPU's double rsqrt and its choice of fused
    # multiply-adds leave differences of a few ulps
    assert rel_err(r["acc"], g["acc"]).max() < 1e-12
    for _ in range(g["steps"] - 1):
        st.step(theta=g["theta"], eps2=g["eps2"], dt=g["dt"], G=g["G"])
    pos = st.in_original_order(st.pos)
    vel = st.in_original_order(st.vel)
    assert np.abs(pos - g["pos"]).max() <= 1e-13 * max(1.0, np.abs(g["pos"]).max())
    assert np.abs(vel - g["vel"]).max() <= 1e-9 * max(1.0, np.abs(g["vel"]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_cuda_path_matches_reference_kernels(nbp, path):
    g = load(path)
    cfg = nbp.SimConfig(timestep=g["dt"], theta=g["theta"], epsilon_squared=g["eps2"], G=g["G"],
                        mode=nbp.NB_MODE_FP64)
    with nbp.NbContext(cfg, g["mass"], g["pos0"], g["vel0"]) as ctx:
        codes, order, box = ctx.debug_morton()
        assert np.array_equal(box, g["box"])
        assert np.array_equal(codes, g["codes"])
        assert np.array_equal(order, g["perm"])
        acc = ctx.accelerations()
        acc_ref = np.empty_like(g["acc"])
        acc_ref[g["orig"]] = g["acc"]
        assert rel_err(acc, acc_ref).max() < 1e-5
        ctx.step(g["steps"])
        pos, vel = ctx.download()
    assert np.abs(pos - g["pos"]).max() <= 1e-12 * max(1.0, np.abs(g["pos"]).max())
    assert np.abs(vel - g["vel"]).max() <= 1e-8 * max(1.0, np.abs(g["vel"]).max())

"""The C++ adapter (n-body-2d_b200/host/BarnesHutB200.cpp) driven by the
reference's own Simulation base class (oracle/_ref/adapter_demo, built from
the reference sources): the drop-in path a maintainer would wire into
create_sim.  It must give the same bodies as the library driven directly."""
import pathlib
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DEMO = pathlib.Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "adapter_demo"


@pytest.mark.skipif(not DEMO.exists(), reason="adapter_demo is built only where the reference "
                    "sources are mounted (oracle/ref/Makefile)")
@pytest.mark.parametrize("mode", [0, 1])
def test_adapter_matches_library(nbp, mode):
    m, p, v = nbp.universes.exponential_disc(4096, 5)
    steps, theta, dt = 5, 0.5, 1e-4
    with tempfile.TemporaryDirectory() as td:
        fin, fout = pathlib.Path(td) / "in.bin", pathlib.Path(td) / "out.bin"
        with open(fin, "wb") as f:
            np.array([m.shape[0], steps, 1, mode], dtype=np.int64).tofile(f)
            # softening_factor 0.003 of a mean pair distance of about 3: eps ~ 0.01
            np.array([theta, 0.003, dt, 1.0], dtype=np.float64).tofile(f)
            for a in (m, p, v):
                a.astype(np.float64).tofile(f)
        subprocess.run([str(DEMO), str(fin), str(fout)], check=True, timeout=120)
        raw = np.fromfile(fout, dtype=np.float64)
    n = m.shape[0]
    eps2 = raw[1]
    assert 1e-6 < eps2 < 1e-2
    pos, vel = raw[2:2 + 2 * n].reshape(n, 2), raw[2 + 2 * n:].reshape(n, 2)
    # the adapter passes the reference's G (Constants.hpp:17) with the masses
    # the demo scaled by 1 / G; the same inputs to the library directly must
    # give the same bits (every kernel of the step is deterministic)
    g_ref = 6.67430e-11
    cfg = nbp.SimConfig(timestep=dt, theta=theta, epsilon_squared=eps2, G=g_ref, mode=mode)
    with nbp.NbContext(cfg, m * (1.0 / g_ref), p, v) as ctx:
        ctx.step(steps)
        pos_l, vel_l = ctx.download()
    assert np.array_equal(pos, pos_l)
    assert np.array_equal(vel, vel_l)

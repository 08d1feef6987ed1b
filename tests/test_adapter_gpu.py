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
            np.array([theta, 0.0, dt, 1.0], dtype=np.float64).tofile(f)
            for a in (m, p, v):
                a.astype(np.float64).tofile(f)
        subprocess.run([str(DEMO), str(fin), str(fout)], check=True, timeout=120)
        raw = np.fromfile(fout, dtype=np.float64)
    n = m.shape[0]
    pos, vel = raw[1:1 + 2 * n].reshape(n, 2), raw[1 + 2 * n:].reshape(n, 2)
    cfg = nbp.SimConfig(timestep=dt, theta=theta, epsilon_squared=0.0, G=1.0, mode=mode)
    with nbp.NbContext(cfg, m, p, v) as ctx:
        ctx.step(steps)
        pos_l, vel_l = ctx.download()
    # the adapter passes G = 6.6743e-11 with masses scaled by 1/G: rounding only
    assert np.abs(pos - pos_l).max() <= 1e-9 * np.abs(pos_l).max()
    assert np.abs(vel - vel_l).max() <= 1e-6 * np.abs(vel_l).max()

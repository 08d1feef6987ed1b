"""Times the reference's own CUDA kernels (BASELINE INFRASTRUCTURE).

oracle/_ref/ref_gpu_harness runs src/Simulation/src/BarnesHutCuda.cu's kernels
unmodified under its own host driver (see oracle/ref/ref_gpu_harness.cu) and
reports the host-clock time per step of steps 1.., which is the reference's
step cost: its driver synchronises with the host at every tree level.  With
download=True every step also ends as BarnesHutCuda::simulate's does, with the
scatter to original order and the copy of all positions and velocities to the
host (CU:498-506, 632-646); without it that per-step download is left out.  The reference kernel keeps a 32-entry traversal stack (CU:400), so
a case runs only after the CPU oracle has replayed every step and found at
most 28 entries in use; deeper cases are refused, not run.
"""
from __future__ import annotations

import pathlib
import subprocess
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
HARNESS = ROOT / "_ref" / "ref_gpu_harness"
STACK_LIMIT = 28


def available() -> bool:
    return HARNESS.exists()


def max_stack(mass, pos, vel, *, theta, steps, eps2, dt, G) -> int:
    from . import RefState

    st = RefState(mass, pos, vel)
    worst = 0
    for _ in range(steps):
        worst = max(worst, st.step(theta=theta, eps2=eps2, dt=dt, G=G)["stats"]["max_stack"])
        if worst > STACK_LIMIT:
            break  # refused already; later steps cannot lower it
    return worst


def time_steps(mass, pos, vel, *, theta, steps, eps2=1e-4, dt=1e-4, G=1.0,
               download: bool = False) -> dict:
    """Seconds per step of the reference GPU path over `steps` timed steps
    (one more, untimed, runs first), or the reason it was not run."""
    if not available():
        return {"unavailable": "oracle/_ref/ref_gpu_harness was not built"}
    worst = max_stack(mass, pos, vel, theta=theta, steps=steps + 1, eps2=eps2, dt=dt, G=G)
    if worst > STACK_LIMIT:
        return {"unavailable": f"refused: the walk needs {worst} of the kernel's 32 stack entries"}
    n = int(mass.shape[0])
    with tempfile.TemporaryDirectory() as td:
        fin, fout = pathlib.Path(td) / "in.bin", pathlib.Path(td) / "out.bin"
        with open(fin, "wb") as f:
            np.array([n, steps + 1, 1 if download else 0, 0], dtype=np.int64).tofile(f)
            np.array([theta, eps2, dt, G], dtype=np.float64).tofile(f)
            for a in (mass, pos, vel):
                np.ascontiguousarray(a, dtype=np.float64).tofile(f)
        subprocess.run([str(HARNESS), str(fin), str(fout)], check=True, timeout=600)
        hdr = np.fromfile(fout, dtype=np.int64, count=4)
    return {"seconds_per_step": float(hdr[3]) * 1e-9, "max_stack": int(worst)}

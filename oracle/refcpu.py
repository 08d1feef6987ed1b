"""Driver for the reference's CPU Barnes-Hut (oracle/_ref/ref_cpu_bh) --
TEST / BASELINE INFRASTRUCTURE.

The binary is built by oracle/ref/Makefile from the reference sources
(src/Simulation/src/BarnesHut.cpp and its dependencies, unmodified) plus the
harness oracle/ref/ref_cpu_bh.cpp, which runs the backend through its public
Simulation interface (run / is_finished).
"""
from __future__ import annotations

import os
import pathlib
import subprocess
import tempfile

import numpy as np

BIN = pathlib.Path(__file__).resolve().parent / "_ref" / "ref_cpu_bh"


def available() -> bool:
    return BIN.exists()


def run(mass, pos, vel, *, theta: float, steps: int, threads: int | None = None,
        eps2: float = 1e-4, dt: float = 1e-4, G: float = 1.0, warmup: int = 0):
    """Advances the bodies `warmup` untimed then `steps` timed steps with the
    reference CPU backend.  Returns (seconds of the timed steps, pos, vel)."""
    if not BIN.exists():
        raise FileNotFoundError(f"{BIN} not built (oracle/ref/Makefile)")
    n = int(np.asarray(mass).shape[0])
    threads = int(threads or os.cpu_count() or 1)
    threads = max(1, min(threads, n))
    with tempfile.TemporaryDirectory() as td:
        fin, fout = pathlib.Path(td) / "in.bin", pathlib.Path(td) / "out.bin"
        with open(fin, "wb") as f:
            np.array([n, steps, threads, warmup], dtype=np.int64).tofile(f)
            np.array([theta, eps2, dt, G], dtype=np.float64).tofile(f)
            np.ascontiguousarray(mass, dtype=np.float64).tofile(f)
            np.ascontiguousarray(pos, dtype=np.float64).tofile(f)
            np.ascontiguousarray(vel, dtype=np.float64).tofile(f)
        subprocess.run([str(BIN), str(fin), str(fout)], check=True)
        raw = np.fromfile(fout, dtype=np.float64)
    seconds = float(raw[0])
    p = raw[1:1 + 2 * n].reshape(n, 2)
    v = raw[1 + 2 * n:1 + 4 * n].reshape(n, 2)
    return seconds, p, v


def time_steps(mass, pos, vel, *, theta: float, steps: int = 1, threads: int | None = None,
               eps2: float = 1e-4, dt: float = 1e-4, G: float = 1.0, warmup: int = 0) -> float:
    """Seconds per timed step of the reference CPU backend."""
    seconds, _, _ = run(mass, pos, vel, theta=theta, steps=steps, threads=threads, eps2=eps2,
                        dt=dt, G=G, warmup=warmup)
    return seconds / steps

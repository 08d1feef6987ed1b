"""Generates the golden vectors in tests/golden/ from the reference's own CUDA
kernels (oracle/_ref/ref_gpu_harness, built by oracle/ref/Makefile from
src/Simulation/src/BarnesHutCuda.cu).  Run on a GPU host:

    python tests/golden/make_golden.py --out tests/golden

Every case is first replayed by the CPU oracle; a case whose per-body walk
would need more than 28 stack entries is refused before the reference kernel
runs, because the reference keeps a 32-entry stack (CU:400).
"""
from __future__ import annotations

import argparse
import pathlib
import subprocess
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
from conftest import load_package  # noqa: E402

import oracle  # noqa: E402

HARNESS = ROOT / "oracle" / "_ref" / "ref_gpu_harness"
EPS2, DT, G = 1e-4, 1e-4, 1.0
MAX_STACK = 28


def cases():
    nb = load_package()
    u = nb.universes
    rng = np.random.default_rng(2024)
    yield "disc4096_t05", u.exponential_disc(4096, 0), 0.5, 3
    yield "collision4096_t05", u.colliding_discs(4096, 1), 0.5, 2
    yield "collision4096_t10", u.colliding_discs(4096, 1), 1.0, 2
    yield "plummer2048_t07", u.plummer_disc(2048, 2), 0.7, 2
    m, p, v = u.exponential_disc(4000, 3)
    p[10:25] = p[5]      # a 16-body level-30 leaf
    p[40] = p[41]        # and a pair
    yield "coincident4000_t05", (m, p, v), 0.5, 2
    yield "coincident4000_t12", (m, p, v), 1.2, 1
    m = rng.random(1000) + 0.5
    yield "uniform1000_t03", (m, rng.random((1000, 2)) * 10 - 5, rng.normal(size=(1000, 2))), 0.3, 2
    yield "tiny3_t05", (np.array([1.0, 2.0, 3.0]), np.array([[0., 0.], [1., 0.], [0., 1.]]),
                        np.zeros((3, 2))), 0.5, 2


def stack_ok(m, p, v, theta, steps) -> int:
    st = oracle.RefState(m, p, v)
    worst = 0
    for _ in range(steps):
        worst = max(worst, st.step(theta=theta, eps2=EPS2, dt=DT, G=G)["stats"]["max_stack"])
    return worst


def run_harness(m, p, v, theta, steps):
    n = m.shape[0]
    with tempfile.TemporaryDirectory() as td:
        fin, fout = pathlib.Path(td) / "in.bin", pathlib.Path(td) / "out.bin"
        with open(fin, "wb") as f:
            np.array([n, steps, 0, 0], dtype=np.int64).tofile(f)
            np.array([theta, EPS2, DT, G], dtype=np.float64).tofile(f)
            for a in (m, p, v):
                np.ascontiguousarray(a, dtype=np.float64).tofile(f)
        subprocess.run([str(HARNESS), str(fin), str(fout)], check=True)
        raw = fout.read_bytes()
    off = 0

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off).copy()
        off += a.nbytes
        return a

    hdr = take(np.int64, 4)
    return dict(nodes_allocated=hdr[1], levels=hdr[2], box=take(np.float64, 4),
                codes=take(np.uint64, n), perm=take(np.int32, n), orig=take(np.int32, n),
                acc=take(np.float64, 2 * n).reshape(n, 2), pos=take(np.float64, 2 * n).reshape(n, 2),
                vel=take(np.float64, 2 * n).reshape(n, 2))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(ROOT / "tests" / "golden"))
    args = ap.parse_args()
    out = pathlib.Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    for name, (m, p, v), theta, steps in cases():
        worst = stack_ok(m, p, v, theta, steps)
        if worst > MAX_STACK:
            print(f"{name}: refused, oracle walk needs {worst} stack entries")
            continue
        r = run_harness(m, p, v, theta, steps)
        np.savez_compressed(out / f"{name}.npz", mass=m, pos0=p, vel0=v, theta=theta, steps=steps,
                            eps2=EPS2, dt=DT, G=G, max_stack=worst, **r)
        print(f"{name}: n={m.shape[0]} theta={theta} steps={steps} stack={worst} "
              f"nodes={r['nodes_allocated']} levels={r['levels']}")


if __name__ == "__main__":
    main()

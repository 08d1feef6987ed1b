"""ctypes binding of the CPU oracle (oracle/liborc.so) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may use
this module, and only as the checker.  The product library never loads it.
The C sources restate the reference GPU step (src/Simulation/src/
BarnesHutCuda.cu); see nbody_oracle.h for the per-function citations.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "liborc.so"


class Box(C.Structure):
    _fields_ = [("x_min", C.c_double), ("x_max", C.c_double), ("y_min", C.c_double),
                ("y_max", C.c_double)]


class Stats(C.Structure):
    _fields_ = [(name, C.c_int64) for name in (
        "nodes_allocated", "nodes_nonempty", "levels", "max_stack", "cell_interactions",
        "body_interactions", "multi_leaves", "max_level")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_P = C.c_void_p


def build() -> pathlib.Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not LIB.exists() or LIB.stat().st_mtime < (HERE / "nbody_oracle.c").stat().st_mtime:
            build()
        lib = C.CDLL(str(LIB))
        lib.orc_bbox_squared.argtypes = [C.c_int64, _P, C.POINTER(Box)]
        lib.orc_morton.argtypes = [C.c_int64, _P, C.POINTER(Box), _P]
        lib.orc_stable_sort.argtypes = [C.c_int64, _P, _P, _P]
        lib.orc_ref_step.argtypes = [C.c_int64, _P, _P, _P, _P, C.c_double, C.c_double,
                                     C.c_double, C.c_double, C.c_int, _P, _P, _P, C.c_int,
                                     C.POINTER(Stats)]
        lib.orc_ref_step.restype = C.c_int
        lib.orc_ref_walk_targets.argtypes = [C.c_int64, _P, _P, _P, _P, C.c_double, C.c_double,
                                             C.c_int64, _P, _P, _P, _P, _P, C.c_int,
                                             C.POINTER(Stats)]
        lib.orc_ref_walk_targets.restype = C.c_int
        lib.orc_allpairs_plummer.argtypes = [C.c_int64, _P, _P, C.c_int64, _P, C.c_double, _P,
                                             C.c_int]
        lib.orc_allpairs_plummer_abs.argtypes = [C.c_int64, _P, _P, C.c_int64, _P, C.c_double,
                                                 _P, C.c_int]
        lib.orc_allpairs_fp32_bound.argtypes = [C.c_int64, _P, _P, C.c_int64, _P, C.c_double,
                                                C.c_double, C.c_double, _P, C.c_int]
        lib.orc_allpairs_cpulaw.argtypes = [C.c_int64, _P, _P, C.c_int64, _P, C.c_double,
                                            C.c_double, _P, C.c_int]
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _threads(nthreads: int | None) -> int:
    return nthreads if nthreads else (os.cpu_count() or 1)


def bbox_squared(pos: np.ndarray) -> np.ndarray:
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    b = Box()
    load().orc_bbox_squared(pos.shape[0], _p(pos), C.byref(b))
    return np.array([b.x_min, b.x_max, b.y_min, b.y_max])


def morton(pos: np.ndarray, box: np.ndarray | None = None) -> np.ndarray:
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    if box is None:
        box = bbox_squared(pos)
    b = Box(*[float(v) for v in box])
    codes = np.empty(pos.shape[0], dtype=np.uint64)
    load().orc_morton(pos.shape[0], _p(pos), C.byref(b), _p(codes))
    return codes


def stable_sort(keys: np.ndarray):
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    out = np.empty_like(keys)
    order = np.empty(keys.shape[0], dtype=np.int32)
    load().orc_stable_sort(keys.shape[0], _p(keys), _p(out), _p(order))
    return out, order


class RefState:
    """Device-order state of the reference GPU backend, advanced on the CPU."""

    def __init__(self, mass, pos, vel, orig=None):
        self.mass = np.array(mass, dtype=np.float64, order="C")
        self.pos = np.array(pos, dtype=np.float64, order="C").reshape(-1, 2)
        self.vel = np.array(vel, dtype=np.float64, order="C").reshape(-1, 2)
        n = self.mass.shape[0]
        self.orig = (np.arange(n, dtype=np.int32) if orig is None
                     else np.array(orig, dtype=np.int32, order="C"))

    @property
    def n(self) -> int:
        return int(self.mass.shape[0])

    def step(self, G=1.0, dt=1e-4, eps2=1e-4, theta=0.5, integrate=True, want_acc=False,
             want_codes=False, nthreads=None):
        acc = np.empty((self.n, 2)) if want_acc else None
        codes = np.empty(self.n, dtype=np.uint64) if want_codes else None
        order = np.empty(self.n, dtype=np.int32) if want_codes else None
        st = Stats()
        rc = load().orc_ref_step(self.n, _p(self.mass), _p(self.pos), _p(self.vel), _p(self.orig),
                                 G, dt, eps2, theta, 1 if integrate else 0, _p(acc), _p(codes),
                                 _p(order), _threads(nthreads), C.byref(st))
        if rc != 0:
            raise MemoryError("oracle step failed to allocate")
        return dict(acc=acc, codes=codes, order=order, stats=st.as_dict())

    def walk_targets(self, targets, eps2=1e-4, theta=0.5, nthreads=None):
        """Sorts the state as a step does (no integration) and walks only the
        bodies whose original indices are `targets`: per target the FP64
        acceleration, cell terms, body terms and deepest DFS stack."""
        tgt = np.ascontiguousarray(targets, dtype=np.int64)
        k = tgt.shape[0]
        acc = np.empty((k, 2))
        cells = np.empty(k, dtype=np.int64)
        pairs = np.empty(k, dtype=np.int64)
        stack = np.empty(k, dtype=np.int64)
        st = Stats()
        rc = load().orc_ref_walk_targets(self.n, _p(self.mass), _p(self.pos), _p(self.vel),
                                         _p(self.orig), eps2, theta, k, _p(tgt), _p(acc),
                                         _p(cells), _p(pairs), _p(stack), _threads(nthreads),
                                         C.byref(st))
        if rc == -2:
            raise IndexError("target index outside [0, n)")
        if rc != 0:
            raise MemoryError("oracle walk failed to allocate")
        return dict(acc=acc, cells=cells, pairs=pairs, stack=stack, stats=st.as_dict())

    def original_order(self):
        """(pos, vel, acc-permutation) mapped back to original body order."""
        inv = np.empty(self.n, dtype=np.int64)
        inv[self.orig] = np.arange(self.n)
        return inv

    def in_original_order(self, arr: np.ndarray) -> np.ndarray:
        out = np.empty_like(arr)
        out[self.orig] = arr
        return out


def allpairs_plummer(mass, pos, targets=None, eps2=1e-4, nthreads=None) -> np.ndarray:
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n = mass.shape[0]
    tgt = np.ascontiguousarray(np.arange(n) if targets is None else targets, dtype=np.int64)
    acc = np.empty((tgt.shape[0], 2))
    load().orc_allpairs_plummer(n, _p(mass), _p(pos), tgt.shape[0], _p(tgt), eps2, _p(acc),
                                _threads(nthreads))
    return acc


def allpairs_plummer_abs(mass, pos, targets=None, eps2=1e-4, nthreads=None) -> np.ndarray:
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n = mass.shape[0]
    tgt = np.ascontiguousarray(np.arange(n) if targets is None else targets, dtype=np.int64)
    out = np.empty(tgt.shape[0])
    load().orc_allpairs_plummer_abs(n, _p(mass), _p(pos), tgt.shape[0], _p(tgt), eps2, _p(out),
                                    _threads(nthreads))
    return out


def allpairs_fp32_bound(mass, pos, center, targets=None, eps2=1e-4, nthreads=None) -> np.ndarray:
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n = mass.shape[0]
    tgt = np.ascontiguousarray(np.arange(n) if targets is None else targets, dtype=np.int64)
    out = np.empty(tgt.shape[0])
    load().orc_allpairs_fp32_bound(n, _p(mass), _p(pos), tgt.shape[0], _p(tgt), eps2,
                                   float(center[0]), float(center[1]), _p(out), _threads(nthreads))
    return out


def allpairs_cpulaw(mass, pos, targets=None, G=1.0, eps2=1e-4, nthreads=None) -> np.ndarray:
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    n = mass.shape[0]
    tgt = np.ascontiguousarray(np.arange(n) if targets is None else targets, dtype=np.int64)
    acc = np.empty((tgt.shape[0], 2))
    load().orc_allpairs_cpulaw(n, _p(mass), _p(pos), tgt.shape[0], _p(tgt), G, eps2, _p(acc),
                               _threads(nthreads))
    return acc

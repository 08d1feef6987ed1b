"""Universe files in the reference's CSV format.

IO::parse_csv / IO::write_csv (src/common_lib/InputOutput/src/
InputOutput.cpp:18-72): a header row, then one body per row with the
columns id, mass, x, y, vel_x, vel_y.  Ids must be unique, as
Bodies::validate requires (src/common_lib/Body/src/Body.cpp:21-32, 99-115).
Numbers are written in the shortest form that reads back to the same double,
without a trailing ".0", as fmt's "{}" writes them.
"""
from __future__ import annotations

import csv

import numpy as np

from .simulation import Bodies

HEADER = ["id", "mass", "x", "y", "vel_x", "vel_y"]


def format_double(v: float) -> str:
    r = repr(float(v))
    return r[:-2] if r.endswith(".0") else r


def read_csv(path) -> Bodies:
    ids, mass, pos, vel = [], [], [], []
    with open(path, newline="") as f:
        rows = csv.reader(f)
        next(rows, None)  # header row
        for lineno, row in enumerate(rows, start=2):
            if not row:
                continue
            if len(row) < 6:
                raise ValueError(f"{path}:{lineno}: expected 6 columns, got {len(row)}")
            ids.append(row[0])
            mass.append(float(row[1]))
            pos.append((float(row[2]), float(row[3])))
            vel.append((float(row[4]), float(row[5])))
    if len(set(ids)) != len(ids):
        seen, dup = set(), None
        for i in ids:
            if i in seen:
                dup = i
                break
            seen.add(i)
        raise ValueError(f"{path}: duplicate body id {dup!r}")
    n = len(ids)
    return Bodies(np.asarray(mass, dtype=np.float64).reshape(n),
                  np.asarray(pos, dtype=np.float64).reshape(n, 2),
                  np.asarray(vel, dtype=np.float64).reshape(n, 2), ids=ids)


def write_csv(path, bodies: Bodies) -> None:
    with open(path, "w", newline="") as f:
        f.write(",".join(HEADER) + "\n")
        for i in range(bodies.n):
            f.write(",".join([bodies.ids[i], format_double(bodies.mass[i]),
                              format_double(bodies.pos[i, 0]), format_double(bodies.pos[i, 1]),
                              format_double(bodies.vel[i, 0]), format_double(bodies.vel[i, 1])])
                    + "\n")

"""Grid metrics of the reference's `grid` routine (src/core/setup.F90:92-247).

Single rank (n_global_min = 0, mpi_routines.F90:282-289), no stretching.
Returns the Fortran-bounded 1-D arrays the hot path reads, as plain numpy
arrays starting at their lower bound: xb(-2:n+2), xc(-1:n+2), dxb(-1:n+2),
dxc(-1:n+1), and likewise for y and z.
"""
from __future__ import annotations

import numpy as np

from .abi import BC_PERIODIC


def axis(n: int, vmin: float, vmax: float, bc_max: int):
    length = vmax - vmin                              # setup.F90:97
    d = length / float(n)                             # :102
    b = np.empty(n + 5, dtype=np.float64)             # xb_global(-2:n+2)
    off = 2
    for i in range(-2, n + 3):                        # :106-108
        b[i + off] = vmin + float(i) * d
    B = lambda i: b[i + off]
    if bc_max == BC_PERIODIC:                         # :113-121
        b[n + 1 + off] = B(n) + (B(1) - B(0))
        b[n + 2 + off] = B(n) + (B(2) - B(0))
        b[-1 + off] = B(0) - (B(n) - B(n - 1))
        b[-2 + off] = B(0) - (B(n) - B(n - 2))
    else:                                             # :122-129
        b[n + 1 + off] = 2.0 * B(n) - B(n - 1)
        b[n + 2 + off] = 2.0 * B(n) - B(n - 2)
        b[-1 + off] = 2.0 * B(0) - B(1)
        b[-2 + off] = 2.0 * B(0) - B(2)
    xb = b.copy()                                     # :133-138
    xc = np.empty(n + 4)                              # xc(-1:n+2)
    db = np.empty(n + 4)                              # dxb(-1:n+2)
    for i in range(-1, n + 3):
        xc[i + 1] = 0.5 * (xb[i - 1 + off] + xb[i + off])
        db[i + 1] = xb[i + off] - xb[i - 1 + off]
    dc = np.empty(n + 3)                              # dxc(-1:n+1)
    for i in range(-1, n + 2):                        # :149-153
        dc[i + 1] = xc[i + 2] - xc[i + 1]
    return {"b": xb, "c": xc, "db": db, "dc": dc}


def grid(nx, ny, nz, x=(0.0, 1.0), y=(0.0, 1.0), z=(0.0, 1.0), bcs=(BC_PERIODIC,) * 3):
    """Metrics for a uniform grid; bcs gives the *_bc_max code per axis."""
    ax = axis(nx, x[0], x[1], bcs[0])
    ay = axis(ny, y[0], y[1], bcs[1])
    az = axis(nz, z[0], z[1], bcs[2])
    return {
        "xb": ax["b"], "xc": ax["c"], "dxb": ax["db"], "dxc": ax["dc"],
        "yb": ay["b"], "yc": ay["c"], "dyb": ay["db"], "dyc": ay["dc"],
        "zb": az["b"], "zc": az["c"], "dzb": az["db"], "dzc": az["dc"],
    }

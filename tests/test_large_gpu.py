"""GPU parity above the benchmark's size, on a ragged grid.

The resistive Orszag-Tang workload (the fields of decks.orszag_tang: rho0,
p0, v = (-sin z, sin x, sin y), B = (-sin z, sin 2x, sin y) / sqrt(4 pi),
eta = 1e-3) on a 384 x 320 x 200 periodic box of side 2 pi: 24.6 M cells,
1.5 times the 256^3 benchmark grid, with every edge a different multiple of
the kernels' tiles and chunks.  Three steps through the oracle and the three
engines:

* the exact engine equals the oracle bit for bit (every state field);
* the FP64 product engine is within 1e-10 relative L2 per field, the FP32
  form within 1e-5;
* mass is conserved to 1e-12 (the remap is conservative on a periodic box,
  xremap.f90:174-182) and div B stays at round-off (constrained transport)
  on every engine.
"""
import math

import numpy as np
import pytest

from conftest import STATE, rel_l2
from lare3d_b200 import decks
from lare3d_b200.abi import State, default_params
from lare3d_b200.grid import grid

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

NX, NY, NZ = 384, 320, 200
STEPS = 3


def ragged_orszag_tang():
    g = 5.0 / 3.0
    p = default_params(gamma=g, visc1=0.1, visc2=0.5, dt_multiplier=0.8,
                       resistive_mhd=1, eta_background=1.0e-3, eta0=0.0, j_max=1.0e10)
    L = 2.0 * math.pi
    m = grid(NX, NY, NZ, (0.0, L), (0.0, L), (0.0, L))
    st = State.zeros(NX, NY, NZ)
    rho0 = 25.0 / (36.0 * math.pi)
    p0 = 5.0 / (12.0 * math.pi)
    st["rho"][...] = rho0
    st["energy"][...] = p0 / ((g - 1.0) * rho0)
    st["vx"][...] = (-np.sin(m["zb"]))[None, None, :]
    st["vy"][...] = np.sin(m["xb"])[:, None, None]
    st["vz"][...] = np.sin(m["yb"])[None, :, None]
    s4 = 1.0 / math.sqrt(4.0 * math.pi)
    st["bx"][...] = (-np.sin(m["zc"]) * s4)[None, None, :]
    st["by"][...] = (np.sin(2.0 * m["xc"]) * s4)[:, None, None]
    st["bz"][...] = (np.sin(m["yc"]) * s4)[None, :, None]
    return decks.Deck("orszag_tang_ragged", p, NX, NY, NZ, m, st, nsteps=STEPS)


def mass(st, m):
    cv = (m["dxb"][2:NX + 2][:, None, None] * m["dyb"][2:NY + 2][None, :, None]
          * m["dzb"][2:NZ + 2][None, None, :])
    return math.fsum((st["rho"][2:NX + 2, 2:NY + 2, 2:NZ + 2] * cv).ravel())


def div_b_scaled(st, m):
    """max |div B| over cells 1..n, times the cell width, over max |B|."""
    bx, by, bz = st["bx"], st["by"], st["bz"]
    dxb = m["dxb"][2:NX + 2][:, None, None]
    dyb = m["dyb"][2:NY + 2][None, :, None]
    dzb = m["dzb"][2:NZ + 2][None, None, :]
    # bx(i) at array index i + 2 along x, cells at index + 1 along y and z
    d = (bx[3:NX + 3, 2:NY + 2, 2:NZ + 2] - bx[2:NX + 2, 2:NY + 2, 2:NZ + 2]) / dxb
    d += (by[2:NX + 2, 3:NY + 3, 2:NZ + 2] - by[2:NX + 2, 2:NY + 2, 2:NZ + 2]) / dyb
    d += (bz[2:NX + 2, 2:NY + 2, 3:NZ + 3] - bz[2:NX + 2, 2:NY + 2, 2:NZ + 2]) / dzb
    bmax = max(float(np.abs(bx).max()), float(np.abs(by).max()), float(np.abs(bz).max()))
    return float(np.abs(d).max()) * float(m["dxb"][2]) / bmax


def test_ragged_orszag_tang_above_benchmark_size(built):
    from lare3d_b200 import gpu
    from oracle import oracle
    d = ragged_orszag_tang()
    m0 = mass(d.state, d.metrics)
    r = oracle.simulation(d)
    r.start(d.state)
    for s in range(1, STEPS + 1):
        r.step(s)
    ref = r.download()
    r.close()
    assert abs(mass(ref, d.metrics) / m0 - 1.0) <= 1e-12
    assert div_b_scaled(ref, d.metrics) < 1e-12
    for precision, tol in ((gpu.EXACT64, 0.0), (gpu.FP64, 1e-10), (gpu.FP32, 1e-5)):
        g = gpu.simulation(d, precision=precision)
        g.start(d.state)
        for s in range(1, STEPS + 1):
            g.step(s)
        got = g.download()
        g.close()
        for f in STATE:
            if tol == 0.0:
                nbad = int(np.count_nonzero(got[f] != ref[f]))
                assert nbad == 0, f"{f}: the exact engine differs from the oracle in {nbad} elements"
            else:
                err = rel_l2(got[f], ref[f])
                print(f"{precision} {f} {err:.3e}")
                assert err <= tol, (precision, f, err)
        if precision != gpu.FP32:
            assert abs(mass(got, d.metrics) / m0 - 1.0) <= 1e-12
            assert div_b_scaled(got, d.metrics) < 1e-12
        else:
            assert abs(mass(got, d.metrics) / m0 - 1.0) <= 1e-6
            assert div_b_scaled(got, d.metrics) < 1e-5

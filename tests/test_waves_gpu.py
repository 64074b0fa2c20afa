"""The linear sound, Alfven and fast waves of tests/test_waves_cpu.py (and Sod's
shock tube of tests/test_shock_tube_cpu.py and the heat wave of
tests/test_heat_wave_cpu.py) through
the three GPU engines, along each axis: the exact engine bit for bit with
the oracle, the FP64 product engine within 1e-10 of it (L2 norm of the
difference of every state field over that of the field or, for fields that
carry only the perturbation or its second-order flows, of a field of the
perturbation's amplitude), and each engine's wave at its analytic speed
within 0.1 % (0.2 % and an amplitude within 0.5 % in FP32, whose rounding is
6e-8 of the background against a perturbation of 1e-4).  Shapes of
64 x 4 x 4 and its rotations exercise the kernels' partial tiles and chunks
on every axis."""
import math

import numpy as np
import pytest

from conftest import STATE
from test_waves_cpu import EPS, measured_mode, run_to_end, wave_deck

pytestmark = pytest.mark.gpu


def scaled_l2(a, b):
    """||a - b|| over max(||b||, ||EPS||): relative for the background
    fields, relative to the perturbation's scale for the perturbation-only
    ones (whose second-order parts are round-off-sized in relative terms)."""
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), EPS * math.sqrt(b.size)))


@pytest.mark.parametrize("kind", ["sound", "alfven", "fast"])
@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_wave_through_engines(built, kind, axis):
    from lare3d_b200 import gpu
    from oracle import oracle
    d, speed, probe, base = wave_deck(kind, axis)
    r = oracle.simulation(d)
    r.start(d.state)
    t_ref = run_to_end(r)
    for precision, tol in ((gpu.EXACT64, 0.0), (gpu.FP64, 1e-10), (gpu.FP32, None)):
        d, _, _, _ = wave_deck(kind, axis)
        g = gpu.simulation(d, precision=precision)
        g.start(d.state)
        t = run_to_end(g)
        assert abs(t - t_ref) <= (1e-12 if precision != gpu.FP32 else 1e-5) * t_ref
        for f in STATE if tol is not None else ():
            a, b = g.get_field(f), r.get_field(f)
            if tol == 0.0:
                assert np.array_equal(a, b), f"{kind} {axis} {f}: exact engine differs from the oracle"
            else:
                err = scaled_l2(a, b)
                assert err <= tol, (kind, axis, precision, f, err)
        phi, amp = measured_mode(g, d, axis, probe, base)
        bar = 1e-3 if precision != gpu.FP32 else 2e-3
        assert abs(phi / (2.0 * math.pi * t) / speed - 1.0) < bar, (precision, phi, t, speed)
        lo, hi = (0.99, 1.001) if precision != gpu.FP32 else (0.98, 1.005)
        assert lo * EPS < amp <= hi * EPS, (precision, amp)
        g.close()


@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_diffusion_through_engines(built, axis):
    """The resistive and conductive modes of tests/test_diffusion_cpu.py: the
    exact engine bit for bit with the oracle, the product engine within
    1e-10 and at the analytic decay rate within 0.2 %."""
    from lare3d_b200 import gpu
    from oracle import oracle
    from test_diffusion_cpu import DT_COND, EPS as E, GAMMA, T0, conduction_deck, mode, resistive_deck, run_resistive
    for case in ("resistive", "conduction"):
        d, lam = (resistive_deck(axis)[:2] if case == "resistive" else conduction_deck(axis))
        r = oracle.simulation(d)
        r.start(d.state)
        if case == "resistive":
            run_resistive(r)
        else:
            r.conduct_heat(DT_COND)
        for precision, tol in ((gpu.EXACT64, 0.0), (gpu.FP64, 1e-10)):
            d = (resistive_deck(axis)[0] if case == "resistive" else conduction_deck(axis)[0])
            g = gpu.simulation(d, precision=precision)
            g.start(d.state)
            if case == "resistive":
                t = run_resistive(g)
                name, base, a0 = "bx by bz".split()[(axis + 1) % 3], 0.0, E
            else:
                g.conduct_heat(DT_COND)
                t = DT_COND
                name, base, a0 = "energy", 2.0 * T0 / (GAMMA - 1.0), 2.0 * T0 * E / (GAMMA - 1.0)
            for f in STATE:
                a, b = g.get_field(f), r.get_field(f)
                if tol == 0.0:
                    assert np.array_equal(a, b), f"{case} {axis} {f}: exact engine differs from the oracle"
                else:
                    assert scaled_l2(a, b) <= tol, (case, axis, f, scaled_l2(a, b))
            _, amp = mode(g, d, axis, name, base)
            assert abs(-math.log(amp / a0) / t / lam - 1.0) < 2e-3, (case, precision)
            g.close()


@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_shock_tube_through_engines(built, axis):
    """Sod's tube of tests/test_shock_tube_cpu.py, shock viscosity on: the
    exact engine bit for bit with the oracle, the product engine within
    1e-10, and every engine within the exact Riemann solution's bars."""
    from lare3d_b200 import gpu
    from oracle import oracle
    from test_shock_tube_cpu import L1_BAR, N, PLATEAU_BAR, SHOCK_BAR, run_tube, tube_deck, tube_errors, tube_profile
    d = tube_deck(axis)
    r = oracle.simulation(d)
    r.start(d.state)
    t_ref = run_tube(r)
    x = d.metrics["xyz"[axis] + "c"][2:2 + N]
    for precision, tol in ((gpu.EXACT64, 0.0), (gpu.FP64, 1e-10), (gpu.FP32, None)):
        d = tube_deck(axis)
        g = gpu.simulation(d, precision=precision)
        g.start(d.state)
        t = run_tube(g)
        assert abs(t - t_ref) <= (1e-12 if precision != gpu.FP32 else 1e-5) * t_ref
        for f in STATE if tol is not None else ():
            a, b = g.get_field(f), r.get_field(f)
            if tol == 0.0:
                assert np.array_equal(a, b), f"sod {axis} {f}: exact engine differs from the oracle"
            else:
                assert scaled_l2(a, b) <= tol, (axis, f, scaled_l2(a, b))
        l1, dxs, dplat = tube_errors(tube_profile(g.get_field("rho"), axis), x, t)
        assert l1 < L1_BAR and abs(dxs) < SHOCK_BAR / N and dplat < PLATEAU_BAR, (precision, l1, dxs * N, dplat)
        g.close()


@pytest.mark.parametrize("axis", [0, 1, 2], ids=["x", "y", "z"])
def test_heat_wave_through_engines(built, axis):
    """The Zel'dovich heat wave of tests/test_heat_wave_cpu.py: the FP64
    engines within 1e-12 (exact; T^2.5 is formed as T*T*sqrt(T), not by pow)
    and 1e-10 (product) of the oracle, every engine within the similarity
    solution's bars."""
    from lare3d_b200 import gpu
    from oracle import oracle
    from test_heat_wave_cpu import NW, advance, heat_wave_deck, wave_errors, wave_profile
    d = heat_wave_deck(axis)
    r = oracle.simulation(d)
    r.start(d.state)
    advance(r)
    ref = r.get_field("energy")
    x = d.metrics["xyz"[axis] + "c"][2:2 + NW]
    for precision, tol in ((gpu.EXACT64, 1e-12), (gpu.FP64, 1e-10), (gpu.FP32, None)):
        d = heat_wave_deck(axis)
        g = gpu.simulation(d, precision=precision)
        g.start(d.state)
        advance(g)
        energy = g.get_field("energy")
        if tol is not None:
            assert scaled_l2(energy, ref) <= tol, (precision, scaled_l2(energy, ref))
        dtc, l1, fronts = wave_errors(x, wave_profile(energy, axis))
        assert dtc < 5e-3 and l1 < 3e-3 and max(abs(f) for f in fronts) < 1.0, (precision, dtc, l1, fronts)
        g.close()

"""GPU parity on the three plain-method workloads at sizes near the benchmark's.

* blast 64^3, 100 steps at CFL 0.8 (the CPU-runnable workload at its size);
* resistive Orszag-Tang at 128^3, 100 steps (the 256^3 benchmark workload at
  half the edge, so that the oracle finishes in about a minute);
* RKL2 conduction at 128^3 (sheared arcade with hot spots), two substeps.

Each oracle run is made once and compared with every engine:

* FP64 product engine (LARE_FP64: FMA contraction, shared reciprocals):
  relative L2 <= 1e-10 per field after the run, energy budgets within 1e-10;
* FP64 exact engine (LARE_FP64_EXACT): bit for bit (conduction, whose T^2.5
  is formed differently from the reference's pow, at relative L2 1e-12);
* energy budgets: the oracle sums in the reference's serial order, whose own
  rounding error over 10^6 - 10^7 positive terms reaches 1e-12 - 1e-11
  relative, while the engines sum in a tree; so both are compared with the
  exactly rounded sum (math.fsum) of the same FP64 products for the internal
  energy: the engines within 1e-13, the oracle within 1e-10; the three
  budgets of engine and oracle agree within 1e-10, and so does the drift of
  the total energy over the run;
* FP32 form: relative L2 <= 1e-5 per field against the FP64 oracle.

div B stays at round-off on every engine: max |div B| * dx / max |B| < 1e-12.
The measured errors are printed (pytest -s shows them).
"""
import math

import numpy as np
import pytest

from conftest import STATE, rel_l2
from lare3d_b200 import decks

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

CASES = {
    "blast64": (lambda: decks.blast(64), 100),
    "orszag_tang128": (lambda: decks.orszag_tang(128), 100),
    "conduction128": (lambda: decks.conduction(128), 2),
}
_cache = {}


def _advance(sim, d, nsteps):
    """nsteps timesteps, or nsteps conduct_heat substeps of the conduction
    workload's fixed dt; returns the RKL2 stage counts of the substeps."""
    stages = []
    for s in range(1, nsteps + 1):
        if d.dt_fixed is not None:
            stages.append(sim.conduct_heat(d.dt_fixed))
        else:
            sim.step(s)
    return stages


def _run(sim, d, nsteps):
    sim.start(d.state)
    e0 = sim.energy()
    stages = _advance(sim, d, nsteps)
    out = {"fields": sim.download(), "energy0": e0, "energy": sim.energy(), "stages": stages}
    sim.close()
    return out


def oracle_run(case):
    if case not in _cache:
        from oracle import oracle
        make, nsteps = CASES[case]
        d = make()
        _cache[case] = (d, _run(oracle.simulation(d), d, nsteps))
    return _cache[case]


def gpu_run(case, precision):
    from lare3d_b200 import gpu
    d, _ = oracle_run(case)
    return _run(gpu.simulation(d, precision=precision), d, CASES[case][1])


def div_b_scaled(st, d):
    from test_oracle_cpu import div_b
    n = d.nx
    dx = float(np.min(d.metrics["dxb"][2:n + 2]))
    bmax = max(float(np.abs(st[k]).max()) for k in ("bx", "by", "bz"))
    return float(np.abs(div_b(st, d.metrics, n)).max()) * dx / bmax


def en_int_exact(st, d):
    """diagnostics.F90:536-556's internal energy, sum of energy*rho*cv over
    cells 1..n with cv = dxb*dyb*dzb (setup.F90:239-245), every product
    rounded in FP64 as the reference forms it and the sum exactly rounded."""
    n = d.nx
    m = d.metrics
    cv = (m["dxb"][2:n + 2][:, None, None] * m["dyb"][2:n + 2][None, :, None]) * m["dzb"][2:n + 2][None, None, :]
    e = st["energy"][2:n + 2, 2:n + 2, 2:n + 2]
    r = st["rho"][2:n + 2, 2:n + 2, 2:n + 2]
    return math.fsum(((e * r) * cv).ravel())


def _fields(case):
    return ["energy"] if oracle_run(case)[0].dt_fixed is not None else STATE


def _report(case, name, errs, extra=""):
    worst = max(errs.values())
    print(f"\n{case} {name}: worst relative L2 {worst:.3e} "
          + " ".join(f"{f}={e:.2e}" for f, e in errs.items()) + extra)


@pytest.mark.parametrize("case", list(CASES))
def test_fp64_product_engine(built, case):
    from lare3d_b200 import gpu
    d, ref = oracle_run(case)
    got = gpu_run(case, gpu.FP64)
    errs = {f: rel_l2(got["fields"][f], ref["fields"][f]) for f in _fields(case)}
    de = max(abs(a - b) / max(abs(b), 1e-300) for a, b in zip(got["energy"][:3], ref["energy"][:3]))
    db = div_b_scaled(got["fields"], d)
    _report(case, "FP64 product", errs, f" energy {de:.2e} divB {db:.2e}")
    assert got["stages"] == ref["stages"]
    for f, e in errs.items():
        assert e <= 1e-10, (f, e)
    assert de <= 1e-10
    assert db < 1e-12


@pytest.mark.parametrize("case", list(CASES))
def test_fp64_exact_engine(built, case):
    from lare3d_b200 import gpu
    d, ref = oracle_run(case)
    got = gpu_run(case, gpu.EXACT64)
    errs = {f: rel_l2(got["fields"][f], ref["fields"][f]) for f in _fields(case)}
    de = max(abs(a - b) / max(abs(b), 1e-300) for a, b in zip(got["energy"][:3], ref["energy"][:3]))
    exact = en_int_exact(got["fields"], d)
    eg = abs(got["energy"][2] - exact) / exact
    eo = abs(ref["energy"][2] - en_int_exact(ref["fields"], d)) / exact
    drift = sum(got["energy"][:3]) - sum(got["energy0"][:3])
    drift_ref = sum(ref["energy"][:3]) - sum(ref["energy0"][:3])
    dd = abs(drift - drift_ref) / abs(sum(ref["energy0"][:3]))
    _report(case, "FP64 exact", errs, f" budgets {de:.2e} en_int vs exact sum: engine {eg:.1e} oracle {eo:.1e}"
                                      f" drift {dd:.1e}")
    assert got["stages"] == ref["stages"]
    if d.dt_fixed is not None:
        for f, e in errs.items():
            assert e <= 1e-12, (f, e)
    else:
        for f in STATE:
            assert np.array_equal(got["fields"][f], ref["fields"][f]), f
    assert eg <= 1e-13 and eo <= 1e-10
    assert de <= 1e-10
    # total-energy drift over the run equals the oracle's
    assert dd <= 1e-10


@pytest.mark.parametrize("case", list(CASES))
def test_fp32_form(built, case):
    from lare3d_b200 import gpu
    d, ref = oracle_run(case)
    got = gpu_run(case, gpu.FP32)
    errs = {f: rel_l2(got["fields"][f], ref["fields"][f]) for f in _fields(case)}
    db = div_b_scaled(got["fields"], d)
    _report(case, "FP32", errs, f" divB {db:.2e}")
    assert got["stages"] == ref["stages"]
    for f, e in errs.items():
        assert e <= 1e-5, (f, e)

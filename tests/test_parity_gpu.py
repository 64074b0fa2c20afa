"""GPU parity: the sm_100a engine against the oracle, through the C ABI.

The exact FP64 engine (LARE_FP64_EXACT) is built without FMA contraction and
keeps the reference's loop ranges and expression order, so every routine of
the MHD step must agree with the oracle BIT FOR BIT (tolerance 0).  The
product FP64 engine (LARE_FP64) is held to relative L2 1e-10 per field after
100 steps (tests/test_configs_gpu.py).  Conduction calls pow(),
whose last bit may differ between CUDA and glibc; its tolerance is a
relative L2 of 1e-12.  The FP32 form is compared with the FP64 oracle at the
1e-5 relative-L2 bar.
"""
import numpy as np
import pytest

from conftest import STATE, rel_l2
from lare3d_b200 import decks
from lare3d_b200.abi import BC_USER, LareError

pytestmark = pytest.mark.gpu

INTERMEDIATE = ["p_visc", "visc_heat", "alpha1", "alpha2", "alpha3", "pressure", "vx1", "vy1", "vz1",
                "visc_dep", "cv1", "rho_v", "cv_v", "fx_visc", "fy_visc", "fz_visc", "eta", "ohmic_dep"]


def pair(deck, precision=None):
    from lare3d_b200 import gpu
    from oracle import oracle
    r = oracle.simulation(deck)
    g = gpu.simulation(deck, precision=gpu.EXACT64 if precision is None else precision)
    r.start(deck.state)
    g.start(deck.state)
    return r, g


def assert_bitwise(g, r, names, tag):
    for f in names:
        a, b = g.get_field(f), r.get_field(f)
        nbad = int(np.count_nonzero(a != b))
        assert nbad == 0, f"{tag}: {f} differs in {nbad} elements (max |d| {np.abs(a - b).max():.3e})"


CASES = [
    ("blast", dict(n=16)),
    ("orszag_tang", dict(n=16)),
    ("orszag_tang", dict(n=12, eta0=2.0e-3, j_max=0.5)),          # anomalous resistivity switch
    ("blast", dict(n=12, xbc_min=BC_USER, xbc_max=BC_USER)),       # BC_USER mirrors in x
    ("blast", dict(n=12, zbc_min=BC_USER, zbc_max=BC_USER, ybc_min=BC_USER, ybc_max=BC_USER)),
    ("blast", dict(n=10, use_viscous_damping=1)),
]


@pytest.mark.parametrize("name,kw", CASES)
def test_routines_bitwise(built, name, kw):
    kw = dict(kw)
    n = kw.pop("n")
    d = getattr(decks, name)(n, **kw)
    if kw.get("use_viscous_damping"):
        from lare3d_b200.abi import alloc
        v3 = alloc("node", n, n, n, 1e-3)
        r, g = pair(d)
        r.upload_aux(visc3=v3)
        g.upload_aux(visc3=v3)
    else:
        r, g = pair(d)
    assert_bitwise(g, r, STATE + ["eta"], "init")
    for st in range(1, 7):
        r.lagrangian_step(st)
        g.lagrangian_step(st)
        assert_bitwise(g, r, STATE + INTERMEDIATE, f"lagrangian_step {st}")
        r.eulerian_remap(st)
        g.eulerian_remap(st)
        # cv1 after the remap is scratch (vertex averages in the reference)
        assert_bitwise(g, r, STATE, f"eulerian_remap {st}")
        r.eta_calc()
        g.eta_calc()
        assert_bitwise(g, r, ["eta"], f"eta_calc {st}")
    sr, sg = r.scalars(), g.scalars()
    assert sr.time == sg.time and sr.dt == sg.dt and sr.dtr == sg.dtr
    assert sr.last_substeps == sg.last_substeps


def test_ragged_grid_bitwise(built):
    """Unequal nx, ny, nz exercise every axis-specific loop range."""
    d = decks.blast(12)
    from lare3d_b200.abi import State
    from lare3d_b200.grid import grid
    nx, ny, nz = 14, 10, 12
    m = grid(nx, ny, nz, (0, 1.4), (0, 1.0), (0, 1.2))
    st = State.zeros(nx, ny, nz)
    rng = np.random.default_rng(3)
    for k in STATE:
        st[k][...] = rng.uniform(0.5, 1.5, st[k].shape) if k in ("rho", "energy") else rng.uniform(-0.3, 0.3, st[k].shape)
    d2 = decks.Deck("ragged", d.params, nx, ny, nz, m, st, nsteps=6)
    r, g = pair(d2)
    for s in range(1, 7):
        r.step(s)
        g.step(s)
        assert_bitwise(g, r, STATE, f"step {s}")


def _ragged_resistive_deck(nx, ny, nz, seed):
    from lare3d_b200.abi import State
    from lare3d_b200.grid import grid
    d = decks.orszag_tang(8, j_max=10.0, eta0=1.0e-3)
    m = grid(nx, ny, nz, (0, 1.1), (0, 0.9), (0, 1.6))
    st = State.zeros(nx, ny, nz)
    rng = np.random.default_rng(seed)
    for k in STATE:
        st[k][...] = rng.uniform(0.5, 1.5, st[k].shape) if k in ("rho", "energy") else rng.uniform(-0.3, 0.3, st[k].shape)
    return decks.Deck("ragged-resistive", d.params, nx, ny, nz, m, st, nsteps=3)


def test_partial_chunks_bitwise(built):
    """Edges that are not multiples of any kernel's chunk (32 and 64 planes
    marched per thread, 29 and 31 outputs per warp, 4 planes per thread),
    with the resistive path on and j_max inside the current range, so both
    eta branches occur: every routine bit for bit."""
    d = _ragged_resistive_deck(45, 38, 67, 11)
    r, g = pair(d)
    for s in range(1, 4):
        r.lagrangian_step(s)
        g.lagrangian_step(s)
        assert_bitwise(g, r, STATE + INTERMEDIATE, f"lagrangian_step {s}")
        r.eulerian_remap(s)
        g.eulerian_remap(s)
        assert_bitwise(g, r, STATE, f"eulerian_remap {s}")
        r.eta_calc()
        g.eta_calc()
        assert_bitwise(g, r, ["eta"], f"eta_calc {s}")
    eta = g.get_field("eta")
    assert (eta > 1.5e-3).any() and (eta < 1.5e-3).any()


def test_partial_chunks_fp32(built):
    """The FP32 form on the same grid (its own kernel choices and planes per
    thread) against the FP64 oracle at the 1e-5 bar."""
    d = _ragged_resistive_deck(45, 38, 67, 12)
    from lare3d_b200 import gpu
    from oracle import oracle
    r = oracle.simulation(d)
    g = gpu.simulation(d, precision=32)
    r.start(d.state)
    g.start(d.state)
    for s in range(1, 4):
        r.step(s)
        g.step(s)
    for f in STATE:
        e = rel_l2(g.get_field(f), r.get_field(f))
        assert e <= 1e-5, f"{f}: rel L2 {e:.2e}"


@pytest.mark.parametrize("b", [(2 ** -0.5, 2 ** -0.5, 0.0), (1.0, 0.0, 0.0)])
def test_open_boundaries_bitwise(built, b):
    """Open (characteristic) boundaries on the x and y sides, both solver
    branches (a field along x sends the x faces to the Alfven-mode one):
    every routine bit for bit, ghosts included."""
    d = decks.open_blast(16, b=b)
    r, g = pair(d)
    for s in range(1, 5):
        r.lagrangian_step(s)
        g.lagrangian_step(s)
        assert_bitwise(g, r, STATE + INTERMEDIATE, f"lagrangian_step {s}")
        r.eulerian_remap(s)
        g.eulerian_remap(s)
        assert_bitwise(g, r, STATE, f"eulerian_remap {s}")
        r.eta_calc()
        g.eta_calc()


@pytest.mark.parametrize("resistive", [0, 1])
def test_open_user_periodic_ragged_bitwise(built, resistive):
    """Open x sides, open y min against a BC_USER y max, periodic z, on a
    ragged grid with a weakly perturbed state whose ghosts (the far field of
    the open sides) are random too, with and without the resistive step."""
    from lare3d_b200.abi import BC_OPEN, BC_PERIODIC, State
    from lare3d_b200.grid import grid
    nx, ny, nz = 20, 18, 14
    d0 = decks.open_blast(8, ybc_max=BC_USER, zbc_min=BC_PERIODIC, zbc_max=BC_PERIODIC, resistive_mhd=resistive,
                          eta_background=1.0e-3, eta0=1.0e-3, j_max=1.0)
    assert d0.params.xbc_min == BC_OPEN
    m = grid(nx, ny, nz, (0, 1.1), (0, 1.0), (0, 0.8))
    st = State.zeros(nx, ny, nz)
    rng = np.random.default_rng(21)
    g = d0.params.gamma
    for k in STATE:
        shape = st[k].shape
        if k == "rho":
            st[k][...] = 1.0 + 0.1 * rng.uniform(-1, 1, shape)
        elif k == "energy":
            st[k][...] = 0.1 / (g - 1.0) * (1.0 + 0.1 * rng.uniform(-1, 1, shape))
        elif k in ("bx", "by"):
            st[k][...] = 0.7 + 0.05 * rng.uniform(-1, 1, shape)
        else:
            st[k][...] = 0.05 * rng.uniform(-1, 1, shape)
    d = decks.Deck("open-ragged", d0.params, nx, ny, nz, m, st, nsteps=4)
    r, gg = pair(d)
    for s in range(1, 5):
        r.step(s)
        gg.step(s)
        assert_bitwise(gg, r, STATE, f"step {s}")


def test_open_boundaries_fp32(built):
    d = decks.open_blast(16)
    from lare3d_b200 import gpu
    from oracle import oracle
    r = oracle.simulation(d)
    g = gpu.simulation(d, precision=32)
    r.start(d.state)
    g.start(d.state)
    for s in range(1, 6):
        r.step(s)
        g.step(s)
    for f in STATE:
        e = rel_l2(g.get_field(f), r.get_field(f))
        assert e <= 1e-5, f"{f}: rel L2 {e:.2e}"


@pytest.mark.slow
def test_blast_64_100_steps(built):
    """Blast at 64^3, 100 steps at CFL 0.8: relative L2 per field <= 1e-10
    (observed: identical)."""
    d = decks.blast(64)
    r, g = pair(d)
    for s in range(1, 101):
        r.step(s)
        g.step(s)
    for f in STATE:
        a, b = g.get_field(f), r.get_field(f)
        assert rel_l2(a, b) <= 1e-10, f
        assert np.array_equal(a, b), f
    er, eg = r.energy(), g.energy()
    for q in range(5):
        assert abs(eg[q] - er[q]) <= 1e-12 * max(1.0, abs(er[q])), q


def test_orszag_tang_32_50_steps(built):
    d = decks.orszag_tang(32)
    r, g = pair(d)
    for s in range(1, 51):
        r.step(s)
        g.step(s)
    for f in STATE:
        assert np.array_equal(g.get_field(f), r.get_field(f)), f


@pytest.mark.parametrize("kperp", [0.0, 1.0e-6, 0.05])
def test_conduction_parity(built, kperp):
    """Reference flux (kperp = 0) and the cross-field extension."""
    d = decks.conduction(16, kappa_perp_ratio=kperp)
    r, g = pair(d)
    for it in range(2):
        assert r.conduct_heat(d.dt_fixed) == g.conduct_heat(d.dt_fixed)
        for f in ("energy", "temperature", "larsen_factor"):
            assert rel_l2(g.get_field(f), r.get_field(f)) <= 1e-12, f


def test_conduction_in_step(built):
    """Conduction inside lagrangian_step (lagran.F90:168-181, set_dt's
    stage cap :1153-1162)."""
    d = decks.conduction(12, kappa_0=1.0e-4)
    r, g = pair(d)
    for s in range(1, 4):
        r.step(s)
        g.step(s)
        for f in STATE:
            assert rel_l2(g.get_field(f), r.get_field(f)) <= 1e-12, (s, f)
    assert r.scalars().n_s_stages == g.scalars().n_s_stages


def test_fp32_form_error(built):
    """FP32 form vs the FP64 oracle after 100 steps (bar: 1e-5 per field)."""
    d = decks.blast(32)
    r, g = pair(d, precision=32)
    for s in range(1, 101):
        r.step(s)
        g.step(s)
    errs = {f: rel_l2(g.get_field(f), r.get_field(f)) for f in STATE}
    worst = max(errs.values())
    assert worst <= 1e-5, errs


def test_energy_budget_parity(built):
    d = decks.orszag_tang(16)
    r, g = pair(d)
    for s in range(1, 6):
        r.step(s)
        g.step(s)
    er, eg = r.energy(), g.energy()
    for q in range(5):
        assert abs(eg[q] - er[q]) <= 1e-12 * max(1e-30, abs(er[q])), (q, er[q], eg[q])


def test_run_matches_steps(built):
    d = decks.blast(12)
    from lare3d_b200 import gpu
    a = gpu.simulation(d, precision=gpu.EXACT64)
    b = gpu.simulation(d, precision=gpu.EXACT64)
    a.start(d.state)
    b.start(d.state)
    for s in range(1, 6):
        a.step(s)
    n, t, dt = b.run(0, 5)
    assert n == 5
    for f in STATE:
        assert np.array_equal(a.get_field(f), b.get_field(f))
    # t_end stops the loop (lare3d.f90:81)
    c = gpu.simulation(d, precision=gpu.EXACT64)
    c.start(d.state)
    n2, t2, _ = c.run(0, 1000, t_end=a.scalars().time * 0.5)
    assert 0 < n2 < 5 and t2 >= a.scalars().time * 0.5


def test_field_roundtrip_and_errors(built):
    d = decks.blast(8)
    from lare3d_b200 import gpu
    g = gpu.simulation(d)
    g.start(d.state)
    x = np.asfortranarray(np.random.default_rng(0).standard_normal(g.get_field("energy").shape))
    g.set_field("energy", x)
    assert np.array_equal(g.get_field("energy"), x)
    with pytest.raises(LareError):
        g.get_field("nope")
    bad = d.state.copy()
    bad["rho"][3, 3, 3] = np.nan
    with pytest.raises(LareError) as e:
        g.upload(bad)
    assert "LARE_ENONFINITE" in str(e.value)


def test_div_b_gpu(built):
    from test_oracle_cpu import div_b
    n = 16
    d = decks.orszag_tang(n)
    from lare3d_b200 import gpu
    g = gpu.simulation(d)
    g.start(d.state)
    for s in range(1, 11):
        g.step(s)
    st = g.download()
    assert np.abs(div_b(st, d.metrics, n)).max() < 1e-12

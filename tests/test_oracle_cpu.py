"""CPU tests of the oracle (the C++ restatement of the reference's Fortran).

The reference ships no tests or golden outputs for this path, so the oracle
is pinned by properties the reference's scheme has by construction:
conservation of mass on periodic boxes (remap is conservative,
xremap.f90:174-182), div B at round-off (constrained transport,
xremap.f90:119-157, lagran.F90:1582-1635), preservation of uniform states,
axis symmetry of 1-D problems under the Strang orderings (remap.f90:71-99),
and a bounds-checked build that aborts on any access outside the
reference's allocated bounds.
"""
import numpy as np
import pytest

from conftest import rel_l2
from lare3d_b200 import decks
from lare3d_b200.abi import BC_PERIODIC, BC_USER, LareError, State, default_params
from lare3d_b200.grid import grid


def oracle_sim(deck, checked=False):
    from oracle import oracle
    return oracle.simulation(deck, checked=checked)


def div_b(st, m, n):
    """Cell-centred divergence of the face field (cells 1..n)."""
    bx, by, bz = st["bx"], st["by"], st["bz"]
    dxb = m["dxb"][2:n + 2][:, None, None]
    dyb = m["dyb"][2:n + 2][None, :, None]
    dzb = m["dzb"][2:n + 2][None, None, :]
    # bx(i) at array index i+2, by(j) at j+2, bz(k) at k+2; cells at index+1
    dbx = (bx[3:n + 3, 2:n + 2, 2:n + 2] - bx[2:n + 2, 2:n + 2, 2:n + 2]) / dxb
    dby = (by[2:n + 2, 3:n + 3, 2:n + 2] - by[2:n + 2, 2:n + 2, 2:n + 2]) / dyb
    dbz = (bz[2:n + 2, 2:n + 2, 3:n + 3] - bz[2:n + 2, 2:n + 2, 2:n + 2]) / dzb
    return dbx + dby + dbz


def mass(st, m, n):
    cv = (m["dxb"][2:n + 2][:, None, None] * m["dyb"][2:n + 2][None, :, None] * m["dzb"][2:n + 2][None, None, :])
    return float(np.sum(st["rho"][2:n + 2, 2:n + 2, 2:n + 2] * cv))


@pytest.mark.parametrize("name", ["blast", "orszag_tang"])
def test_bounds_checked_run(built, name):
    d = getattr(decks, name)(10)
    s = oracle_sim(d, checked=True)
    s.start(d.state)
    for st in range(1, 7):  # all six Strang orderings
        s.step(st)
    out = s.download()
    assert all(np.isfinite(v).all() for v in out.arrays.values())


def test_bounds_checked_conduction(built):
    d = decks.conduction(10)
    s = oracle_sim(d, checked=True)
    s.start(d.state)
    ns = s.conduct_heat(d.dt_fixed)
    assert ns >= 3 and ns % 2 == 1
    assert np.isfinite(s.download()["energy"]).all()


@pytest.mark.parametrize("name", ["blast", "orszag_tang"])
def test_mass_conservation(built, name):
    n = 12
    d = getattr(decks, name)(n)
    s = oracle_sim(d)
    s.start(d.state)
    m0 = mass(s.download(), d.metrics, n)
    for st in range(1, 9):
        s.step(st)
    m1 = mass(s.download(), d.metrics, n)
    assert abs(m1 - m0) / m0 < 1e-13


def test_div_b_round_off(built):
    n = 12
    d = decks.orszag_tang(n)
    s = oracle_sim(d)
    s.start(d.state)
    b0 = np.abs(div_b(s.download(), d.metrics, n)).max()
    for st in range(1, 7):
        s.step(st)
    st = s.download()
    bmag = np.abs(st["by"]).max()
    db = np.abs(div_b(st, d.metrics, n)).max()
    assert b0 < 1e-12
    assert db < 1e-12 * max(1.0, bmag) / (2 * np.pi / n)


def test_uniform_state_preserved(built):
    n = 8
    d = decks.blast(n)
    st = d.state
    st["energy"][...] = 0.9
    for k, v in (("bx", 0.3), ("by", -0.2), ("bz", 0.1)):
        st[k][...] = v
    s = oracle_sim(d)
    s.start(st)
    for k in range(1, 4):
        s.step(k)
    out = s.download()
    for k in ("rho", "energy", "bx", "by", "bz"):
        a = out[k]
        assert np.ptp(a) <= 1e-14 * max(1.0, np.abs(a).max()), k
    for k in ("vx", "vy", "vz"):
        assert np.abs(out[k]).max() < 1e-14


def _planar(n, axis):
    """1-D shock tube along `axis` on a periodic cube."""
    d = decks.blast(n)
    m = d.metrics
    c = [m["xc"], m["yc"], m["zc"]][axis]
    shape = [1, 1, 1]
    shape[axis] = -1
    prof = np.where(np.abs(c - 0.5) < 0.2, 1.0, 0.125).reshape(shape)
    st = d.state
    st["rho"][...] = np.broadcast_to(prof, st["rho"].shape)
    st["energy"][...] = np.broadcast_to(np.where(prof > 0.5, 2.5, 2.0), st["energy"].shape)
    for k in ("bx", "by", "bz"):
        st[k][...] = 0.0
    return d


def test_axis_symmetry(built):
    n = 12
    res = []
    for ax in range(3):
        d = _planar(n, ax)
        s = oracle_sim(d)
        s.start(d.state)
        for k in range(1, 7):
            s.step(k)
        out = s.download()
        rho = out["rho"][2:n + 2, 2:n + 2, 2:n + 2]
        res.append(np.moveaxis(rho, ax, 0)[:, 0, 0])
        # the profile stays planar
        r = np.moveaxis(rho, ax, 0)
        assert np.ptp(r - r[:, :1, :1]) < 1e-13
    assert rel_l2(res[1], res[0]) < 1e-12
    assert rel_l2(res[2], res[0]) < 1e-12


def test_user_boundaries_run(built):
    n = 10
    d = decks.blast(n, xbc_min=BC_USER, xbc_max=BC_USER, zbc_min=BC_USER, zbc_max=BC_USER)
    s = oracle_sim(d, checked=True)
    s.start(d.state)
    for k in range(1, 4):
        s.step(k)
    out = s.download()
    # v = 0 on the boundary node and in its ghosts (boundary.f90:259-293)
    vx = out["vx"]
    assert np.all(vx[0:3, :, :] == 0.0) and np.all(vx[n + 2:, :, :] == 0.0)
    assert np.all(vx[:, :, 0:3] == 0.0)


def test_invalid_arguments(built):
    from oracle import oracle
    d = decks.blast(8)
    with pytest.raises(LareError):
        from lare3d_b200.abi import Simulation
        Simulation(oracle.binding(), d.params, 3, 8, 8, d.metrics)
    s = oracle_sim(d)
    with pytest.raises(LareError):
        s.get_field("no_such_array")


def _layered(kperp, n=12):
    """B along x, T varying in y only: field-aligned conduction has nothing
    to do; only a cross-field conductivity moves heat."""
    from lare3d_b200 import decks
    from oracle import oracle
    d = decks.conduction(n, kappa_perp_ratio=kperp)
    st = d.state
    st["bx"][...] = 1.0
    st["by"][...] = 0.0
    st["bz"][...] = 0.0
    y = np.arange(-1, n + 3) / n
    T = 1.0 + 0.5 * np.sin(2 * np.pi * y)
    g = d.params.gamma
    st["energy"][...] = np.broadcast_to((T * 2.0 / (g - 1.0))[None, :, None], st["energy"].shape)
    st["rho"][...] = 1.0
    s = oracle.simulation(d)
    s.start(st)
    e0 = s.get_field("energy").copy()
    s.conduct_heat(50.0 * decks.dt_parab_estimate(st, d.metrics, d.params, n))
    return e0, s.get_field("energy")


def test_kappa_perp_extension_moves_heat_across_the_field(built):
    e0, e_par = _layered(0.0)
    _, e_perp = _layered(0.05)
    core = (slice(2, -2),) * 3
    # field-aligned only: the min_b regulariser (1e-10 of |B|^2) is all that leaks
    assert np.max(np.abs(e_par[core] - e0[core])) < 1e-8 * np.max(np.abs(e0[core]))
    # with kappa_perp the y profile relaxes: peaks cool, troughs warm
    d = e_perp[core] - e0[core]
    assert np.max(np.abs(d)) > 1e-4 * np.max(np.abs(e0[core]))
    dev = e0[core] - e0[core].mean()
    assert np.corrcoef(dev.ravel(), d.ravel())[0, 1] < -0.5
    assert d.ravel()[np.argmax(dev)] < 0 < d.ravel()[np.argmin(dev)]


# ---------------------------------------------------------------------------
# Open (characteristic) boundaries, openboundary.f90


@pytest.mark.parametrize("b", [(2 ** -0.5, 2 ** -0.5, 0.0), (1.0, 0.0, 0.0)])
def test_open_boundaries_bounds_checked(built, b):
    """Both solvers (fast mode; Alfven mode where the far field has no
    transverse B) stay inside the reference's array bounds."""
    d = decks.open_blast(12, b=b)
    s = oracle_sim(d, checked=True)
    s.start(d.state)
    for st in range(1, 7):
        s.step(st)
    assert all(np.isfinite(v).all() for v in s.download().arrays.values())


def test_open_boundaries_keep_a_uniform_state(built):
    d = decks.open_blast(10)
    d.state["energy"][...] = 0.1 / (d.params.gamma - 1.0)
    s = oracle_sim(d)
    s.start(d.state)
    a = s.download()
    for st in range(1, 7):
        s.step(st)
    c = s.download()
    for f in ("rho", "energy", "vx", "vy", "vz", "bx", "by", "bz"):
        assert np.abs(c[f] - a[f]).max() < 1e-12, f


def test_open_boundaries_let_waves_out(built):
    """A pressure pulse in a box open on four sides loses mass and keeps
    little kinetic energy, while the same pulse in a periodic box keeps its
    mass exactly and rings."""
    n = 16
    out = {}
    for name, over in (("open", {}), ("periodic", dict(xbc_min=BC_PERIODIC, xbc_max=BC_PERIODIC,
                                                       ybc_min=BC_PERIODIC, ybc_max=BC_PERIODIC))):
        d = decks.open_blast(n, **over)
        s = oracle_sim(d)
        s.start(d.state)
        m0 = mass(s.download(), d.metrics, n)
        for st in range(1, 81):
            s.step(st)
        out[name] = ((mass(s.download(), d.metrics, n) - m0) / m0, s.energy()[1])
    assert out["open"][0] < -1e-3
    assert abs(out["periodic"][0]) < 1e-13
    assert out["open"][1] < 0.2 * out["periodic"][1]


def test_gravity_free_fall(built):
    """Uniform state in a uniform gravity g (lagran.F90:379): no pressure or
    magnetic force, so after one step every vertex has vz = -g dt."""
    d = decks.blast(10)
    st = d.state
    st["energy"][...] = 0.1 / ((d.params.gamma - 1.0) * 1.0)
    g0 = 0.7
    s = oracle_sim(d)
    s.start(st, grav=np.full(d.metrics["zc"].shape, g0))
    s.step(1)
    dt = s.scalars().dt
    vz = s.get_field("vz")[2:-2, 2:-2, 2:-2]
    assert np.abs(vz + g0 * dt).max() <= 1e-13 * g0 * dt
    assert np.abs(s.get_field("vx")).max() <= 1e-13 * g0 * dt


def test_gravity_bounds_checked(built):
    d = decks.blast(8)
    s = oracle_sim(d, checked=True)
    zc = d.metrics["zc"]
    s.start(d.state, grav=np.ascontiguousarray(0.5 * (1.0 + 0.3 * np.sin(2.0 * np.pi * zc))))
    for st in range(1, 4):
        s.step(st)


def test_boris_limits_the_alfven_speed(built):
    """boris with a binding va_max (lagran.F90:1104-1109): gamma_boris < 1
    where B^2/rho >= va_max^2, equal to 1/(1 + B^2/(rho va_max^2)) there, and
    the CFL step grows because the fast speed drops."""
    va = 0.3
    d = decks.orszag_tang(12, boris=1, va_max=va)
    s = oracle_sim(d, checked=True)
    s.start(d.state)
    s.step(1)
    d0 = decks.orszag_tang(12)
    s0 = oracle_sim(d0)
    s0.start(d0.state)
    s0.step(1)
    assert s.scalars().dt > s0.scalars().dt
    gb = s.get_field("gamma_boris")
    assert 0.0 < gb.min() < 0.6 and gb.max() == 1.0


def test_restart_first_set_dt(built):
    """A context created with restart set: its first set_dt takes
    dt_from_restart and returns before advancing the time or recomputing
    dtr (lagran.F90:1080-1086); the next one computes dt from the state."""
    d = decks.blast(8)
    d.params.restart, d.params.dt_from_restart = 1, 1.25e-3
    s = oracle_sim(d, checked=True)
    s.start(d.state, time=0.5)
    s.step(1)
    sc = s.scalars()
    assert sc.dt == 1.25e-3 and sc.time == 0.5
    s.step(2)
    sc = s.scalars()
    assert sc.dt != 1.25e-3 and sc.time == 0.5 + sc.dt

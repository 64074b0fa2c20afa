"""GPU parity of the partially ionised plasma (neutral.f90) and of conduction
next to open boundaries.

Without conduction the FP64 engine agrees with the oracle BIT FOR BIT here
too: the neutral fraction's bisection runs the same operations on both
sides, with the same exponential (Cody-Waite reduction and a Taylor
polynomial, written out in the engine and in the oracle), so every branch
of the bisection goes the same way.  With conduction the last bit of pow()
may differ between CUDA and glibc (relative L2 bar 1e-12, as for the other
conduction tests); the neutral fraction then inherits that difference.  The
FP32 form is held to the 1e-5 relative-L2 bar."""
import numpy as np
import pytest

from conftest import STATE, rel_l2
from lare3d_b200 import decks
from lare3d_b200.abi import BC_USER, EOS_ION, EOS_PI, LareError

pytestmark = pytest.mark.gpu


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
    dict(eos_number=EOS_ION, cowling=True),
    dict(eos_number=EOS_PI, cowling=True),
    dict(eos_number=EOS_ION, cowling=False),
    dict(eos_number=EOS_ION, cowling=True, xbc_min=BC_USER, xbc_max=BC_USER),
]


@pytest.mark.parametrize("kw", CASES)
def test_partially_ionised_bitwise(built, kw):
    d = decks.partially_ionised(16, eta_bar=1e-2, **kw)
    r, g = pair(d)
    names = STATE + ["xi_n"] + (["eta_perp"] if kw["cowling"] else [])
    assert_bitwise(g, r, names, "start")
    for s in range(1, 5):
        r.step(s)
        g.step(s)
        assert_bitwise(g, r, names + ["pressure", "eta", "ohmic_dep", "visc_dep"], f"step {s}")
    sr, sg = r.scalars(), g.scalars()
    assert (sr.time, sr.dt, sr.dtr, sr.last_substeps) == (sg.time, sg.dt, sg.dtr, sg.last_substeps)
    # a sum over the grid: the device adds block partial sums, the oracle
    # runs the reference's serial loop
    assert abs(sg.total_ohmic_heating - sr.total_ohmic_heating) <= 1e-12 * abs(sr.total_ohmic_heating)


@pytest.mark.parametrize("eos", [EOS_ION, EOS_PI])
def test_partially_ionised_with_conduction(built, eos):
    """The RKL2 stages re-solve xi_n after each stage (conduct.f90:404) and
    take the temperature with the per-cell xi_n."""
    d = decks.partially_ionised(12, eos_number=eos, eta_bar=1e-2, conduction=1, kappa_0=1.0e-1)
    r, g = pair(d)
    for s in range(1, 4):
        r.step(s)
        g.step(s)
        assert r.scalars().n_s_stages == g.scalars().n_s_stages
        for f in STATE + ["xi_n", "eta_perp", "temperature"]:
            assert rel_l2(g.get_field(f), r.get_field(f)) <= 1e-12, (s, f)
    assert r.scalars().n_s_stages >= 3


def test_partially_ionised_fp32(built):
    d = decks.partially_ionised(16, eta_bar=1e-2)
    r, g = pair(d, precision=32)
    for s in range(1, 6):
        r.step(s)
        g.step(s)
    for f in STATE + ["xi_n", "eta_perp"]:
        e = rel_l2(g.get_field(f), r.get_field(f))
        assert e <= 1e-5, f"{f}: rel L2 {e:.2e}"


def test_empty_temperature_bracket_is_an_error(built):
    """A cell with negative energy: the kernel flags LARE_EEOS and returns
    (the reference stops); the call reports it."""
    from lare3d_b200 import gpu
    d = decks.partially_ionised(8)
    d.state["energy"][5, 5, 5] = -1.0
    g = gpu.simulation(d)
    with pytest.raises(LareError) as ei:
        g.start(d.state)
    assert ei.value.code == -9


def test_open_boundaries_with_conduction(built):
    """Conduction next to open sides: every RKL2 stage buffer keeps the
    energy's ghosts there, as the reference's Y(3) does."""
    d = decks.open_blast(16, conduction=1, kappa_0=10.0)
    r, g = pair(d)
    for s in range(1, 4):
        r.step(s)
        g.step(s)
        assert r.scalars().n_s_stages == g.scalars().n_s_stages
        for f in STATE:
            assert rel_l2(g.get_field(f), r.get_field(f)) <= 1e-12, (s, f)
    assert r.scalars().n_s_stages >= 3


@pytest.mark.parametrize("cond", [0, 1])
def test_radiative_losses(built, cond):
    """Optically thin radiation (radiative.f90) alone and next to
    conduction (lagran.F90:168-181 adds both energy changes to energy0).
    The band powers come from pow(), so the bar is 1e-12 as for conduction."""
    d = decks.radiative_blast(16, conduction=cond, kappa_0=2.0e-2)
    r, g = pair(d)
    for s in range(1, 4):
        r.step(s)
        g.step(s)
        for f in STATE:
            assert rel_l2(g.get_field(f), r.get_field(f)) <= 1e-12, (s, f)
    if cond:
        assert r.scalars().n_s_stages == g.scalars().n_s_stages >= 3


def test_radiative_losses_fp32(built):
    d = decks.radiative_blast(16)
    r, g = pair(d, precision=32)
    for s in range(1, 6):
        r.step(s)
        g.step(s)
    for f in STATE:
        e = rel_l2(g.get_field(f), r.get_field(f))
        assert e <= 1e-5, f"{f}: rel L2 {e:.2e}"


@pytest.mark.parametrize("name", ["orszag_tang", "open_blast"])
def test_rke_bitwise(built, name):
    """rke: every cell's kinetic-energy defect is the reference's sum, in
    the reference's order, so delta_ke (cells 1:n, after the remap) and the
    corrected energy agree bit for bit."""
    d = getattr(decks, name)(16, rke=1)
    r, g = pair(d)
    n = 16
    inner = (slice(2, n + 2),) * 3
    for s in range(1, 5):
        r.lagrangian_step(s)
        g.lagrangian_step(s)
        r.eulerian_remap(s)
        g.eulerian_remap(s)
        a, b = g.get_field("delta_ke")[inner], r.get_field("delta_ke")[inner]
        assert np.count_nonzero(a != b) == 0, f"step {s}: delta_ke differs (max {np.abs(a - b).max():.3e})"
        r.energy_correction()
        g.energy_correction()
        r.eta_calc()
        g.eta_calc()
        assert_bitwise(g, r, STATE, f"step {s}")
    # and through lare_gpu_step
    for s in range(5, 7):
        r.step(s)
        g.step(s)
        assert_bitwise(g, r, STATE, f"step {s}")


def test_widened_physics_together_with_open_sides(built):
    """Partially ionised with Cowling resistivity, rke and open x/y sides in
    one deck: FP64 bit for bit over four steps."""
    from lare3d_b200.abi import BC_OPEN
    d = decks.partially_ionised(16, eta_bar=1e-2, rke=1, xbc_min=BC_OPEN, xbc_max=BC_OPEN, ybc_min=BC_OPEN,
                                ybc_max=BC_OPEN)
    r, g = pair(d)
    for s in range(1, 5):
        r.step(s)
        g.step(s)
        assert_bitwise(g, r, STATE + ["xi_n", "eta_perp"], f"step {s}")


def test_rke_fp32(built):
    d = decks.orszag_tang(16, rke=1)
    r, g = pair(d, precision=32)
    for s in range(1, 6):
        r.step(s)
        g.step(s)
    for f in STATE:
        e = rel_l2(g.get_field(f), r.get_field(f))
        assert e <= 1e-5, f"{f}: rel L2 {e:.2e}"


@pytest.mark.parametrize("name", ["orszag_tang", "blast"])
def test_cooling_term_bitwise(built, name):
    """cooling_term's two moving averages (viscous in the corrector, ohmic
    in each resistive sub-cycle) and the energies they cool, bit for bit."""
    d = getattr(decks, name)(16, cooling_term=1, alpha_av=0.05)
    r, g = pair(d)
    for s in range(1, 5):
        r.step(s)
        g.step(s)
        assert_bitwise(g, r, STATE + ["cool_term_v", "cool_term_b"], f"step {s}")


def test_cooling_term_fp32(built):
    d = decks.orszag_tang(16, cooling_term=1, alpha_av=0.05)
    r, g = pair(d, precision=32)
    for s in range(1, 6):
        r.step(s)
        g.step(s)
    for f in STATE:
        e = rel_l2(g.get_field(f), r.get_field(f))
        assert e <= 1e-5, f"{f}: rel L2 {e:.2e}"


def test_coronal_heating_bitwise(built):
    """The user_defined_heating hook with a caller-set heating rate."""
    from lare3d_b200.abi import alloc
    d = decks.orszag_tang(16, coronal_heating=1)
    r, g = pair(d)
    rng = np.random.default_rng(3)
    heat = np.asfortranarray(alloc("cell", 16, 16, 16) + 1e-2 * rng.random(alloc("cell", 16, 16, 16).shape))
    r.set_field("heat_in", heat)
    g.set_field("heat_in", heat)
    for s in range(1, 5):
        r.step(s)
        g.step(s)
        assert_bitwise(g, r, STATE, f"step {s}")
    assert np.array_equal(g.get_field("heat_in"), heat)

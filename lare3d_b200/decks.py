"""Synthetic initial states (the user-deck layer, cf. src/initial_conditions.f90
and src/control.f90) for the three plain-method workloads:

* ``blast``          3-D MHD blast, 64^3 periodic unit cube, 100 steps at CFL 0.8
* ``orszag_tang``    resistive 3-D Orszag-Tang-type vortex, 256^3 periodic
                     [0, 2pi]^3, eta = 1e-3, 200 steps
* ``conduction``     sheared arcade B = curl(A_y e_y), A_y = cos(kx) exp(-kz),
                     isobaric Gaussian hot spots, kappa_par ~ T^{5/2}, RKL2

and for the widened physics: ``open_blast`` (characteristic boundaries),
``partially_ionised`` (neutral fraction, Cowling resistivity) and
``radiative_blast`` (optically thin losses); ``rke`` and ``cooling_term`` are
switches on any deck.

Each returns a :class:`Deck` with control parameters, grid metrics and the
Fortran-bounded state; ghost cells are filled by the caller's
boundary_conditions (lare3d.f90:65).  Random perturbations come from the
reference's KISS generator (random_generator.f90) seeded with
random_init_local(seed).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .abi import BC_OPEN, BC_PERIODIC, BC_USER, EOS_ION, LareParams, State, default_params
from .grid import grid

_HERE = os.path.dirname(os.path.abspath(__file__))
_host_lib = None


def host_lib():
    global _host_lib
    if _host_lib is None:
        path = os.path.join(_HERE, "liblare_host.so")
        if not os.path.exists(path):
            raise RuntimeError("liblare_host.so is not built; run __graft_entry__.build()")
        lib = C.CDLL(path)
        lib.lare_kiss_fill.argtypes = [C.c_int, C.c_long, C.POINTER(C.c_double)]
        lib.lare_kiss_fill.restype = None
        _host_lib = lib
    return _host_lib


def kiss_uniform(seed: int, n: int) -> np.ndarray:
    """n KISS draws in [0,1) after random_init_local(seed)."""
    out = np.empty(n, dtype=np.float64)
    host_lib().lare_kiss_fill(int(seed), int(n), out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


@dataclass
class Deck:
    name: str
    params: LareParams
    nx: int
    ny: int
    nz: int
    metrics: dict
    state: State
    nsteps: int
    grav: Optional[np.ndarray] = None
    dt_fixed: Optional[float] = None   # conduction operator timing only
    info: dict = field(default_factory=dict)


def _coords(m, nx, ny, nz):
    """Broadcastable coordinate arrays for cells (-1:n+2) and nodes (-2:n+2)."""
    xc = m["xc"][:, None, None]
    yc = m["yc"][None, :, None]
    zc = m["zc"][None, None, :]
    xb = m["xb"][:, None, None]
    yb = m["yb"][None, :, None]
    zb = m["zb"][None, None, :]
    return xc, yc, zc, xb, yb, zb


def blast(n: int = 64, **over) -> Deck:
    g = 5.0 / 3.0
    p = default_params(gamma=g, visc1=0.1, visc2=0.5, dt_multiplier=0.8)
    for k, v in over.items():
        setattr(p, k, v)
    m = grid(n, n, n, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0))
    st = State.zeros(n, n, n)
    xc, yc, zc, *_ = _coords(m, n, n, n)
    r = np.sqrt((xc - 0.5) ** 2 + (yc - 0.5) ** 2 + (zc - 0.5) ** 2)
    pres = np.where(r < 0.1, 10.0, 0.1)
    st["rho"][...] = 1.0
    st["energy"][...] = np.asfortranarray(pres / ((g - 1.0) * 1.0))
    b0 = 1.0 / math.sqrt(2.0)
    st["bx"][...] = b0
    st["by"][...] = b0
    st["bz"][...] = 0.0
    return Deck("blast", p, n, n, n, m, st, nsteps=100)


def open_blast(n: int = 64, b=(1.0 / math.sqrt(2.0), 1.0 / math.sqrt(2.0), 0.0), p_in: float = 0.3,
               **over) -> Deck:
    """A pressure pulse off-centre towards x min in a box with open
    (characteristic) boundaries on the x and y sides and periodic z
    (openboundary.f90).  The ghosts of the open sides carry the ambient
    state, which serves as the far field.  A field along x only makes the
    x faces take the Alfven-mode solver (no transverse far field).  The
    reference's characteristic boundary is linearised about the far field:
    a strong wave leaving the box (inner pressure many times the ambient)
    drives its ghost density to TINY, so the default overpressure is 3:1."""
    g = 5.0 / 3.0
    p = default_params(gamma=g, visc1=0.1, visc2=0.5, dt_multiplier=0.8,
                       xbc_min=BC_OPEN, xbc_max=BC_OPEN, ybc_min=BC_OPEN, ybc_max=BC_OPEN)
    for k, v in over.items():
        setattr(p, k, v)
    m = grid(n, n, n, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0))
    st = State.zeros(n, n, n)
    xc, yc, zc, *_ = _coords(m, n, n, n)
    r = np.sqrt((xc - 0.25) ** 2 + (yc - 0.5) ** 2 + (zc - 0.5) ** 2)
    pres = np.where(r < 0.15, p_in, 0.1)
    st["rho"][...] = 1.0
    st["energy"][...] = np.asfortranarray(pres / ((g - 1.0) * 1.0))
    st["bx"][...] = b[0]
    st["by"][...] = b[1]
    st["bz"][...] = b[2]
    return Deck("open_blast", p, n, n, n, m, st, nsteps=100)


# Physical constants of shared_data.F90:36-57 (SI).
_MU0 = 4.0e-7 * math.pi
_KB = 1.3806488e-23
_MH = 1.672621777e-27
_ME = 9.10938291e-31
_HP = 6.62606957e-34
_CHI = 2.17870364e-18   # ionisation potential of hydrogen


def neutral_constants(eos_number: int, B_norm: float = 0.1, L_norm: float = 1.0e6, rho_norm: float = 1.67e-4,
                      mf: float = 1.2, sigma_in: float = 5.0e-19) -> dict:
    """The ionisation model's constants as the reference holds them after
    setup_neutral (neutral.f90:31-63) and normalise_transport
    (normalise.f90:25-51), for the normalisation of control.f90:46-60."""
    mbar = _MH * mf
    f_bar = (2.0 * math.pi * (_ME / _HP) * (_KB / _HP)) ** 1.5
    t_bar = _CHI / _KB
    r_bar = 4.0 / mbar
    eta_bar = 2.0 * mbar / (math.sqrt(16.0 * _KB / (math.pi * mbar)) * sigma_in)
    pressure0 = B_norm ** 2 / _MU0
    energy0 = pressure0 / rho_norm
    v0 = math.sqrt(energy0)
    temp_norm = (mbar / _KB) * energy0
    t_bar = t_bar / temp_norm
    r_bar = r_bar * rho_norm / temp_norm ** 1.5
    eta_bar_0 = (_MU0 * L_norm * v0) * rho_norm ** 2 * math.sqrt(temp_norm) / B_norm ** 2
    eta_bar = eta_bar / eta_bar_0
    ionise_pot = _CHI / (energy0 * mbar) if eos_number == EOS_ION else 0.0
    return dict(f_bar=f_bar, t_bar=t_bar, r_bar=r_bar, tr=6420.0 / temp_norm, eta_bar=eta_bar, ionise_pot=ionise_pot)


def get_neutral(t_v, rho_v, c: dict):
    """neutral.f90:140-153 in numpy (initial conditions only)."""
    bof = 1.0 / (0.5 * c["f_bar"] * c["tr"] * np.sqrt(t_v)) * np.exp(
        (0.25 * (t_v / c["tr"] - 1.0) + 1.0) * c["t_bar"] / t_v)
    r = 0.5 * (-1.0 + np.sqrt(1.0 + c["r_bar"] * rho_v * bof))
    return r / (1.0 + r)


def partially_ionised(n: int = 32, eos_number: int = EOS_ION, cowling: bool = True, T0: float = 1.8,
                      dT: float = 0.4, v0: float = 0.3, eta_bar: Optional[float] = None, **over) -> Deck:
    """A partially ionised Orszag-Tang-type vortex on the periodic [0, 2pi]^3
    (neutral.f90, eos_number EOS_ION or EOS_PI, optionally with Cowling
    resistivity): uniform density 1, a temperature of T0 +- dT around a
    normalised 1.8 (about 12,500 K under the default normalisation, where
    hydrogen is some 5 % ionised at this density), and the energy set from
    it as initial_conditions.f90:69-87 does.  The physical eta_bar of the
    default normalisation makes eta_perp some 1e-8; pass a larger eta_bar
    to give the Cowling terms weight."""
    g = 5.0 / 3.0
    c = neutral_constants(eos_number)
    if eta_bar is not None:
        c["eta_bar"] = eta_bar
    p = default_params(gamma=g, visc1=0.1, visc2=0.5, dt_multiplier=0.8, resistive_mhd=1,
                       eta_background=1.0e-3, eta0=0.0, j_max=1.0e10, eos_number=eos_number,
                       cowling_resistivity=1 if cowling else 0, **c)
    for k, v in over.items():
        setattr(p, k, v)
    L = 2.0 * math.pi
    m = grid(n, n, n, (0.0, L), (0.0, L), (0.0, L))
    st = State.zeros(n, n, n)
    xc, yc, zc, xb, yb, zb = _coords(m, n, n, n)
    ones_c = np.ones((n + 4, n + 4, n + 4))
    T = (T0 + dT * np.sin(xc) * np.sin(yc) * np.cos(zc)) * ones_c
    rho = ones_c.copy()
    xi = get_neutral(T, rho, c)
    st["rho"][...] = rho
    st["energy"][...] = np.asfortranarray((T * (2.0 - xi) + (1.0 - xi) * p.ionise_pot * (g - 1.0)) / (g - 1.0))
    ones_n = np.ones((n + 5, n + 5, n + 5))
    st["vx"][...] = np.asfortranarray(-v0 * np.sin(zb) * ones_n)
    st["vy"][...] = np.asfortranarray(v0 * np.sin(xb) * ones_n)
    st["vz"][...] = np.asfortranarray(v0 * np.sin(yb) * ones_n)
    s4 = 1.0 / math.sqrt(4.0 * math.pi)
    st["bx"][...] = (-np.sin(m["zc"]) * s4)[None, None, :]
    st["by"][...] = (np.sin(2.0 * m["xc"]) * s4)[:, None, None]
    st["bz"][...] = (np.sin(m["yc"]) * s4)[None, :, None]
    return Deck("partially_ionised", p, n, n, n, m, st, nsteps=20, info={"eos_number": eos_number})


def normalisation(B_norm: float = 0.1, L_norm: float = 1.0e6, rho_norm: float = 1.67e-4, mf: float = 1.2) -> dict:
    """temp_norm and time_norm as normalise_transport forms them
    (normalise.f90:25-34), with rho_norm and mf, for lare_params."""
    mbar = _MH * mf
    energy0 = (B_norm ** 2 / _MU0) / rho_norm
    return dict(temp_norm=(mbar / _KB) * energy0, time_norm=L_norm / math.sqrt(energy0), rho_norm=rho_norm, mf=mf)


def radiative_blast(n: int = 16, rho_norm: float = 1.0e-11, **over) -> Deck:
    """The blast deck with optically thin radiative losses on
    (radiative.f90) under a coronal normalisation (B_norm 1e-3 T,
    L_norm 1e6 m): the ambient pressure rises along x so that the ambient
    temperature sweeps the loss table's bands from 3.5e4 K to 3.5e6 K, and
    the hot core (above the table's 1e7 K) is left alone, as the reference
    leaves it."""
    d = blast(n, radiation=1, **normalisation(B_norm=1.0e-3, L_norm=1.0e6, rho_norm=rho_norm))
    for k, v in over.items():
        setattr(d.params, k, v)
    g = d.params.gamma
    xc, yc, zc, *_ = _coords(d.metrics, n, n, n)
    r = np.sqrt((xc - 0.5) ** 2 + (yc - 0.5) ** 2 + (zc - 0.5) ** 2)
    pres = np.where(r < 0.1, 10.0, 0.1 * xc ** 2 + 0.001) * np.ones((n + 4, n + 4, n + 4))
    d.state["energy"][...] = np.asfortranarray(pres / (g - 1.0))
    d.name = "radiative_blast"
    return d


def example_heating(d: Deck, time_norm: float, rho_norm: float, L_norm: float) -> np.ndarray:
    """The heating rate of the reference's example hook (radiative.f90:69-93
    user_defined_heating): 0.1 exp(-x^2 - y^2 - z^2) W/m^3 on cells 1:n,
    zero on the ghosts, converted to Lare units; for the cell field
    "heat_in" of a deck with coronal_heating on."""
    from .abi import alloc
    n0, n1, n2 = d.nx, d.ny, d.nz
    h = alloc("cell", n0, n1, n2)
    xc, yc, zc, *_ = _coords(d.metrics, n0, n1, n2)
    rate = 0.1 * np.exp(-xc ** 2 - yc ** 2 - zc ** 2) * np.ones(h.shape)
    h[2:n0 + 2, 2:n1 + 2, 2:n2 + 2] = rate[2:n0 + 2, 2:n1 + 2, 2:n2 + 2]
    return np.asfortranarray(h * time_norm ** 3 / (rho_norm * L_norm ** 2))


def _curl_edges(Ax, Ay, Az, m, n):
    """Discrete curl of periodic edge fields onto the face arrays.

    Ax[i,j,k]: x-cell i, y-node j, z-node k; Ay: x-node, y-cell, z-node;
    Az: x-node, y-node, z-cell.  A lattice index is the Fortran cell or node
    index modulo n.  Each face takes the circulation of its four bounding
    edges divided by its actual widths, over the face array's full Fortran
    extent (ghosts are refreshed by bfield_bcs afterwards).
    """
    def w(lo, hi):
        return np.arange(lo, hi + 1) % n

    def width(arr, lo, hi):          # metric stored from Fortran index -1
        return arr[np.arange(lo, hi + 1) + 1]

    dxb, dyb, dzb = m["dxb"], m["dyb"], m["dzb"]
    # bx(-2:n+2, -1:n+2, -1:n+2)
    i, j, k = w(-2, n + 2), w(-1, n + 2), w(-1, n + 2)
    jm, km = w(-2, n + 1), w(-2, n + 1)
    bx = ((Az[np.ix_(i, j, k)] - Az[np.ix_(i, jm, k)]) / width(dyb, -1, n + 2)[None, :, None]
          - (Ay[np.ix_(i, j, k)] - Ay[np.ix_(i, j, km)]) / width(dzb, -1, n + 2)[None, None, :])
    # by(-1:n+2, -2:n+2, -1:n+2)
    i, j, k = w(-1, n + 2), w(-2, n + 2), w(-1, n + 2)
    im, km = w(-2, n + 1), w(-2, n + 1)
    by = ((Ax[np.ix_(i, j, k)] - Ax[np.ix_(i, j, km)]) / width(dzb, -1, n + 2)[None, None, :]
          - (Az[np.ix_(i, j, k)] - Az[np.ix_(im, j, k)]) / width(dxb, -1, n + 2)[:, None, None])
    # bz(-1:n+2, -1:n+2, -2:n+2)
    i, j, k = w(-1, n + 2), w(-1, n + 2), w(-2, n + 2)
    im, jm = w(-2, n + 1), w(-2, n + 1)
    bz = ((Ay[np.ix_(i, j, k)] - Ay[np.ix_(im, j, k)]) / width(dxb, -1, n + 2)[:, None, None]
          - (Ax[np.ix_(i, j, k)] - Ax[np.ix_(i, jm, k)]) / width(dyb, -1, n + 2)[None, :, None])
    return np.asfortranarray(bx), np.asfortranarray(by), np.asfortranarray(bz)


def orszag_tang(n: int = 256, seed: int = 7, amp: float = 1.0e-3, **over) -> Deck:
    g = 5.0 / 3.0
    p = default_params(gamma=g, visc1=0.1, visc2=0.5, dt_multiplier=0.8,
                       resistive_mhd=1, eta_background=1.0e-3, eta0=0.0, j_max=1.0e10)
    for k, v in over.items():
        setattr(p, k, v)
    L = 2.0 * math.pi
    m = grid(n, n, n, (0.0, L), (0.0, L), (0.0, L))
    st = State.zeros(n, n, n)
    xc, yc, zc, xb, yb, zb = _coords(m, n, n, n)
    rho0 = 25.0 / (36.0 * math.pi)
    p0 = 5.0 / (12.0 * math.pi)
    st["rho"][...] = rho0
    st["energy"][...] = p0 / ((g - 1.0) * rho0)
    ones_n = np.ones((n + 5, n + 5, n + 5))
    st["vx"][...] = np.asfortranarray(-np.sin(zb) * ones_n)
    st["vy"][...] = np.asfortranarray(np.sin(xb) * ones_n)
    st["vz"][...] = np.asfortranarray(np.sin(yb) * ones_n)
    s4 = 1.0 / math.sqrt(4.0 * math.pi)
    bx = st["bx"]
    by = st["by"]
    bz = st["bz"]
    bx[...] = (-np.sin(m["zc"]) * s4)[None, None, :]
    by[...] = (np.sin(2.0 * m["xc"]) * s4)[:, None, None]
    bz[...] = (np.sin(m["yc"]) * s4)[None, :, None]
    if amp != 0.0:
        r = kiss_uniform(seed, 3 * n ** 3)
        A = [(2.0 * r[q * n ** 3:(q + 1) * n ** 3] - 1.0).reshape((n, n, n), order="F") * amp for q in range(3)]
        dbx, dby, dbz = _curl_edges(A[0], A[1], A[2], m, n)
        bx += dbx
        by += dby
        bz += dbz
    return Deck("orszag_tang", p, n, n, n, m, st, nsteps=200, info={"seed": seed, "amp": amp})


def conduction(n: int = 256, seed: int = 11, nspots: int = 8, T0: float = 1.0,
               kappa_0: float = 1.0e-3, dt_ratio: float = 50.0, kappa_perp_ratio: float = 1.0e-6,
               **over) -> Deck:
    """Sheared-arcade conduction workload: x, y periodic; z BC_USER.
    kappa_perp_ratio = kappa_perp / kappa_par of the workload (an extension:
    the reference has no cross-field term; 0 gives its flux exactly)."""
    g = 5.0 / 3.0
    p = default_params(gamma=g, conduction=1, heat_flux_limiter=1, flux_limiter=0.1,
                       kappa_0=kappa_0, dt_multiplier=0.9, kappa_perp_ratio=kappa_perp_ratio,
                       zbc_min=BC_USER, zbc_max=BC_USER)
    for k, v in over.items():
        setattr(p, k, v)
    m = grid(n, n, n, (0.0, 1.0), (0.0, 1.0), (0.0, 1.0), bcs=(BC_PERIODIC, BC_PERIODIC, BC_USER))
    st = State.zeros(n, n, n)
    xc, yc, zc, xb, yb, zb = _coords(m, n, n, n)
    k = 2.0 * math.pi / 1.0
    # A_y on y-edges (xb_i, yc_j, zb_k); B = curl(A_y e_y):
    # bx = -dA_y/dz on x-faces, bz = dA_y/dx on z-faces (by = 0).
    Ay = np.cos(k * m["xb"])[:, None] * np.exp(-k * m["zb"])[None, :]   # (x node -2:n+2, z node -2:n+2)
    dzb = m["dzb"]
    dxb = m["dxb"]
    # bx(i, j, kc) for kc in -1:n+2 uses Ay(i, kc) - Ay(i, kc-1)
    bxz = -(Ay[:, 1:] - Ay[:, :-1]) / dzb[None, :]            # (-2:n+2, -1:n+2)
    st["bx"][...] = bxz[:, None, :]
    bzx = (Ay[1:, :] - Ay[:-1, :]) / dxb[:, None]             # (-1:n+2, -2:n+2)
    st["bz"][...] = bzx[:, None, :]
    st["by"][...] = 0.0
    # Temperature: T0 + sum of Gaussian hot spots (amplitude 10*T0, sigma = 8 cells)
    sig = 8.0 / n
    r = kiss_uniform(seed, 3 * nspots)
    T = np.full((n + 4, n + 4, n + 4), T0)
    for s in range(nspots):
        cx, cy, cz = r[3 * s], r[3 * s + 1], 0.2 + 0.6 * r[3 * s + 2]
        dx = np.abs(xc - cx)
        dx = np.minimum(dx, 1.0 - dx)
        dy = np.abs(yc - cy)
        dy = np.minimum(dy, 1.0 - dy)
        dz = zc - cz
        T = T + 10.0 * T0 * np.exp(-(dx * dx + dy * dy + dz * dz) / (2.0 * sig * sig))
    pres0 = 1.0
    xi = p.xi_n
    st["rho"][...] = np.asfortranarray(pres0 / T)
    st["energy"][...] = np.asfortranarray(T * (2.0 - xi) / (g - 1.0))
    # dt from the explicit limit of calc_s_stages (conduct.f90:80-129).
    dtp = dt_parab_estimate(st, m, p, n)
    d = Deck("conduction", p, n, n, n, m, st, nsteps=10, dt_fixed=dt_ratio * dtp,
             info={"seed": seed, "nspots": nspots, "dt_parab": dtp, "dt_ratio": dt_ratio})
    return d


def dt_parab_estimate(st: State, m: dict, p: LareParams, n: int) -> float:
    """numpy restatement of conduct.f90:64-129 (temperature, Larsen factor,
    explicit conduction limit), used only to pick a workload dt."""
    g = p.gamma
    xi = p.xi_n
    e = st["energy"]
    T = (g - 1.0) / (2.0 - xi) * (e - (1.0 - xi) * p.ionise_pot)      # (-1:n+2)^3
    Ti = T[1:n + 2, 1:n + 2, 1:n + 2]                                   # 0:n
    dxb = m["dxb"][1:n + 2][:, None, None]
    dyb = m["dyb"][1:n + 2][None, :, None]
    dzb = m["dzb"][1:n + 2][None, None, :]
    rho = st["rho"][1:n + 2, 1:n + 2, 1:n + 2]
    temp = Ti ** 2.5
    q_fs = p.flux_limiter * 42.85 * rho * Ti ** 1.5
    qx = -p.kappa_0 * temp * (T[2:n + 3, 1:n + 2, 1:n + 2] - T[0:n + 1, 1:n + 2, 1:n + 2]) * 0.5 / dxb
    qy = -p.kappa_0 * temp * (T[1:n + 2, 2:n + 3, 1:n + 2] - T[1:n + 2, 0:n + 1, 1:n + 2]) * 0.5 / dyb
    qz = -p.kappa_0 * temp * (T[1:n + 2, 1:n + 2, 2:n + 3] - T[1:n + 2, 1:n + 2, 0:n + 1]) * 0.5 / dzb
    lf = q_fs / np.sqrt(q_fs * q_fs + qx * qx + qy * qy + qz * qz)
    if not p.heat_flux_limiter:
        lf = np.ones_like(lf)
    lf = lf[1:, 1:, 1:]
    t = temp[1:, 1:, 1:]
    r = rho[1:, 1:, 1:]
    h2 = np.minimum(np.minimum(dxb[1:] ** 2, dyb[:, 1:] ** 2), dzb[:, :, 1:] ** 2)
    dtp = np.min(r * h2 / (2.0 * p.kappa_0 * lf * t))
    return float(p.dt_multiplier * dtp / math.sqrt(3.0))


DECKS = {"blast": blast, "orszag_tang": orszag_tang, "conduction": conduction}

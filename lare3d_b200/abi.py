"""ctypes mirror of include/lare_gpu.h and a generic binding over it.

The same binding drives any library that exports the lare_gpu.h entry
points under some prefix; the product uses it for ``liblare_gpu.so``
(prefix ``lare_gpu_``).  Arrays cross the boundary as Fortran-ordered
float64 numpy arrays with the reference's bounds (mpi_routines.F90:295-327).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np

BC_PERIODIC = 1
BC_USER = 2
BC_OPEN = 3

EOS_IDEAL = 1
EOS_ION = 2
EOS_PI = 3

LARE_OK = 0
ERRORS = {
    -1: "LARE_EINVAL",
    -2: "LARE_ECUDA",
    -3: "LARE_ENOMEM",
    -4: "LARE_EDT",
    -5: "LARE_ESTAGES",
    -6: "LARE_ENOTFOUND",
    -7: "LARE_ENONFINITE",
    -8: "LARE_ETOOLARGE",
    -9: "LARE_EEOS",
}


class LareParams(C.Structure):
    """struct lare_params (include/lare_gpu.h)."""

    _fields_ = [
        ("gamma", C.c_double),
        ("visc1", C.c_double),
        ("visc2", C.c_double),
        ("eta_background", C.c_double),
        ("eta0", C.c_double),
        ("j_max", C.c_double),
        ("kappa_0", C.c_double),
        ("flux_limiter", C.c_double),
        ("ionise_pot", C.c_double),
        ("xi_n", C.c_double),
        ("va_max", C.c_double),
        ("dt_multiplier", C.c_double),
        ("dt_from_restart", C.c_double),
        ("kappa_perp_ratio", C.c_double),
        ("resistive_mhd", C.c_int),
        ("conduction", C.c_int),
        ("heat_flux_limiter", C.c_int),
        ("use_viscous_damping", C.c_int),
        ("boris", C.c_int),
        ("restart", C.c_int),
        ("xbc_min", C.c_int),
        ("xbc_max", C.c_int),
        ("ybc_min", C.c_int),
        ("ybc_max", C.c_int),
        ("zbc_min", C.c_int),
        ("zbc_max", C.c_int),
        ("eos_number", C.c_int),
        ("cowling_resistivity", C.c_int),
        ("f_bar", C.c_double),
        ("t_bar", C.c_double),
        ("r_bar", C.c_double),
        ("tr", C.c_double),
        ("eta_bar", C.c_double),
        ("radiation", C.c_int),
        ("temp_norm", C.c_double),
        ("time_norm", C.c_double),
        ("rho_norm", C.c_double),
        ("mf", C.c_double),
        ("rke", C.c_int),
        ("cooling_term", C.c_int),
        ("alpha_av", C.c_double),
        ("coronal_heating", C.c_int),
    ]


class LareScalars(C.Structure):
    """struct lare_scalars (include/lare_gpu.h)."""

    _fields_ = [
        ("time", C.c_double),
        ("dt", C.c_double),
        ("dtr", C.c_double),
        ("total_visc_heating", C.c_double),
        ("total_ohmic_heating", C.c_double),
        ("n_s_stages", C.c_int),
        ("peak_substeps", C.c_int),
        ("last_substeps", C.c_int),
        ("steps_taken", C.c_int),
    ]


def default_params(**kw) -> LareParams:
    """Control values of the shipped deck where the hot path reads them
    (src/control.f90:42-206), with gamma = 5/3 (setup.F90:46)."""
    p = LareParams()
    p.gamma = 5.0 / 3.0
    p.visc1 = 0.1
    p.visc2 = 0.5
    p.eta_background = 0.0
    p.eta0 = 0.0
    p.j_max = 1.0e10
    p.kappa_0 = 0.0
    p.flux_limiter = 0.1
    p.ionise_pot = 0.0
    p.xi_n = 0.0
    p.va_max = 10.0
    p.dt_multiplier = 0.9
    p.dt_from_restart = 0.0
    p.kappa_perp_ratio = 0.0
    p.resistive_mhd = 0
    p.conduction = 0
    p.heat_flux_limiter = 1
    p.use_viscous_damping = 0
    p.boris = 0
    p.restart = 0
    for s in ("xbc_min", "xbc_max", "ybc_min", "ybc_max", "zbc_min", "zbc_max"):
        setattr(p, s, BC_PERIODIC)
    p.eos_number = EOS_IDEAL
    p.cowling_resistivity = 0
    p.radiation = 0
    p.rke = 0
    p.cooling_term = 0
    p.alpha_av = 0.05
    p.coronal_heating = 0
    p.mf = 1.2
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def bounds(kind: str, nx: int, ny: int, nz: int):
    """(lo, hi) Fortran bounds of the reference's arrays by staggering."""
    n = (nx, ny, nz)
    if kind == "cell":
        return (-1, -1, -1), (nx + 2, ny + 2, nz + 2)
    if kind == "node":
        return (-2, -2, -2), (nx + 2, ny + 2, nz + 2)
    if kind in ("bx", "by", "bz"):
        d = "xyz".index(kind[1])
        lo = [-1, -1, -1]
        lo[d] = -2
        return tuple(lo), tuple(v + 2 for v in n)
    raise KeyError(kind)


def alloc(kind: str, nx: int, ny: int, nz: int, fill: float = 0.0) -> np.ndarray:
    lo, hi = bounds(kind, nx, ny, nz)
    shape = tuple(h - l + 1 for l, h in zip(lo, hi))
    return np.full(shape, fill, dtype=np.float64, order="F")


STATE_KINDS = {
    "rho": "cell",
    "energy": "cell",
    "vx": "node",
    "vy": "node",
    "vz": "node",
    "bx": "bx",
    "by": "by",
    "bz": "bz",
}


@dataclass
class State:
    """The persistent hot-path state, Fortran-ordered with ghost cells."""

    nx: int
    ny: int
    nz: int
    arrays: Dict[str, np.ndarray] = field(default_factory=dict)

    @classmethod
    def zeros(cls, nx, ny, nz):
        s = cls(nx, ny, nz)
        for name, kind in STATE_KINDS.items():
            s.arrays[name] = alloc(kind, nx, ny, nz)
        return s

    def __getitem__(self, k):
        return self.arrays[k]

    def __setitem__(self, k, v):
        self.arrays[k] = v

    def copy(self):
        return State(self.nx, self.ny, self.nz, {k: v.copy(order="F") for k, v in self.arrays.items()})


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags.f_contiguous:
        raise TypeError("arrays must be float64 Fortran-contiguous")
    return a.ctypes.data_as(C.POINTER(C.c_double))


class LareError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Binding:
    """A context of a library exporting the lare_gpu.h ABI under ``prefix``."""

    def __init__(self, lib: C.CDLL, prefix: str):
        self.lib = lib
        self.prefix = prefix
        dp = C.POINTER(C.c_double)
        f = self._fn
        f("init", [C.POINTER(LareParams), C.c_int, C.c_int, C.c_int] + [dp] * 6 + [C.c_int, C.POINTER(C.c_void_p)], optional_precision=True)
        f("upload", [C.c_void_p] + [dp] * 8)
        f("upload_aux", [C.c_void_p] + [dp] * 4)
        f("set_time", [C.c_void_p, C.c_double, C.c_double])
        f("lagrangian_step", [C.c_void_p, C.c_int])
        f("eulerian_remap", [C.c_void_p, C.c_int])
        f("eta_calc", [C.c_void_p])
        f("boundary_conditions", [C.c_void_p])
        f("step", [C.c_void_p, C.c_int, dp, dp])
        f("conduct_heat", [C.c_void_p, C.c_double, C.POINTER(C.c_int)])
        f("energy", [C.c_void_p, dp])
        f("download", [C.c_void_p] + [dp] * 8)
        f("get_field", [C.c_void_p, C.c_char_p, dp])
        f("set_field", [C.c_void_p, C.c_char_p, dp])
        f("field_bounds", [C.c_void_p, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)])
        f("get_scalars", [C.c_void_p, C.POINTER(LareScalars)])
        le = getattr(lib, prefix + "last_error")
        le.argtypes = [C.c_void_p]
        le.restype = C.c_char_p
        de = getattr(lib, prefix + "destroy")
        de.argtypes = [C.c_void_p]
        de.restype = None
        if hasattr(lib, prefix + "field_device"):
            f("conduct_heat_stages", [C.c_void_p, C.c_double, C.c_int])
            f("conduction_stages", [C.c_void_p, C.c_double, C.POINTER(C.c_int)])
            f("field_device", [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int),
                               C.POINTER(C.c_int), C.POINTER(C.c_int)])
        if hasattr(lib, prefix + "neutral_fraction"):
            f("neutral_fraction", [C.c_void_p])
            f("perpendicular_resistivity", [C.c_void_p])
            f("energy_correction", [C.c_void_p])
        if hasattr(lib, prefix + "run"):
            f("run", [C.c_void_p, C.c_int, C.c_int, C.c_double, C.POINTER(C.c_int), dp, dp])
        if hasattr(lib, prefix + "launch_count"):
            lc = getattr(lib, prefix + "launch_count")
            lc.argtypes = [C.c_void_p]
            lc.restype = C.c_longlong
        if hasattr(lib, prefix + "profile"):
            f("profile", [C.c_void_p, C.c_int])
            pr = getattr(lib, prefix + "profile_report")
            pr.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
            pr.restype = C.c_int

    def _fn(self, name, argtypes, optional_precision=False):
        fn = getattr(self.lib, self.prefix + name)
        if optional_precision and self.prefix != "lare_gpu_":
            argtypes = argtypes[:-2] + argtypes[-1:]
        fn.argtypes = argtypes
        fn.restype = C.c_int

    def call(self, ctx, name, *args):
        rc = getattr(self.lib, self.prefix + name)(ctx, *args)
        if rc != LARE_OK:
            msg = getattr(self.lib, self.prefix + "last_error")(ctx)
            raise LareError(rc, msg.decode() if msg else "")
        return rc


class Simulation:
    """One context (device or oracle) holding a Lare3d state.

    Method names follow the reference's module procedures so that a driver
    loop reads like src/core/lare3d.f90:80-89.
    """

    def __init__(self, binding: Binding, params: LareParams, nx, ny, nz, metrics, precision=64):
        self.b = binding
        self.nx, self.ny, self.nz = nx, ny, nz
        self.params = params
        self.precision = precision
        ctx = C.c_void_p()
        m = [np.ascontiguousarray(metrics[k], dtype=np.float64) for k in ("dxb", "dxc", "dyb", "dyc", "dzb", "dzc")]
        self._metrics = m
        ptrs = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in m]
        fn = getattr(binding.lib, binding.prefix + "init")
        if binding.prefix == "lare_gpu_":
            rc = fn(C.byref(params), nx, ny, nz, *ptrs, precision, C.byref(ctx))
        else:
            rc = fn(C.byref(params), nx, ny, nz, *ptrs, C.byref(ctx))
        if rc != LARE_OK:
            raise LareError(rc, "init failed")
        self.ctx = ctx

    # ---- state transfer
    def upload(self, st: State):
        a = st.arrays
        self.b.call(self.ctx, "upload", *[_ptr(a[k]) for k in ("rho", "energy", "vx", "vy", "vz", "bx", "by", "bz")])

    def upload_aux(self, eta=None, visc3=None, grav=None, gamma_boris=None):
        g = None if grav is None else np.ascontiguousarray(grav, dtype=np.float64)
        self.b.call(self.ctx, "upload_aux", _ptr(eta), _ptr(visc3), None if g is None else g.ctypes.data_as(C.POINTER(C.c_double)), _ptr(gamma_boris))

    def download(self, out: Optional[State] = None) -> State:
        st = out if out is not None else State.zeros(self.nx, self.ny, self.nz)
        a = st.arrays
        self.b.call(self.ctx, "download", *[_ptr(a[k]) for k in ("rho", "energy", "vx", "vy", "vz", "bx", "by", "bz")])
        return st

    def field_bounds(self, name):
        lo = (C.c_int * 3)()
        hi = (C.c_int * 3)()
        self.b.call(self.ctx, "field_bounds", name.encode(), lo, hi)
        return tuple(lo), tuple(hi)

    def get_field(self, name) -> np.ndarray:
        lo, hi = self.field_bounds(name)
        out = np.zeros(tuple(h - l + 1 for l, h in zip(lo, hi)), dtype=np.float64, order="F")
        self.b.call(self.ctx, "get_field", name.encode(), _ptr(out))
        return out

    def set_field(self, name, arr):
        self.b.call(self.ctx, "set_field", name.encode(), _ptr(np.asfortranarray(arr, dtype=np.float64)))

    # ---- hot path
    def set_time(self, time, dt):
        self.b.call(self.ctx, "set_time", C.c_double(time), C.c_double(dt))

    def lagrangian_step(self, step):
        self.b.call(self.ctx, "lagrangian_step", int(step))

    def eulerian_remap(self, step):
        self.b.call(self.ctx, "eulerian_remap", int(step))

    def eta_calc(self):
        self.b.call(self.ctx, "eta_calc")

    def boundary_conditions(self):
        self.b.call(self.ctx, "boundary_conditions")

    def energy_correction(self):
        self.b.call(self.ctx, "energy_correction")

    def neutral_fraction(self):
        self.b.call(self.ctx, "neutral_fraction")

    def perpendicular_resistivity(self):
        self.b.call(self.ctx, "perpendicular_resistivity")

    def step(self, step):
        t = C.c_double()
        d = C.c_double()
        self.b.call(self.ctx, "step", int(step), C.byref(t), C.byref(d))
        return t.value, d.value

    def run(self, first_step, nsteps, t_end=1e30):
        n = C.c_int()
        t = C.c_double()
        d = C.c_double()
        self.b.call(self.ctx, "run", int(first_step), int(nsteps), C.c_double(t_end), C.byref(n), C.byref(t), C.byref(d))
        return n.value, t.value, d.value

    def conduct_heat(self, dt):
        s = C.c_int()
        self.b.call(self.ctx, "conduct_heat", C.c_double(dt), C.byref(s))
        return s.value

    def conduct_heat_stages(self, dt, n_stages):
        self.b.call(self.ctx, "conduct_heat_stages", C.c_double(dt), int(n_stages))

    def conduction_stages(self, dt):
        s = C.c_int()
        self.b.call(self.ctx, "conduction_stages", C.c_double(dt), C.byref(s))
        return s.value

    def field_device(self, name):
        """(device address of Fortran element (0,0,0), sx, sxy, element bytes)."""
        o = C.c_void_p()
        sx, sxy, eb = C.c_int(), C.c_int(), C.c_int()
        self.b.call(self.ctx, "field_device", name.encode(), C.byref(o), C.byref(sx), C.byref(sxy), C.byref(eb))
        return int(o.value or 0), sx.value, sxy.value, eb.value

    def energy(self):
        out = (C.c_double * 5)()
        self.b.call(self.ctx, "energy", out)
        return list(out)

    def scalars(self) -> LareScalars:
        s = LareScalars()
        self.b.call(self.ctx, "get_scalars", C.byref(s))
        return s

    def profile(self, enable: bool):
        self.b.call(self.ctx, "profile", 1 if enable else 0)

    def profile_report(self):
        """Per-launch-site timing: list of dicts sorted by total time."""
        fn = getattr(self.b.lib, self.b.prefix + "profile_report")
        need = fn(self.ctx, None, 0)
        buf = C.create_string_buffer(max(need, 1))
        fn(self.ctx, buf, len(buf))
        out = []
        for line in buf.value.decode().splitlines():
            site, cnt, ms, by, words = line.split("\t")
            out.append({"site": site, "launches": int(cnt), "ms": float(ms), "bytes": float(by), "words": int(words)})
        return out

    def launch_count(self) -> int:
        return int(getattr(self.b.lib, self.b.prefix + "launch_count")(self.ctx))

    def close(self):
        if getattr(self, "ctx", None):
            getattr(self.b.lib, self.b.prefix + "destroy")(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- the reference's initialisation tail (lare3d.f90:65-74)
    def start(self, st: State, eta=None, grav=None, visc3=None, time=0.0, dt=0.0):
        self.upload(st)
        self.upload_aux(eta=eta, grav=grav, visc3=visc3)
        self.set_time(time, dt)
        self.boundary_conditions()
        self.eta_calc()
        if self.params.eos_number not in (0, EOS_IDEAL):
            self.neutral_fraction()
        if self.params.cowling_resistivity:
            self.perpendicular_resistivity()

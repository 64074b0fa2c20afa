"""CPU checks of the drop-in boundary: the product library loads without a
GPU, exports every entry point include/lare_gpu.h declares, and rejects bad
arguments on the host before touching the device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from lare3d_b200 import decks
from lare3d_b200.abi import LareParams, default_params


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"\b(lare_(?:gpu|sur|ens)_\w+)\s*\(", txt)))


def test_exports_every_declared_symbol(built):
    from lare3d_b200 import gpu
    lib = gpu.library()
    names = declared("lare_gpu.h")
    assert len(names) >= 20
    sur = declared("lare_surrogate.h")
    assert len(sur) == 13
    assert {"lare_ens_create", "lare_ens_launch", "lare_ens_sync", "lare_ens_destroy"} <= set(names)
    missing = [n for n in names + sur if not hasattr(lib, n)]
    assert not missing, missing


def test_surrogate_host_side_argument_checks(built):
    """Bad shapes and null pointers are rejected before any launch."""
    from lare3d_b200 import gpu
    lib = gpu.library()
    f = lib.lare_sur_conv
    f.argtypes = [C.c_int] * 4 + [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                  C.c_int, C.c_void_p, C.c_void_p]
    p = C.c_void_p(16)
    assert f(16, 32, 1, 0, None, 24, 0, p, None, p, 22, 1, None, None) == -1      # null input
    assert f(16, 32, 1, 0, p, 24, 0, p, None, p, 21, 1, None, None) == -1         # wrong output edge
    assert f(16, 32, 1, 0, p, 24, 1, p, None, p, 24, 1, None, None) == -1         # pad must be 0 or 2
    assert f(24, 32, 1, 0, p, 24, 0, p, None, p, 22, 1, None, None) == -1         # channel pair
    assert f(32, 8, 0, 1, p, 24, 0, p, None, p, 22, 1, p, None) == -1             # mask with FP32 out
    w = lib.lare_sur_conv_wgrad_work
    w.argtypes = [C.c_int] * 4
    w.restype = C.c_longlong
    assert w(32, 32, 16, 64) == ((16 ** 3 * 64 + 2047) // 2048) * 27 * 32 * 32
    r = lib.lare_sur_recheck
    r.argtypes = [C.c_int, C.c_void_p] + [C.c_int] * 4 + [C.c_void_p] + [C.c_int] * 13 + [C.c_double] * 4 + \
        [C.c_void_p] * 3
    # window (96 columns) narrower than the checked patches (20 + 6 * 16)
    assert r(4, p, 261, 261 * 261, 256, 256, p, 120, 120 * 101, 96, 96, 0, 0, 20, 20, 0, 6, 4, 16, 16,
             5 / 3, 0.0, 0.0, 1e-3, p, p, None) == -1


def test_division_check_argument_checks(built):
    from lare3d_b200 import gpu
    lib = gpu.library()
    f = lib.lare_gpu_check_division
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    p = C.c_void_p(16)
    assert f(p, p, -1, p, None) == -1
    assert f(None, p, 4, p, None) == -1
    assert f(p, p, 4, None, None) == -1
    assert f(None, None, 0, None, None) == 0     # nothing to do, nothing launched


def test_struct_layout_matches_header():
    txt = open(os.path.join(ROOT, "include", "lare_gpu.h")).read()
    body = txt[txt.index("typedef struct lare_params"):txt.index("} lare_params;")]
    fields = re.findall(r"\b(double|int)\s+([\w\s,]+);", body)
    flat = []
    for ty, names in fields:
        for nm in names.split(","):
            flat.append((ty, nm.strip()))
    py = [(("double" if t is C.c_double else "int"), n) for n, t in LareParams._fields_]
    assert flat == py


def test_host_side_argument_checks(built):
    from lare3d_b200 import gpu
    lib = gpu.library()
    d = decks.blast(8)
    out = C.c_void_p()
    m = [np.ascontiguousarray(d.metrics[k]) for k in ("dxb", "dxc", "dyb", "dyc", "dzb", "dzc")]
    ptr = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in m]
    lib.lare_gpu_init.restype = C.c_int
    # n < 4, bad precision, an unknown BC code and a half-periodic direction
    # (open on one side, periodic on the other) are rejected on the host.
    assert lib.lare_gpu_init(C.byref(d.params), 3, 8, 8, *ptr, 64, C.byref(out)) == -1
    assert lib.lare_gpu_init(C.byref(d.params), 8, 8, 8, *ptr, 16, C.byref(out)) == -1
    p = default_params(xbc_min=7, xbc_max=7)
    assert lib.lare_gpu_init(C.byref(p), 8, 8, 8, *ptr, 64, C.byref(out)) == -1
    p = default_params(xbc_min=3)
    assert lib.lare_gpu_init(C.byref(p), 8, 8, 8, *ptr, 64, C.byref(out)) == -1
    # grids whose padded box reaches 2^31 points (32-bit device indices) are
    # refused before the device or the metrics are touched: the smallest
    # such cube, and a thin grid
    assert lib.lare_gpu_init(C.byref(d.params), 1285, 1285, 1285, *ptr, 64, C.byref(out)) == -8
    assert lib.lare_gpu_init(C.byref(d.params), 4, 4, 20000000, *ptr, 32, C.byref(out)) == -8
    assert not out.value
    # calls on a null context fail cleanly
    lib.lare_gpu_eta_calc.restype = C.c_int
    assert lib.lare_gpu_eta_calc(None) == -1
    lib.lare_gpu_last_error.restype = C.c_char_p
    assert lib.lare_gpu_last_error(None) == b"null context"


def test_kiss_matches_restatement(built):
    from lare3d_b200.kiss import seeded
    k = seeded(12345)
    py = np.array([k.random() for _ in range(2000)])
    c = decks.kiss_uniform(12345, 2000)
    assert np.array_equal(py, c)
    assert py.min() >= 0.0 and py.max() < 1.0


def test_grid_metrics():
    from lare3d_b200.grid import grid
    m = grid(8, 8, 8, (0.0, 1.0), (0.0, 2.0), (-1.0, 1.0))
    assert np.allclose(m["dxb"], 1 / 8) and np.allclose(m["dyb"], 2 / 8) and np.allclose(m["dzb"], 2 / 8)
    assert np.allclose(m["dxc"], 1 / 8)
    assert m["xb"][2] == 0.0 and abs(m["xb"][10] - 1.0) < 1e-15
    from lare3d_b200.abi import BC_USER
    u = grid(8, 8, 8, bcs=(BC_USER,) * 3)
    assert abs(u["xb"][0] - (-2 / 8)) < 1e-15   # extrapolated ghost faces


def test_decks_are_consistent(built):
    d = decks.orszag_tang(8)
    for k, a in d.state.arrays.items():
        assert a.flags.f_contiguous and np.isfinite(a).all(), k
    c = decks.conduction(8)
    assert c.dt_fixed > 0 and c.params.conduction == 1


def test_widened_physics_argument_checks(built):
    """lare_gpu_init rejects, on the host and before any device call, an
    unknown EOS code and a partially ionised, Cowling or radiative run
    without its constants; the oracle rejects the EOS code too."""
    from lare3d_b200 import gpu
    from lare3d_b200.abi import EOS_ION
    lib = gpu.library()
    d = decks.blast(8)
    m = [np.ascontiguousarray(d.metrics[k]) for k in ("dxb", "dxc", "dyb", "dyc", "dzb", "dzc")]
    ptr = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in m]
    lib.lare_gpu_init.restype = C.c_int
    out = C.c_void_p()
    bad = [default_params(eos_number=4), default_params(eos_number=-1),
           default_params(eos_number=EOS_ION),                      # no ionisation constants
           default_params(cowling_resistivity=1),                   # likewise
           default_params(radiation=1)]                             # no normalisation
    for p in bad:
        assert lib.lare_gpu_init(C.byref(p), 8, 8, 8, *ptr, 64, C.byref(out)) == -1
        assert not out.value
    c = decks.neutral_constants(EOS_ION)
    ok = default_params(eos_number=EOS_ION, **c)
    assert lib.lare_gpu_init(C.byref(ok), 8, 8, 8, *ptr, 64, C.byref(out)) in (0, -2)   # -2: no device here
    if out.value:
        lib.lare_gpu_destroy(out)
    from oracle import oracle
    rlib = oracle.library()
    rout = C.c_void_p()
    rlib.lare_ref_init.restype = C.c_int
    assert rlib.lare_ref_init(C.byref(default_params(eos_number=5)), 8, 8, 8, *ptr, C.byref(rout)) == -1

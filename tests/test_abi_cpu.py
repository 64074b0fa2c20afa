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
    return sorted(set(re.findall(r"\b(lare_gpu_\w+)\s*\(", txt)))


def test_exports_every_declared_symbol(built):
    from lare3d_b200 import gpu
    lib = gpu.library()
    names = declared("lare_gpu.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


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
    # n < 4, bad precision and unsupported BC_OPEN are rejected on the host.
    assert lib.lare_gpu_init(C.byref(d.params), 3, 8, 8, *ptr, 64, C.byref(out)) == -1
    assert lib.lare_gpu_init(C.byref(d.params), 8, 8, 8, *ptr, 16, C.byref(out)) == -1
    p = default_params(xbc_min=3)
    assert lib.lare_gpu_init(C.byref(p), 8, 8, 8, *ptr, 64, C.byref(out)) == -1
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

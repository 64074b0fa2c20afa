"""ctypes loader for the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It exposes the oracle through the same Simulation interface as
the device library so a parity test drives both with identical calls.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from lare3d_b200.abi import Binding, Simulation

HERE = os.path.dirname(os.path.abspath(__file__))
_libs = {}


def build(quiet=True):
    """Compile the oracle with its Makefile (gcc/g++ only)."""
    out = subprocess.run(["make", "-C", HERE, "all"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def library(checked: bool = False) -> C.CDLL:
    name = "liblare_ref_chk.so" if checked else "liblare_ref.so"
    if name not in _libs:
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            build()
        _libs[name] = C.CDLL(path)
    return _libs[name]


def binding(checked: bool = False) -> Binding:
    lib = library(checked)
    b = Binding(lib, "lare_ref_")
    lib.lare_ref_num_threads.restype = C.c_int
    return b


def num_threads() -> int:
    return int(library().lare_ref_num_threads())


def simulation(deck, checked: bool = False) -> Simulation:
    return Simulation(binding(checked), deck.params, deck.nx, deck.ny, deck.nz, deck.metrics)

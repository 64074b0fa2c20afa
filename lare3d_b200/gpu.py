"""Loader for the sm_100a engine (``liblare_gpu.so``).

This is the product path: it binds only the CUDA library.  There is no CPU
fallback; without the built library or a GPU, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os

from .abi import Binding, Simulation

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblare_gpu.so")
_lib = None


def library() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m lare3d_b200.build`")
        _lib = C.CDLL(LIB_PATH)
        _lib.lare_gpu_stream.argtypes = [C.c_void_p]
        _lib.lare_gpu_stream.restype = C.c_void_p
    return _lib


def binding() -> Binding:
    return Binding(library(), "lare_gpu_")


# Precision codes of lare_gpu_init (include/lare_gpu.h).
FP64 = 64        # FP64 drop-in (product): FMA contraction, shared reciprocals
EXACT64 = 65     # FP64 with the reference's arithmetic, bit for bit
FP32 = 32        # FP32 form


def simulation(deck, precision: int = FP64) -> Simulation:
    """A device context holding ``deck``'s grid and control parameters."""
    return Simulation(binding(), deck.params, deck.nx, deck.ny, deck.nz, deck.metrics, precision=precision)


def stream_of(sim: Simulation) -> int:
    """cudaStream_t of a context (as an integer handle)."""
    return int(library().lare_gpu_stream(sim.ctx) or 0)

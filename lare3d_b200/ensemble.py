"""Batched ensembles: many independent blast / Orszag-Tang runs of uneven grid
sizes advanced together by one CUDA graph launch per 6 steps (lare_ens_* in
include/lare_gpu.h), with the block shape of every member's point kernels
chosen by a measuring autotuner.

The reference runs one simulation per MPI job; an ensemble has no
counterpart there.  Each member is an ordinary context (the FP32 form by
default), so every member's result is that of the same run stepped alone,
bit for bit (checked by the tests).  Member states also serve as
conduction inputs for the surrogate's training pairs (``snapshot_pairs``).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import decks, gpu
from .abi import LARE_OK, LareError

# Block shapes (bx, by) the autotuner tries for the point kernels.
BLOCKS = ((32, 4), (64, 4), (128, 2), (32, 8), (64, 2), (128, 1), (256, 1), (32, 2))
STEPS_PER_LAUNCH = 6   # the remap's sweep-order period (remap.f90)


def _lib():
    lib = gpu.library()
    if not getattr(lib, "_ens_bound", False):
        v, i = C.c_void_p, C.c_int
        lib.lare_ens_create.argtypes = [C.POINTER(v), i, i, C.POINTER(v)]
        lib.lare_ens_create.restype = i
        lib.lare_ens_launch.argtypes = [v, i]
        lib.lare_ens_launch.restype = i
        lib.lare_ens_sync.argtypes = [v, C.POINTER(i)]
        lib.lare_ens_sync.restype = i
        lib.lare_ens_stream.argtypes = [v]
        lib.lare_ens_stream.restype = v
        lib.lare_ens_destroy.argtypes = [v]
        lib.lare_ens_destroy.restype = None
        lib.lare_gpu_set_block.argtypes = [v, i, i]
        lib.lare_gpu_set_block.restype = i
        lib._ens_bound = True
    return lib


def set_block(sim, bx, by):
    rc = _lib().lare_gpu_set_block(sim.ctx, int(bx), int(by))
    if rc != LARE_OK:
        raise LareError(rc, "set_block")


# ---------------------------------------------------------------------------
# Members

@dataclass
class MemberSpec:
    kind: str        # "blast" or "orszag_tang"
    n: int
    beta: float      # plasma beta 2p/B^2 of the background
    eta: float       # eta_background (resistive)
    seed: int


def member_specs(count=48, seed=2024, n_min=32, n_max=128, step=8, beta=(0.01, 10.0), eta=(1e-4, 1e-2)):
    """A seeded mix: kind 50/50, edge uniform over multiples of `step` in
    [n_min, n_max], beta and eta log-uniform over the given ranges."""
    rng = np.random.default_rng(seed)
    sizes = np.arange(n_min, n_max + 1, step)
    out = []
    for i in range(count):
        kind = "blast" if rng.random() < 0.5 else "orszag_tang"
        n = int(rng.choice(sizes))
        b = float(math.exp(rng.uniform(math.log(beta[0]), math.log(beta[1]))))
        e = float(math.exp(rng.uniform(math.log(eta[0]), math.log(eta[1]))))
        out.append(MemberSpec(kind, n, b, e, int(rng.integers(1, 1 << 30))))
    return out


def member_deck(spec: MemberSpec):
    """The deck of one member: the blast or Orszag-Tang deck at edge n, its
    field scaled to the requested background beta, resistive with eta."""
    if spec.kind == "blast":
        d = decks.blast(spec.n, resistive_mhd=1, eta_background=spec.eta, eta0=0.0, j_max=1.0e10)
        beta0 = 2.0 * 0.1 / 1.0                        # p = 0.1, |B| = 1
    elif spec.kind == "orszag_tang":
        d = decks.orszag_tang(spec.n, seed=spec.seed % 100000 + 1, eta_background=spec.eta)
        p0 = 5.0 / (12.0 * math.pi)
        beta0 = 2.0 * p0 / (3.0 / (8.0 * math.pi))     # <|B|^2> = 3 / (8 pi)
    else:
        raise ValueError(spec.kind)
    s = math.sqrt(beta0 / spec.beta)
    for k in ("bx", "by", "bz"):
        d.state[k][...] *= s
    d.info.update({"beta": spec.beta, "eta": spec.eta, "kind": spec.kind})
    return d


# ---------------------------------------------------------------------------
# The ensemble

class Ensemble:
    """Contexts for every deck, one eager step each, then one graph per
    launch of STEPS_PER_LAUNCH steps of all members."""

    def __init__(self, deck_list: Sequence, precision=32, blocks: Optional[Dict[int, Tuple[int, int]]] = None,
                 fields: Optional[Dict[int, Dict[str, np.ndarray]]] = None):
        self.decks = list(deck_list)
        self.sims = []
        for i, d in enumerate(self.decks):
            s = gpu.simulation(d, precision=precision)
            s.start(d.state)
            for name, arr in ((fields or {}).get(i) or {}).items():  # e.g. a member's heat_in
                s.set_field(name, arr)
            if blocks and d.nx in blocks:
                set_block(s, *blocks[d.nx])
            self.sims.append(s)
        for s in self.sims:
            s.step(1)                  # first-call set-up happens eagerly
        self.steps = 1
        arr = (C.c_void_p * len(self.sims))(*[s.ctx.value for s in self.sims])
        h = C.c_void_p()
        rc = _lib().lare_ens_create(arr, len(self.sims), STEPS_PER_LAUNCH, C.byref(h))
        if rc != LARE_OK:
            self.close()
            raise LareError(rc, "lare_ens_create")
        self.h = h

    @property
    def stream(self) -> int:
        return int(_lib().lare_ens_stream(self.h) or 0)

    def launch(self, nlaunch=1):
        rc = _lib().lare_ens_launch(self.h, int(nlaunch))
        if rc != LARE_OK:
            raise LareError(rc, "lare_ens_launch")
        self.steps += nlaunch * STEPS_PER_LAUNCH

    def sync(self):
        bad = C.c_int(-1)
        rc = _lib().lare_ens_sync(self.h, C.byref(bad))
        if rc != LARE_OK:
            raise LareError(rc, f"ensemble member {bad.value}")

    def cells(self) -> int:
        return sum(d.nx * d.ny * d.nz for d in self.decks)

    def close(self):
        if getattr(self, "h", None):
            _lib().lare_ens_destroy(self.h)
            self.h = None
        for s in self.sims:
            s.close()
        self.sims = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(n, precision=32, blocks=BLOCKS, launches=2, kind="orszag_tang"):
    """Time one graph launch of a scratch member of edge n for every block
    shape; return (best shape, {shape: ms per step})."""
    import torch
    spec = MemberSpec(kind, n, 1.0, 1e-3, 1)
    times = {}
    for bx, by in blocks:
        d = member_deck(spec)
        e = Ensemble([d], precision=precision, blocks={n: (bx, by)})
        st = torch.cuda.ExternalStream(e.stream)
        e.launch(1)                                  # warm-up
        e.sync()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        e.launch(launches)
        b.record(st)
        e.sync()
        times[(bx, by)] = a.elapsed_time(b) / (launches * STEPS_PER_LAUNCH)
        e.close()
    best = min(times, key=times.get)
    return best, times


def autotune_sizes(sizes, precision=32):
    """Best block shape per distinct edge."""
    return {n: autotune(n, precision)[0] for n in sorted(set(sizes))}


def snapshot_pairs(ens: Ensemble, members, dt_ratio=50.0, kappa_0=1.0e-3, meta=None):
    """Conduction before/after pairs from ensemble member states: each member
    state (rho, energy, B) is loaded into a conduction context of the same
    grid and advanced by one plain RKL2 step of dt_ratio x its explicit
    limit.  Returns [(features [5][n][n][n], dT [n][n][n])] on the device."""
    import torch
    from . import surrogate as S
    from .abi import BC_PERIODIC
    meta = meta or {"t_scale": 0.1, "rho_scale": 1.0}
    out = []
    for i in members:
        d = ens.decks[i]
        st = ens.sims[i].download()
        p = decks.default_params(gamma=d.params.gamma, conduction=1, heat_flux_limiter=1, flux_limiter=0.1,
                                 kappa_0=kappa_0, dt_multiplier=0.9)
        cd = decks.Deck(d.name + "_conduction", p, d.nx, d.ny, d.nz, d.metrics, st, nsteps=1)
        dt = dt_ratio * decks.dt_parab_estimate(st, d.metrics, p, d.nx)
        sim = gpu.simulation(cd, precision=32)
        sim.start(st)
        n = d.nx
        feat = torch.empty((5, n, n, n), dtype=torch.float32, device="cuda")
        dT = torch.empty((n, n, n), dtype=torch.float32, device="cuda")
        S.extract(sim, feat, dT, 0, meta)
        sim.conduct_heat(dt)
        S.extract(sim, None, dT, 1, meta)
        torch.cuda.synchronize()
        sim.close()
        out.append((feat, dT))
    return out

"""Learned conduction surrogate (the "learned form" beside the plain RKL2 step).

A 4-layer 3-D convolutional network (3^3 kernels, 32 channels, bf16 weights
and activations, FP32 accumulation) maps a window of (T, rho, b-hat) to the
temperature change of one RKL2 conduction step (conduct.f90:299-416) of a
fixed dt on the window's centre.  Everything that touches data runs in the
kernels of ``csrc/surrogate.cu`` (include/lare_surrogate.h); this module
holds the orchestration:

* ``Network``     - master FP32 weights, Adam state, bf16 packed copies,
                    forward / backward / train_step over device buffers;
* ``generate``    - before/after pairs produced by the GPU engine's own RKL2
                    on seeded conduction decks;
* ``train``       - minibatch training on random windows of those pairs;
* ``SurrogateConduction`` - one conduction step of a resident state by the
                    network, with a sampled column of 16^3 patches re-run by
                    plain RKL2 in a window engine; a re-checked patch whose
                    relative temperature error exceeds the bound is replaced
                    by the RKL2 result (patch-wise rejection), and a step in
                    which more than ``fallback_fraction`` of the checked
                    patches are rejected is redone by plain RKL2 for the whole
                    grid (fallback).

The surrogate has no counterpart in the reference; plain RKL2 arbitrates its accuracy.
torch supplies device memory and streams only.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import gpu
from .abi import BC_USER, EOS_IDEAL, LARE_OK, LareError

# (cin padded, cout of the master weights, cin used, cout used by the forward)
LAYERS = ((16, 32, 7, 32), (32, 32, 32, 32), (32, 32, 32, 32), (32, 16, 32, 1))
HALO = 4                 # cells trimmed per face by the four valid convolutions
PATCH = 16               # edge of a re-check / rejection patch
TRAIN_WIN = PATCH + 2 * HALO
INFER_PATCH = 64         # edge of the centre of one inference window
PRED_C = LAYERS[-1][3]   # channels of the FP32 output (channel 0 is dT)
GRAD_C = LAYERS[-1][1]   # channels of the output gradient


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the learned conduction surrogate needs a CUDA device")
    return torch


class _Lib:
    """ctypes view of include/lare_surrogate.h in liblare_gpu.so."""

    def __init__(self):
        lib = gpu.library()
        v, i, d, f, ll = C.c_void_p, C.c_int, C.c_double, C.c_float, C.c_longlong
        sig = {
            "conv": [i, i, i, i, v, i, i, v, v, v, i, i, v, v],
            "conv_wgrad": [i, i, v, v, i, i, i, v, v, v, v],
            "mse": [v, i, v, ll, i, v, v, v, v],
            "adam": [v, v, v, v, i, f, f, f, f, i, v],
            "pack": [v, i, i, i, v, v, v],
            "extract": [i, v, v, v, v, v, i, i, i, i, i, d, d, d, f, f, v, v, i, v],
            "gather": [v, i, i, i, v, i, i, i, v, v, f, v, v],
            "apply": [i, v, i, i, i, i, i, v, i, v, i, i, i, d, v],
            "copy_column": [i, v, i, i, i, i, v, i, i, i, i, i, i, i, i, v],
            "recheck": [i, v, i, i, i, i, v, i, i, i, i, i, i, i, i, i, i, i, i, i, d, d, d, d, v, v, v],
        }
        for name, args in sig.items():
            fn = getattr(lib, "lare_sur_" + name)
            fn.argtypes = args
            fn.restype = C.c_int
            setattr(self, name, self._checked(fn, name))
        w = lib.lare_sur_conv_wgrad_work
        w.argtypes = [i, i, i, i]
        w.restype = ll
        self.wgrad_work = w
        lib.lare_sur_set_engine.argtypes = [i]
        lib.lare_sur_set_engine.restype = i
        lib.lare_sur_status.argtypes = [i]
        lib.lare_sur_status.restype = i
        self.set_engine = lambda tc: lib.lare_sur_set_engine(1 if tc else 0)
        self.status = lambda clear=True: lib.lare_sur_status(1 if clear else 0)

    @staticmethod
    def _checked(fn, name):
        def call(*a):
            rc = fn(*a)
            if rc != LARE_OK:
                raise LareError(rc, "lare_sur_" + name)
        return call


_LIB = None


def lib() -> _Lib:
    global _LIB
    if _LIB is None:
        _LIB = _Lib()
    return _LIB


def _p(t) -> int:
    return t.data_ptr()


class Network:
    """Weights, optimiser state and device buffers of the surrogate network.

    Master weights of layer l are FP32 [27][cout][cin] (cout, cin from
    ``LAYERS``; padded channels stay exactly zero because their gradients
    are zero), followed by the FP32 bias [cout], in one flat vector so that
    one Adam launch updates everything.
    """

    def __init__(self, seed: int = 0, stream: Optional[int] = None):
        torch = _torch()
        self.torch = torch
        self.stream = stream
        self.wo, self.bo = [], []
        o = 0
        for cin, cout, _cr, _cf in LAYERS:
            self.wo.append(o)
            o += 27 * cout * cin
            self.bo.append(o)
            o += cout
        self.n = o
        flat = np.zeros(o, np.float32)
        rng = np.random.default_rng(seed)
        for l, (cin, cout, cin_r, _cf) in enumerate(LAYERS):
            last = l == len(LAYERS) - 1
            cout_r = 1 if last else cout
            std = math.sqrt(2.0 / (27.0 * cin_r)) * (0.1 if last else 1.0)
            w = np.zeros((27, cout, cin), np.float32)
            w[:, :cout_r, :cin_r] = (rng.standard_normal((27, cout_r, cin_r)) * std).astype(np.float32)
            flat[self.wo[l]:self.wo[l] + w.size] = w.ravel()
        dev = torch.device("cuda")
        self.p = torch.from_numpy(flat).to(dev)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.t = 0
        self.wf = [torch.empty(27 * cf * cin, dtype=torch.bfloat16, device=dev) for cin, _c, _r, cf in LAYERS]
        self.wb = [torch.empty(27 * cin * cout, dtype=torch.bfloat16, device=dev) for cin, cout, _r, _f in LAYERS]
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
        self.meta = {"t_scale": 0.1, "rho_scale": 1.0, "dt_scale": 1.0, "dt": 0.0}
        self._bufs = {}
        self._packed = False

    # -- parameters
    def weights(self, l):
        cin, cout, _r, _f = LAYERS[l]
        return self.p[self.wo[l]:self.wo[l] + 27 * cout * cin].view(27, cout, cin)

    def bias(self, l):
        return self.p[self.bo[l]:self.bo[l] + LAYERS[l][1]]

    def wgrad(self, l):
        cin, cout, _r, _f = LAYERS[l]
        return self.g[self.wo[l]:self.wo[l] + 27 * cout * cin].view(27, cout, cin)

    def bgrad(self, l):
        return self.g[self.bo[l]:self.bo[l] + LAYERS[l][1]]

    def set_params(self, W, B):
        """Load weights [27][cout][cin] and biases (numpy) of every layer."""
        torch = self.torch
        for l in range(len(LAYERS)):
            self.weights(l).copy_(torch.from_numpy(np.asarray(W[l], np.float32)))
            self.bias(l).copy_(torch.from_numpy(np.asarray(B[l], np.float32)))
        self._packed = False

    def pack(self):
        L = lib()
        for l, (cin, cout, _r, cf) in enumerate(LAYERS):
            L.pack(_p(self.p) + 4 * self.wo[l], cin, cout, cf, _p(self.wf[l]), _p(self.wb[l]), self.stream)
        self._packed = True

    def save(self, path):
        meta = {k: np.float64(v) for k, v in self.meta.items()}
        np.savez(path, params=self.p.detach().cpu().numpy(), **meta)

    def load(self, path):
        z = np.load(path)
        p = z["params"].astype(np.float32)
        if p.size != self.n:
            raise ValueError(f"{path}: {p.size} parameters, expected {self.n}")
        self.p.copy_(self.torch.from_numpy(p))
        for k in self.meta:
            if k in z:
                self.meta[k] = float(z[k])
        self._packed = False

    # -- device buffers for a batch of nb windows of edge win
    def buffers(self, nb, win, train):
        key = (nb, win, train)
        b = self._bufs.get(key)
        if b is not None:
            return b
        torch = self.torch
        dev = torch.device("cuda")
        bf = torch.bfloat16
        d = [win - 2 * k for k in range(5)]       # edges: x, a1, a2, a3, out
        b = {"x": torch.empty(nb * d[0] ** 3 * 16, dtype=bf, device=dev)}
        for l in range(3):
            b[f"a{l + 1}"] = torch.empty(nb * d[l + 1] ** 3 * 32, dtype=bf, device=dev)
        b["out"] = torch.empty(nb * d[4] ** 3 * PRED_C, dtype=torch.float32, device=dev)
        if train:
            b["tgt"] = torch.empty(nb * d[4] ** 3, dtype=torch.float32, device=dev)
            b["dy4"] = torch.empty(nb * d[4] ** 3 * GRAD_C, dtype=bf, device=dev)
            for l in (3, 2, 1):
                b[f"dz{l}"] = torch.empty(nb * d[l] ** 3 * 32, dtype=bf, device=dev)
            L = lib()
            work = max(L.wgrad_work(cin, cout, d[l + 1], nb) for l, (cin, cout, _r, _f) in enumerate(LAYERS))
            b["work"] = torch.empty(max(work, nb * d[4] ** 3 // 256 + 1), dtype=torch.float32, device=dev)
        b["d"] = d
        self._bufs[key] = b
        return b

    def forward(self, b, nb):
        """Forward pass on b["x"] (already gathered); output in b["out"]."""
        if not self._packed:
            self.pack()
        L = lib()
        d = b["d"]
        src = b["x"]
        for l in range(4):
            cin, cout, _r, cf = LAYERS[l]
            last = l == 3
            dst = b["out"] if last else b[f"a{l + 1}"]
            L.conv(cin, cf, 0 if last else 1, 1 if last else 0, _p(src), d[l], 0, _p(self.wf[l]),
                   _p(self.p) + 4 * self.bo[l], _p(dst), d[l + 1], nb, None, self.stream)
            src = dst

    def backward(self, b, nb):
        """Gradients of the MSE of b["out"] against b["tgt"] into self.g."""
        L = lib()
        d = b["d"]
        count = nb * d[4] ** 3
        L.mse(_p(b["out"]), PRED_C, _p(b["tgt"]), count, GRAD_C, _p(self.loss), _p(b["dy4"]), _p(b["work"]),
              self.stream)
        dy = b["dy4"]
        acts = [b["x"], b["a1"], b["a2"], b["a3"]]
        for l in (3, 2, 1, 0):
            cin, cout, _r, _f = LAYERS[l]
            L.conv_wgrad(cin, cout, _p(dy), _p(acts[l]), d[l], d[l + 1], nb, _p(b["work"]),
                         _p(self.g) + 4 * self.wo[l], _p(self.g) + 4 * self.bo[l], self.stream)
            if l > 0:
                # dL/d(pre-activation of layer l-1) = full conv of dy with the
                # flipped weights, masked by the ReLU of that layer's output
                L.conv(cout, cin, 0, 0, _p(dy), d[l + 1], 2, _p(self.wb[l]), None, _p(b[f"dz{l}"]), d[l], nb,
                       _p(acts[l]), self.stream)
                dy = b[f"dz{l}"]

    def adam(self, lr, b1=0.9, b2=0.999, eps=1e-8):
        self.t += 1
        lib().adam(_p(self.p), _p(self.g), _p(self.m), _p(self.v), self.n, lr, b1, b2, eps, self.t, self.stream)
        self._packed = False

    def train_step(self, b, nb, lr):
        self.forward(b, nb)
        self.backward(b, nb)
        self.adam(lr)


# ---------------------------------------------------------------------------
# Training data: before/after pairs of the engine's own RKL2.

def _fields(sim):
    return {k: sim.field_device(k) for k in ("energy", "rho", "bx", "by", "bz")}


def extract(sim, feat, tout, tmode, meta, stream=None):
    """Feature extraction from a resident state (see lare_sur_extract)."""
    f = _fields(sim)
    e, sx, sxy, eb = f["energy"]
    p = sim.params
    lib().extract(eb, e, f["rho"][0], f["bx"][0], f["by"][0], f["bz"][0], sx, sxy, sim.nx, sim.ny, sim.nz,
                  p.gamma, p.xi_n, p.ionise_pot, meta["t_scale"], meta["rho_scale"],
                  None if feat is None else _p(feat), None if tout is None else _p(tout), tmode,
                  stream if stream is not None else gpu.stream_of(sim))


def generate(seeds, n=256, steps=4, dt=None, precision=32, meta=None, log=None):
    """Run the conduction deck for every seed and keep, per RKL2 step, the
    features before the step and dT = T_after - T_before.

    Returns (store [S][5][n][n][n], dT [S][n][n][n], dt) on the device; dt is
    the first seed's workload dt unless given, and every step uses it.
    """
    from . import decks
    torch = _torch()
    meta = meta or {"t_scale": 0.1, "rho_scale": 1.0}
    S = len(seeds) * steps
    store = torch.empty((S, 5, n, n, n), dtype=torch.float32, device="cuda")
    dT = torch.empty((S, n, n, n), dtype=torch.float32, device="cuda")
    idx = 0
    for seed in seeds:
        t0 = time.time()
        d = decks.conduction(n, seed=int(seed))
        if dt is None:
            dt = d.dt_fixed
        sim = gpu.simulation(d, precision=precision)
        sim.start(d.state)
        for _ in range(steps):
            extract(sim, store[idx], dT[idx], 0, meta)
            sim.conduct_heat(dt)
            extract(sim, None, dT[idx], 1, meta)
            idx += 1
        torch.cuda.synchronize()
        sim.close()
        if log:
            log(f"seed {seed}: {steps} RKL2 steps at {n}^3 in {time.time() - t0:.1f} s")
    return store, dT, dt


def train(net: Network, store, dT, iters, nb=64, lr=1e-3, seed=0, log=None, log_every=200, lr_decay=True,
          active_fraction=0.5, active_quantile=0.9):
    """Minibatch training on random training windows of the pairs.

    Window origins are drawn so that the predicted 16^3 centre lies inside
    the grid in z (x and y wrap).  Conduction changes T appreciably only
    near the hot spots, so a fraction ``active_fraction`` of every batch is
    drawn around the 16^3 tiles whose max |dT| is above the
    ``active_quantile`` quantile of all tiles (origins jittered by up to
    half a tile); the rest is uniform.  Returns the loss history
    [(iteration, loss)]."""
    torch = _torch()
    S = store.shape[0]
    nz, ny, nx = store.shape[2:]
    rng = np.random.default_rng(seed)
    b = net.buffers(nb, TRAIN_WIN, True)
    o = np.stack([rng.integers(0, S, (iters, nb)), rng.integers(0, nx, (iters, nb)),
                  rng.integers(0, ny, (iters, nb)), rng.integers(-HALO, nz - PATCH - HALO + 1, (iters, nb))],
                 axis=2).astype(np.int64)
    na = int(round(active_fraction * nb))
    if na > 0 and nz % PATCH == 0 and ny % PATCH == 0 and nx % PATCH == 0:
        act = dT.abs().view(S, nz // PATCH, PATCH, ny // PATCH, PATCH, nx // PATCH, PATCH).amax(dim=(2, 4, 6))
        thr = torch.quantile(act.flatten().float()[:1 << 24], active_quantile)
        tiles = (act > thr).nonzero().cpu().numpy()          # (s, pz, py, px)
        if len(tiles):
            pick = tiles[rng.integers(0, len(tiles), (iters, na))]
            jit = rng.integers(-PATCH // 2, PATCH // 2 + 1, (iters, na, 3))
            o[:, :na, 0] = pick[..., 0]
            o[:, :na, 1] = pick[..., 3] * PATCH - HALO + jit[..., 0]
            o[:, :na, 2] = pick[..., 2] * PATCH - HALO + jit[..., 1]
            o[:, :na, 3] = np.clip(pick[..., 1] * PATCH - HALO + jit[..., 2], -HALO, nz - PATCH - HALO)
    org = torch.from_numpy(o.astype(np.int32)).to("cuda")
    torch.cuda.synchronize()
    scale = 1.0 / net.meta["dt_scale"]
    hist = []
    L = lib()
    for it in range(iters):
        L.gather(_p(store), nx, ny, nz, _p(org[it]), nb, TRAIN_WIN, HALO, _p(b["x"]), _p(dT), scale, _p(b["tgt"]),
                 net.stream)
        rate = lr * (0.5 * (1.0 + math.cos(math.pi * it / iters)) if lr_decay else 1.0)
        net.train_step(b, nb, rate)
        if it == 0 or (it + 1) % log_every == 0 or it == iters - 1:
            v = float(net.loss.item())
            hist.append((it + 1, v))
            if log:
                log(f"iter {it + 1}: loss {v:.4e}")
    return hist


def dt_scale_of(dT) -> float:
    """Output normalisation: the RMS of dT over the training pairs."""
    return float(dT.double().pow(2).mean().sqrt().item()) or 1.0


# ---------------------------------------------------------------------------
# The surrogate conduction step.

def window_metrics(metrics, n, x0, wn, axis):
    """Metric arrays of a window of wn cells starting at grid cell x0 (0-based)
    of a periodic axis: every Fortran index i of the window reads the grid's
    value at ((x0 + i - 1) mod n) + 1."""
    out = {}
    for name, lo, hi_off in (("d%sb" % axis, -1, 2), ("d%sc" % axis, -1, 1)):
        g = metrics[name]
        w = np.empty(wn + hi_off - lo + 1)
        for i in range(lo, wn + hi_off + 1):
            gi = ((x0 + i - 1) % n) + 1
            w[i - lo] = g[gi - lo]
        out[name] = w
    return out


@dataclass
class StepInfo:
    stages: int = 0
    checked: int = 0
    rejected: int = 0
    max_err: float = 0.0
    fallback: bool = False
    column: tuple = (0, 0)
    errs: Optional[np.ndarray] = None


class SurrogateConduction:
    """Conduction steps of dt on a resident FP32/FP64 state, by the network.

    Each step: the grid's RKL2 stage count s (calc_s_stages); features of the
    state; the network on 72^3 windows whose 64^3 centres tile the grid; dT
    applied to the energy.  Meanwhile, on the window engine's own stream, one
    full-height column of (col x col) cells plus a halo of at least s + 2
    cells per side in x and y is re-run by plain RKL2 with the same s: the
    error of RKL2 on a truncated window moves in by one cell per stage (the
    stencil and the Larsen factor reach one cell each), so the column's
    result is the whole-grid RKL2 result there.  Every 16^3 patch of the
    column whose max relative temperature error exceeds ``bound`` is replaced
    by the RKL2 values (patch-wise rejection); if more than
    ``fallback_fraction`` of the column's patches are rejected, the step is
    redone by plain RKL2 on the whole grid (fallback).  The checked column
    moves every step (seeded).  With col = 64 on a 256^3 grid the check
    covers 1/16 of the patches (6.25%).

    The window engine's metrics are those of the column at x = y = 0; on a
    uniform periodic axis whose spacing is a power of two (the 256^3 unit
    box) every column has bit-identical metrics.
    """

    def __init__(self, sim, deck, net: Network, dt, bound=1e-3, col=64, fallback_fraction=0.5, seed=0,
                 check=True):
        if sim.params.eos_number not in (0, EOS_IDEAL):
            # the network and its re-check take T with one xi_n for the whole grid
            raise ValueError("the conduction surrogate needs EOS_IDEAL (a constant neutral fraction)")
        torch = _torch()
        self.torch = torch
        self.sim, self.deck, self.net, self.dt = sim, deck, net, float(dt)
        self.bound, self.col, self.fallback_fraction = float(bound), int(col), float(fallback_fraction)
        self.check = check
        if sim.nx % INFER_PATCH or sim.ny % INFER_PATCH or sim.nz % INFER_PATCH:
            raise ValueError("grid edges must be multiples of 64")
        if self.col % PATCH or sim.nx % self.col or sim.ny % self.col:
            raise ValueError("column edge must be a multiple of 16 dividing nx and ny")
        self.stream = gpu.stream_of(sim)
        net.stream = self.stream
        self.rng = np.random.default_rng(seed)
        nxw, nyw, nzw = sim.nx // INFER_PATCH, sim.ny // INFER_PATCH, sim.nz // INFER_PATCH
        self.nb = nxw * nyw * nzw
        o = [(0, x * INFER_PATCH - HALO, y * INFER_PATCH - HALO, z * INFER_PATCH - HALO)
             for z in range(nzw) for y in range(nyw) for x in range(nxw)]
        self.org = torch.tensor(o, dtype=torch.int32, device="cuda")
        self.feat = torch.empty((1, 5, sim.nz, sim.ny, sim.nx), dtype=torch.float32, device="cuda")
        self.bufs = net.buffers(self.nb, INFER_PATCH + 2 * HALO, False)
        self.win = None
        self.halo_w = 0
        self.err = torch.zeros((self.col // PATCH) ** 2 * (sim.nz // PATCH), dtype=torch.float32, device="cuda")
        self.nrej = torch.zeros(1, dtype=torch.int32, device="cuda")
        p = sim.params
        self.out_scale = net.meta["dt_scale"] * (2.0 - p.xi_n) / (p.gamma - 1.0)
        _e, sx, sxy, eb = sim.field_device("energy")
        self.eb = eb
        dt_ = torch.float32 if eb == 4 else torch.float64
        self.energy0 = torch.empty(sxy * (sim.nz + 5), dtype=dt_, device="cuda")
        self.e0_origin = _p(self.energy0) + eb * (2 + 2 * sx + 2 * sxy)

    def close(self):
        if self.win is not None:
            self.win.close()
            self.win = None

    def _window(self, s):
        """(Re)build the window engine for a halo of at least s + 2 cells."""
        need = s + 2
        if self.win is not None and self.halo_w >= need:
            return
        self.close()
        from .abi import Simulation
        h = max(need, 16)
        wn = self.col + 2 * h
        p = self.deck.params
        wp = type(p)()
        C.memmove(C.byref(wp), C.byref(p), C.sizeof(p))
        wp.xbc_min = wp.xbc_max = wp.ybc_min = wp.ybc_max = BC_USER
        m = dict(self.deck.metrics)
        m.update(window_metrics(self.deck.metrics, self.sim.nx, 0, wn, "x"))
        m.update(window_metrics(self.deck.metrics, self.sim.ny, 0, wn, "y"))
        self.win = Simulation(gpu.binding(), wp, wn, wn, self.sim.nz, m,
                              precision=getattr(self.sim, "precision", 32 if self.eb == 4 else 64))
        self.halo_w = h
        self.wn = wn

    def _copy_energy(self, to_saved):
        """energy <-> the saved copy (whole padded box, periodic x and y)."""
        sim = self.sim
        e, sx, sxy, eb = sim.field_device("energy")
        a, b = (e, self.e0_origin) if to_saved else (self.e0_origin, e)
        src = (C.c_void_p * 1)(a)
        dst = (C.c_void_p * 1)(b)
        lib().copy_column(eb, src, sx, sxy, sim.nx, sim.ny, dst, sx, sxy, sim.nx, sim.ny, sim.nz, 0, 0, 1,
                          self.stream)

    def step(self) -> StepInfo:
        torch = self.torch
        sim, L = self.sim, lib()
        info = StepInfo()
        s = sim.conduction_stages(self.dt)
        info.stages = s
        e, sx, sxy, eb = sim.field_device("energy")
        if self.check:
            self._window(s)
            ncx, ncy = sim.nx // self.col, sim.ny // self.col
            cx, cy = int(self.rng.integers(0, ncx)), int(self.rng.integers(0, ncy))
            info.column = (cx, cy)
            x0, y0 = cx * self.col - self.halo_w, cy * self.col - self.halo_w
            fs, fw = _fields(sim), _fields(self.win)
            names = ("energy", "rho", "bx", "by", "bz")
            src = (C.c_void_p * 5)(*[fs[k][0] for k in names])
            dst = (C.c_void_p * 5)(*[fw[k][0] for k in names])
            _w, wsx, wsxy, _ = fw["energy"]
            L.copy_column(eb, src, sx, sxy, sim.nx, sim.ny, dst, wsx, wsxy, self.wn, self.wn, sim.nz, x0, y0, 5,
                          self.stream)
            self._copy_energy(True)
            torch.cuda.synchronize()
            # queued on the window engine's stream; overlaps the network below
            self.win.boundary_conditions()
            self.win.conduct_heat_stages(self.dt, s)
        extract(sim, self.feat[0], None, 0, self.net.meta, self.stream)
        b = self.bufs
        L.gather(_p(self.feat), sim.nx, sim.ny, sim.nz, _p(self.org), self.nb, INFER_PATCH + 2 * HALO, HALO,
                 _p(b["x"]), None, 0.0, None, self.stream)
        self.net.forward(b, self.nb)
        L.apply(eb, e, sx, sxy, sim.nx, sim.ny, sim.nz, _p(b["out"]), PRED_C, _p(self.org), self.nb, INFER_PATCH,
                HALO, self.out_scale, self.stream)
        if self.check:
            torch.cuda.synchronize()
            ew, wsx, wsxy, _ = self.win.field_device("energy")
            npx = self.col // PATCH
            npz = sim.nz // PATCH
            L.recheck(eb, e, sx, sxy, sim.nx, sim.ny, ew, wsx, wsxy, self.wn, self.wn, x0, y0, cx * self.col,
                      cy * self.col, 0,
                      npx, npx, npz, PATCH, sim.params.gamma, sim.params.xi_n, sim.params.ionise_pot,
                      self.bound, _p(self.err), _p(self.nrej), self.stream)
            torch.cuda.synchronize()
            info.checked = npx * npx * npz
            info.rejected = int(self.nrej.item())
            self.nrej.zero_()
            info.errs = self.err.cpu().numpy()
            info.max_err = float(info.errs.max())
            if info.rejected > self.fallback_fraction * info.checked:
                info.fallback = True
                self._copy_energy(False)
                torch.cuda.synchronize()
                sim.boundary_conditions()
                sim.conduct_heat_stages(self.dt, s)
                return info
        sim.boundary_conditions()
        return info


# ---------------------------------------------------------------------------
# Training entry point: python -m lare3d_b200.surrogate --out PATH

DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "surrogate_conduction_256.npz")
TRAIN_SEEDS = tuple(range(101, 113))   # 12 hot-spot layouts x 4 RKL2 steps x 4096 tiles = 196,608 patch pairs


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the conduction surrogate on the GPU engine's own RKL2 pairs")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=4, help="RKL2 steps per seed")
    ap.add_argument("--seeds", type=int, default=len(TRAIN_SEEDS))
    ap.add_argument("--iters", type=int, default=60000)
    ap.add_argument("--nb", type=int, default=64)
    ap.add_argument("--lr", type=float, default=5e-4)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    a = ap.parse_args(argv)
    torch = _torch()
    t0 = time.time()
    store, dT, dt = generate(TRAIN_SEEDS[:a.seeds], n=a.n, steps=a.steps, log=print)
    t_gen = time.time() - t0
    net = Network(seed=0)
    net.meta["dt_scale"] = dt_scale_of(dT)
    net.meta["dt"] = dt
    t0 = time.time()
    hist = train(net, store, dT, iters=a.iters, nb=a.nb, lr=a.lr, log=print, log_every=1000)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    net.save(a.out)
    print(json.dumps({"out": a.out, "pairs": int(store.shape[0]) * (a.n // PATCH) ** 3, "dt": dt,
                      "dt_scale": net.meta["dt_scale"], "generate_s": t_gen, "train_s": t_train,
                      "ms_per_iter": 1e3 * t_train / a.iters, "final_loss": hist[-1][1]}))


if __name__ == "__main__":
    main()

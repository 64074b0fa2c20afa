"""Throughput benchmark of the Lagrangian-remap timestep (one JSON line).

Workload (N = 1): the resistive 3-D Orszag-Tang vortex on a 256^3 periodic
[0, 2pi]^3 box, FP64 drop-in, one step = lagrangian_step + eulerian_remap +
eta_calc (lare3d.f90:84-87).  Metric: cell-updates/s = nx*ny*nz*steps / time.
Synthetic state generated on the host (no datasets exist for this code).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

* ``value``: device-resident throughput, CUDA events on the engine's stream
  around K steps, max over ranks; 8 state arrays of 141 MB each exceed L2.
* ``e2e``: the same metric through the C ABI with Fortran-layout host
  buffers in pinned memory: every step uploads the state, steps, downloads.
* ``roofline``: the dominant kernel of one profiled step; achieved =
  algorithmic bytes / event-timed duration; peak = measured HBM copy rate.
* ``cpu_baseline``: the oracle on the host cores, one step of the workload.
* N > 1: independent replicas (the single-GPU path has no exchange step).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from lare3d_b200 import replicas  # noqa: E402  (process-group plumbing; no torch import at module load)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", "--edge", dest="n", type=int, default=256)  # --edge: the spelling torchrun passes through
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--out-dir", default=os.path.join(ROOT, "bench_out"),
                    help="where the clock samples and per-site profile tables go")
    ap.add_argument("--case", default=None, choices=["mhd64", "mhd64x", "mhd32", "rkl64", "rkl32", "conv"],
                    help="run one small case of a hot path and exit (for targeted ncu captures): "
                         "two Orszag-Tang steps at --n^3 (FP64 product, FP64 exact, FP32), one RKL2 "
                         "conduction step, or the surrogate network forward on --n windows")
    return ap.parse_args()


OUT_DIR = os.path.join(ROOT, "bench_out")


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.path = os.path.join(OUT_DIR, f"clocks_rank{index}.csv")

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
            # nvidia-smi takes a while to start: wait for its first sample so
            # that the samples cover the timed region
            t0 = time.time()
            while time.time() - t0 < 3.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    return replicas.env()


def max_over_ranks(v, ws):
    return replicas.max_over_ranks(v, ws, "cuda")


def barrier(ws):
    replicas.barrier(ws)


def cpu_baseline(deck, steps=1):
    """The oracle on the host cores: one warm-up step and `steps` timed."""
    from oracle import oracle
    sim = oracle.simulation(deck)
    sim.start(deck.state)
    sim.step(1)
    t = time.perf_counter()
    for s in range(2, 2 + steps):
        sim.step(s)
    el = (time.perf_counter() - t) / steps
    sim.close()
    n3 = deck.nx * deck.ny * deck.nz
    return {"value": n3 / el, "unit": "cell-updates/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{steps} step(s) of the {deck.nx}^3 workload after 1 warm-up step, {el:.2f} s/step"}


def dump_profile(prof, name):
    """Write the per-launch-site table of one profiled step to the output folder."""
    path = os.path.join(OUT_DIR, name)
    os.makedirs(os.path.dirname(path), exist_ok=True)
    total = sum(p["ms"] for p in prof) or 1.0
    with open(path, "w") as f:
        f.write("site\tlaunches\tms\tshare\tGB/s\twords\n")
        for p in prof:
            gbs = p["bytes"] / (p["ms"] * 1e-3) / 1e9 if p["ms"] > 0 else 0.0
            f.write(f"{p['site']}\t{p['launches']}\t{p['ms']:.4f}\t{p['ms'] / total:.3f}\t{gbs:.0f}\t{p['words']}\n")


def time_steps(sim, torch, stream, first, k):
    """CUDA events around k device-resident steps on the engine's stream."""
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        e0.record(stream)
    sim.run(first, k)
    with torch.cuda.stream(stream):
        e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1000.0


def physics_forms(torch, n, ref_value, steps=3):
    """The widened physics at n^3, FP64, each through lare_gpu_run: open
    (characteristic) boundaries, the partially ionised EOS with Cowling
    resistivity at the default normalisation's physical eta_bar, optically
    thin radiation, and rke with cooling_term on the Orszag-Tang vortex.
    Whole steps (with their own dt and sub-cycles), after one warm-up step;
    value = cell-updates/s, ratio = value / the plain FP64 step's."""
    from lare3d_b200 import decks, gpu
    cases = [
        ("open_boundaries", lambda: decks.open_blast(n)),
        ("partially_ionised_cowling", lambda: decks.partially_ionised(n)),
        ("radiation", lambda: decks.radiative_blast(n)),
        ("rke_cooling_term", lambda: decks.orszag_tang(n, rke=1, cooling_term=1)),
    ]
    out = {}
    for name, make in cases:
        d = make()
        sim = gpu.simulation(d, precision=64)
        sim.start(d.state)
        sim.run(0, 1)
        stream = torch.cuda.ExternalStream(gpu.stream_of(sim))
        el = time_steps(sim, torch, stream, 1, steps)
        v = n ** 3 * steps / el
        out[name] = {"value": v, "unit": "cell-updates/s", "ms_per_step": 1e3 * el / steps,
                     "ratio_to_plain_step": v / ref_value, "substeps": sim.scalars().last_substeps,
                     "deck": d.name}
        sim.close()
        del sim, d
    return out


def surrogate_form(torch, cdeck, plain):
    """The learned conduction step at 256^3 (FP32 state) against plain FP32
    RKL2 from the same state, with the committed trained weights."""
    import numpy as np
    from lare3d_b200 import gpu
    from lare3d_b200 import surrogate as S
    if not os.path.exists(S.DEFAULT_WEIGHTS):
        return {"unavailable": "no trained weights (python -m lare3d_b200.surrogate)"}
    net = S.Network(seed=0)
    net.load(S.DEFAULT_WEIGHTS)
    dt = net.meta["dt"]
    n = cdeck.nx
    n3 = n ** 3
    ref = gpu.simulation(cdeck, precision=32)
    ref.start(cdeck.state)
    e_start = ref.get_field("energy")
    stages = ref.conduct_heat(dt)
    g = (cdeck.params.gamma - 1.0) / (2.0 - cdeck.params.xi_n)
    T_ref = g * ref.get_field("energy")[2:-2, 2:-2, 2:-2]
    T_0 = g * e_start[2:-2, 2:-2, 2:-2]
    # plain RKL2 at the surrogate's dt, timed the same way
    stp = torch.cuda.ExternalStream(gpu.stream_of(ref))
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a0.record(stp)
    for _ in range(3):
        ref.conduct_heat(dt)
    a1.record(stp)
    a1.synchronize()
    t_plain = a0.elapsed_time(a1) / 1000.0 / 3
    ref.close()
    sim = gpu.simulation(cdeck, precision=32)
    sim.start(cdeck.state)
    sc = S.SurrogateConduction(sim, cdeck, net, dt, bound=1e-3, col=64, seed=0)
    info = sc.step()
    T_sur = g * sim.get_field("energy")[2:-2, 2:-2, 2:-2]
    rel = np.abs(T_sur - T_ref) / np.abs(T_ref)
    rel0 = np.abs(T_0 - T_ref) / np.abs(T_ref)
    st = torch.cuda.ExternalStream(sc.stream)
    times = {}
    for chk in (True, False):
        sc.check = chk
        sim.set_field("energy", e_start)
        sim.boundary_conditions()
        torch.cuda.synchronize()
        a0.record(st)
        for _ in range(3):
            sc.step()
        a1.record(st)
        a1.synchronize()
        times[chk] = a0.elapsed_time(a1) / 1000.0 / 3
    a0.record(st)
    net.forward(sc.bufs, sc.nb)
    a1.record(st)
    a1.synchronize()
    t_fwd = a0.elapsed_time(a1) / 1000.0
    d = sc.bufs["d"]
    flops = sum(2 * 27 * cin * cf * d[l + 1] ** 3 * sc.nb for l, (cin, _c, _r, cf) in enumerate(S.LAYERS))
    sc.close()
    sim.close()
    out = {"value": n3 / times[True], "unit": "cell-updates/s (one conduction step incl. 1/16 re-check)",
           "ms_per_step": 1e3 * times[True], "ms_per_step_no_recheck": 1e3 * times[False],
           "plain_rkl2_fp32_ms_same_dt": 1e3 * t_plain, "speedup_vs_plain_rkl2": t_plain / times[True],
           "stages": stages, "network_forward_ms": 1e3 * t_fwd,
           "network_tflops": flops / t_fwd / 1e12, "network_flops_per_step": flops,
           # after the step (re-checked patches already replaced where they
           # failed), over every cell of the grid: the 1e-3 bound is enforced
           # on the re-checked patches only (1/16 of the grid per step); the
           # other patches keep the network's error
           "rel_T_err_vs_rkl2": {"rms": float(np.sqrt(np.mean(rel ** 2))), "max_all_patches": float(rel.max()),
                                 "frac_cells_over_1e-3": float(np.mean(rel > 1e-3)),
                                 "frac_patches_over_1e-3": float(np.mean(
                                     rel.reshape(n // 16, 16, n // 16, 16, n // 16, 16).max(axis=(1, 3, 5)) > 1e-3))},
           "rel_T_err_without_network": {"rms": float(np.sqrt(np.mean(rel0 ** 2))), "max": float(rel0.max()),
                                         "frac_cells_over_1e-3": float(np.mean(rel0 > 1e-3))},
           "recheck": {"patches": info.checked, "rejected": info.rejected,
                       "max_err_rechecked_patches_before_rejection": info.max_err, "bound": 1e-3,
                       "fallback": info.fallback},
           "weights": os.path.relpath(S.DEFAULT_WEIGHTS, ROOT)}
    return out


def ensemble_form(torch, count=48, launches=3):
    """48 blast / Orszag-Tang members of uneven sizes (32^3..128^3), FP32,
    one graph launch per 6 steps of all members; block shapes from the
    autotuner (measured at 32, 64, 96 and 128, nearest edge used)."""
    from lare3d_b200 import ensemble as E
    t0 = time.perf_counter()
    reps = (32, 64, 96, 128)
    tuned = {n: E.autotune(n, kind="blast", launches=1) for n in reps}
    t_tune = time.perf_counter() - t0
    specs = E.member_specs(count)
    blocks = {sp.n: tuned[min(reps, key=lambda r: abs(r - sp.n))][0] for sp in specs}
    ds = [E.member_deck(sp) for sp in specs]
    ens = E.Ensemble(ds, precision=32, blocks=blocks)
    st = torch.cuda.ExternalStream(ens.stream)
    ens.launch(1)
    ens.sync()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    ens.launch(launches)
    b.record(st)
    ens.sync()
    el = a.elapsed_time(b) / 1000.0
    cells = ens.cells()
    steps = launches * E.STEPS_PER_LAUNCH
    # the same members stepped one after another through lare_gpu_step
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for sim in ens.sims:
        first = sim.scalars().steps_taken
        for k in range(E.STEPS_PER_LAUNCH):
            sim.step(first + k + 1)
    torch.cuda.synchronize()
    el_seq = time.perf_counter() - t1
    ens.close()
    return {"value": cells * steps / el, "unit": "cell-updates/s (all members)", "members": count,
            "cells": cells, "steps": steps, "ms_per_step": 1e3 * el / steps,
            "sizes": sorted(sp.n for sp in specs),
            "sequential_lare_gpu_step_value": cells * E.STEPS_PER_LAUNCH / el_seq,
            "speedup_vs_sequential": (cells * steps / el) / (cells * E.STEPS_PER_LAUNCH / el_seq),
            "autotuned_blocks": {str(n): list(tuned[n][0]) for n in reps},
            "autotune_ms_per_step": {str(n): {f"{k[0]}x{k[1]}": round(v, 4) for k, v in tuned[n][1].items()}
                                     for n in reps},
            "autotune_s": t_tune, "dtype": "f32"}


def accuracy_forms(deck, steps=100):
    """Per-field relative L2 after `steps` steps of the workload at its full
    size: the FP64 product engine and the FP32 form against the exact FP64
    engine, which reproduces the oracle bit for bit (the GPU parity tests
    check that against the oracle itself on this workload at 128^3 for 100
    steps); the oracle would need minutes per step here."""
    import numpy as np
    from lare3d_b200 import gpu
    fields = ("rho", "energy", "vx", "vy", "vz", "bx", "by", "bz")
    states = {}
    for name, prec in (("exact", gpu.EXACT64), ("fp64", gpu.FP64), ("fp32", gpu.FP32)):
        s = gpu.simulation(deck, precision=prec)
        s.start(deck.state)
        s.run(0, steps)
        states[name] = s.download()
        s.close()
    ref = states["exact"]
    out = {}
    for name in ("fp64", "fp32"):
        errs = {}
        for f in fields:
            b = ref[f]
            errs[f] = float(np.linalg.norm(states[name][f] - b) / np.linalg.norm(b))
        out[name] = {"steps": steps, "rel_l2_vs_fp64_exact": errs, "worst": max(errs.values())}
    return out


def workload(n):
    """The workload name both arms print (same deck, same metric)."""
    return f"resistive Orszag-Tang {n}^3 periodic, FP64, eta=1e-3, CFL 0.8"


def run_case(what, n):
    """A small, self-contained run of one hot path, for a targeted ncu
    capture (ncu -k <kernel> -c 1 ... python bench.py --case <what> --n <n>)."""
    import torch
    from lare3d_b200 import decks, gpu
    if what in ("mhd64", "mhd64x", "mhd32"):
        d = decks.orszag_tang(n)
        s = gpu.simulation(d, precision={"mhd64": 64, "mhd64x": gpu.EXACT64, "mhd32": 32}[what])
        s.start(d.state)
        for k in range(1, 3):
            s.step(k)
    elif what in ("rkl64", "rkl32"):
        d = decks.conduction(n)
        s = gpu.simulation(d, precision=64 if what == "rkl64" else 32)
        s.start(d.state)
        s.conduct_heat(d.dt_fixed)
    else:
        from lare3d_b200 import surrogate as S
        net = S.Network(seed=0)
        b = net.buffers(n, S.INFER_PATCH + 2 * S.HALO, False)
        b["x"].normal_()
        net.forward(b, n)
    torch.cuda.synchronize()
    print("ok", what, n)


def run_reference(args):
    ws, rank, _ = dist_setup(args)
    if rank != 0:
        return
    from lare3d_b200 import decks
    deck = decks.orszag_tang(args.n)
    from oracle import oracle
    sim = oracle.simulation(deck)
    sim.start(deck.state)
    step = 0
    for _ in range(args.warmup):
        step += 1
        sim.step(step)
    t = time.perf_counter()
    for _ in range(args.steps):
        step += 1
        sim.step(step)
    el = time.perf_counter() - t
    n3 = deck.nx * deck.ny * deck.nz
    v = n3 * args.steps / el
    out = {
        "impl": "reference", "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded KISS perturbation of the Orszag-Tang state)",
        "config": {"workload": workload(args.n), "grid": [args.n] * 3,
                   "l2": "inputs larger than L2 (8 state arrays x 141 MB)"},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": oracle.num_threads(), "kind": "port",
                         "sample": f"{args.steps} steps after {args.warmup} warm-up steps (Fortran reference not buildable: no Fortran compiler)"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    global OUT_DIR
    args = parse()
    OUT_DIR = args.out_dir
    if args.case:
        return run_case(args.case, args.n)
    if args.impl == "reference":
        return run_reference(args)
    ws, rank, local = dist_setup(args)
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    replicas.init(ws, "nccl")

    from lare3d_b200 import decks, gpu
    from lare3d_b200.abi import State

    n = args.n
    deck = decks.orszag_tang(n)
    sim = gpu.simulation(deck, precision=64)
    sim.start(deck.state)
    stream = torch.cuda.ExternalStream(gpu.stream_of(sim))
    step = 0
    sim.run(step, args.warmup)
    step += args.warmup

    # ---- device-resident timed region
    clocks = Clocks(local)
    barrier(ws)
    clocks.start()
    l0 = sim.launch_count()
    el = time_steps(sim, torch, stream, step, args.steps)
    launches = sim.launch_count() - l0
    step += args.steps
    ck = clocks.stop()
    el_max = max_over_ranks(el, ws)
    n3 = n ** 3
    value = replicas.whole_job_rate(ws, n3 * args.steps, el_max)

    # ---- roofline of the dominant kernel (one profiled step)
    sim.profile(True)
    sim.run(step, 1)
    step += 1
    sim.profile(False)
    prof = sim.profile_report()
    dump_profile(prof, f"profile_fp64_rank{rank}.tsv")
    total_ms = sum(p["ms"] for p in prof)
    top = max((p for p in prof if p["words"] > 0), key=lambda p: p["ms"])
    hbm, peak_kind = peaks()
    per_launch_bytes = top["bytes"] / top["launches"]
    per_launch_s = top["ms"] / top["launches"] / 1e3
    achieved = per_launch_bytes / per_launch_s / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        # measured DRAM bytes per launch, keyed by routine, word count and grid
        for t in json.load(open(tpath)):
            if (t["routine"], t["words"], t["launches"], t["grid"]) == (top["site"].split(":")[0], top["words"],
                                                                         top["launches"], n):
                traffic = t["bytes_per_launch"]
    # the whole step as well: algorithmic bytes of every profiled launch over their summed time
    step_bytes = sum(p["bytes"] for p in prof)
    step_gbs = step_bytes / (total_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": traffic, "kernel": top["site"], "share": top["ms"] / total_ms,
                "peak_kind": peak_kind, "algorithmic_bytes_per_launch": per_launch_bytes,
                "step_achieved": step_gbs, "step_frac": step_gbs / hbm,
                # algorithmic bytes of the whole step per cell (16 words = 128 B is the
                # irreducible read and write of the eight state fields)
                "step_bytes_per_cell": step_bytes / n ** 3, "step_words_per_cell": step_bytes / n ** 3 / 8}

    # ---- end to end through the C ABI with pinned host buffers
    host = {}
    for k, a in deck.state.arrays.items():
        t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
        h = t.numpy().reshape(a.shape, order="F")
        h[...] = a
        host[k] = (t, h)
    st = State(n, n, n, {k: v[1] for k, v in host.items()})
    bi = sum(v[1].nbytes for v in host.values())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    sim.upload(st)
    barrier(ws)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.e2e_steps):
        step += 1
        sim.upload(st)
        sim.step(step)
        sim.download(st)
    e1.record(stream)
    e1.synchronize()
    e2e_el = max_over_ranks(e0.elapsed_time(e1) / 1000.0, ws)
    e2e = {"value": replicas.whole_job_rate(ws, n3 * args.e2e_steps, e2e_el), "unit": "cell-updates/s",
           "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bi, "steps": args.e2e_steps}
    # the floor a step through host buffers cannot beat: the same bytes copied
    # by plain pinned-memory copies (one per array, each way) plus the
    # device-resident step
    big = max(v[0].numel() for v in host.values())
    dev = torch.empty(big, dtype=torch.float64, device="cuda")
    back = torch.empty(big, dtype=torch.float64, pin_memory=True)
    cs = torch.cuda.Stream()  # a stream of torch's own (the engine's is destroyed with the context)
    torch.cuda.synchronize()
    with torch.cuda.stream(cs):
        e0.record(cs)
        for t, _ in host.values():
            dev[:t.numel()].copy_(t, non_blocking=True)
        e1.record(cs)
        e1.synchronize()
        t_h2d = e0.elapsed_time(e1) / 1000.0
        e0.record(cs)
        for t, _ in host.values():
            back[:t.numel()].copy_(dev[:t.numel()], non_blocking=True)
        e1.record(cs)
        e1.synchronize()
        t_d2h = e0.elapsed_time(e1) / 1000.0
    torch.cuda.synchronize()
    del dev, back
    floor_s = t_h2d + t_d2h + el_max / args.steps
    e2e["copy_floor"] = {"h2d_gbs": bi / t_h2d / 1e9, "d2h_gbs": bi / t_d2h / 1e9,
                         "ms_per_step": 1e3 * floor_s, "e2e_over_floor": (e2e_el / args.e2e_steps) / floor_s}

    # ---- the other forms (FP32, RKL2 conduction, ...), one GPU only: with
    # replicas the other ranks would wait for them at the closing barrier
    forms = {}
    if ws == 1 and not args.no_forms:
        s32 = gpu.simulation(deck, precision=32)
        s32.start(deck.state)
        s32.run(0, 2)
        st32 = torch.cuda.ExternalStream(gpu.stream_of(s32))
        el32 = time_steps(s32, torch, st32, 2, args.steps)
        s32.profile(True)
        s32.run(2 + args.steps, 1)
        s32.profile(False)
        dump_profile(s32.profile_report(), "profile_fp32_rank0.tsv")
        forms["fp32"] = {"value": n3 * args.steps / el32, "unit": "cell-updates/s",
                         "ms_per_step": 1e3 * el32 / args.steps, "speedup_vs_fp64": (n3 * args.steps / el32) / value}
        s32.close()
        sx = gpu.simulation(deck, precision=gpu.EXACT64)
        sx.start(deck.state)
        sx.run(0, 2)
        stx = torch.cuda.ExternalStream(gpu.stream_of(sx))
        elx = time_steps(sx, torch, stx, 2, args.steps)
        forms["fp64_exact"] = {"value": n3 * args.steps / elx, "unit": "cell-updates/s",
                               "ms_per_step": 1e3 * elx / args.steps,
                               "note": "LARE_FP64_EXACT: the reference's arithmetic bit for bit (parity build)"}
        sx.close()
        cdeck = decks.conduction(n)
        for prec in (64, 32):
            sc = gpu.simulation(cdeck, precision=prec)
            sc.start(cdeck.state)
            sc.conduct_heat(cdeck.dt_fixed)
            stc = torch.cuda.ExternalStream(gpu.stream_of(sc))
            a0 = torch.cuda.Event(enable_timing=True)
            a1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a0.record(stc)
            reps = 3
            for _ in range(reps):
                ns = sc.conduct_heat(cdeck.dt_fixed)
            a1.record(stc)
            a1.synchronize()
            elc = a0.elapsed_time(a1) / 1000.0 / reps
            forms[f"conduction_rkl2_fp{prec}"] = {"value": n3 / elc, "unit": "cell-updates/s (one conduct_heat substep)",
                                                  "ms_per_substep": 1e3 * elc, "stages": ns,
                                                  "dt_over_dt_parab": cdeck.info["dt_ratio"]}
            sc.close()
        forms["surrogate_conduction"] = surrogate_form(torch, cdeck, forms.get("conduction_rkl2_fp32"))
        forms["ensemble"] = ensemble_form(torch)
        forms["physics_fp64"] = physics_forms(torch, n, value)
        acc = accuracy_forms(deck)
        forms["fp32"]["rel_l2_vs_fp64_exact"] = acc["fp32"]
        forms["fp64_product_accuracy"] = acc["fp64"]

    cpu = None
    if ws == 1 and not args.no_cpu_baseline:  # the host-core baseline is an N = 1 figure
        cpu = cpu_baseline(deck, steps=1)

    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded KISS perturbation of the Orszag-Tang state)",
            "config": {"workload": workload(n), "grid": [n, n, n],
                       "l2": "inputs larger than L2 (8 state arrays x 141 MB)",
                       "parallelism": f"replicas x{ws}"},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": launches,
            "clocks": ck,
            "top_kernels": [{k: p[k] for k in ("site", "launches", "ms", "words")} for p in prof[:8]],
            # last, so that a tail of the output keeps them: the widened
            # physics and the ensemble first, the FP32 form at the very end
            "forms": {k: forms[k] for k in ("physics_fp64", "ensemble", "surrogate_conduction",
                                            "conduction_rkl2_fp64", "conduction_rkl2_fp32", "fp64_exact",
                                            "fp64_product_accuracy", "fp32")
                      if k in forms},
        }
        print(json.dumps(line), flush=True)
    torch.cuda.synchronize()
    sim.close()
    barrier(ws)
    replicas.finish(ws)


if __name__ == "__main__":
    main()

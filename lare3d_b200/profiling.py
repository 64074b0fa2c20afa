"""Nsight Compute helpers for the profiles/ notes.

    python -m lare3d_b200.profiling drive <workload> <size>
        a small, self-contained run of one hot path for a targeted capture
        (`ncu -k <kernel> -c 1 ... python -m lare3d_b200.profiling drive ...`):
          mhd64 N / mhd32 N  two Orszag-Tang steps at N^3, FP64 / FP32
          rkl64 N / rkl32 N  one RKL2 conduction step of the conduction deck
          conv NB            the surrogate network forward on NB 72^3 windows
    python -m lare3d_b200.profiling launches <launch-list.csv>
        per-kernel launches, total device time and share, from a
        `ncu --metrics gpu__time_duration.sum --csv` launch list
    python -m lare3d_b200.profiling metrics <report.ncu-rep>
        the roofline-relevant counters of each captured launch
"""
from __future__ import annotations

import collections
import csv
import re
import subprocess
import sys


def _short(name: str) -> str:
    m = re.search(r"k_box(?:_mb<\d+, |<)void (?:lare::)?(\w+)<([^>]*)>\(.*?\)::\[lambda\(int, int, int\) \(instance (\d+)\)\]>", name)
    if m:
        return f"{m.group(1)}<{m.group(2)}> lambda {m.group(3)}"
    m = re.search(r"k_box_(sum|min)<\d+, void (?:lare::)?(\w+)<", name)
    if m:
        return f"{m.group(2)} box_{m.group(1)}"
    m = re.search(r"void (?:lare::|<unnamed>::)?(\w+(?:<[^()]*>)?)", name)
    return m.group(1) if m else name[:60]


def launches(path: str) -> str:
    rows = list(csv.reader(open(path)))
    hi = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    h = rows[hi]
    ki, mi, ui, vi = h.index("Kernel Name"), h.index("Metric Name"), h.index("Metric Unit"), h.index("Metric Value")
    agg = collections.OrderedDict()
    for r in rows[hi + 1:]:
        if len(r) <= vi or r[mi] != "gpu__time_duration.sum":
            continue
        k = _short(r[ki])
        t = float(r[vi].replace(",", "")) * (1e-3 if r[ui] == "ns" else (1e3 if r[ui] == "ms" else 1.0))  # -> us
        a = agg.setdefault(k, [0, 0.0])
        a[0] += 1
        a[1] += t
    total = sum(v[1] for v in agg.values())
    lines = ["| kernel | launches | total us | share |", "|---|---|---|---|"]
    for k, (n, t) in sorted(agg.items(), key=lambda kv: -kv[1][1]):
        lines.append(f"| {k} | {n} | {t:.1f} | {100 * t / total:.1f}% |")
    lines.append(f"| TOTAL | {sum(v[0] for v in agg.values())} | {total:.1f} | |")
    return "\n".join(lines)


WANT = ["gpu__time_duration.sum", "dram__bytes.sum.per_second", "dram__cycles_active.avg.pct_of_peak_sustained_elapsed",
        "sm__throughput.avg.pct_of_peak_sustained_elapsed", "sm__issue_active.avg.pct_of_peak_sustained_elapsed",
        "sm__warps_active.avg.pct_of_peak_sustained_active", "launch__registers_per_thread", "launch__grid_size",
        "launch__block_size", "sm__pipe_fp64_cycles_active.avg.pct_of_peak_sustained_active",
        "sm__pipe_tensor_cycles_active.avg.pct_of_peak_sustained_active", "l1tex__t_sector_hit_rate.pct",
        "lts__t_sector_hit_rate.pct",
        "smsp__average_warps_issue_stalled_long_scoreboard_per_issue_active.ratio",
        "smsp__average_warps_issue_stalled_barrier_per_issue_active.ratio",
        "smsp__average_warps_issue_stalled_wait_per_issue_active.ratio"]


def metrics(path: str) -> str:
    out = subprocess.run(["ncu", "-i", path, "--page", "raw", "--csv"], capture_output=True, text=True).stdout
    rows = list(csv.reader(out.splitlines()))
    h, u = rows[0], rows[1]
    res = []
    for r in rows[2:]:
        d = dict(zip(h, r))
        units = dict(zip(h, u))
        lines = [_short(d["Kernel Name"])]
        for k in WANT:
            if k in d:
                lines.append(f"  {k} = {d[k]} {units[k]}")
        if "dram__bytes.sum.per_second" in d and "gpu__time_duration.sum" in d:
            bw = float(d["dram__bytes.sum.per_second"].replace(",", ""))
            bw *= {"Tbyte/s": 1e12, "Gbyte/s": 1e9, "Mbyte/s": 1e6}.get(units["dram__bytes.sum.per_second"], 1.0)
            t = float(d["gpu__time_duration.sum"].replace(",", ""))
            t *= {"ns": 1e-9, "us": 1e-6, "usecond": 1e-6, "ms": 1e-3, "msecond": 1e-3}.get(
                units["gpu__time_duration.sum"], 1e-6)
            lines.append(f"  dram bytes (read + write) = {bw * t / 1e6:.1f} MB")
        res.append("\n".join(lines))
    return "\n".join(res)


def drive(what: str, n: int) -> None:
    import torch
    from . import decks, gpu
    if what in ("mhd64", "mhd32"):
        d = decks.orszag_tang(n)
        s = gpu.simulation(d, precision=64 if what == "mhd64" else 32)
        s.start(d.state)
        for k in range(1, 3):
            s.step(k)
    elif what in ("rkl64", "rkl32"):
        d = decks.conduction(n)
        s = gpu.simulation(d, precision=64 if what == "rkl64" else 32)
        s.start(d.state)
        s.conduct_heat(d.dt_fixed)
    elif what == "conv":
        from . import surrogate as S
        net = S.Network(seed=0)
        b = net.buffers(n, S.INFER_PATCH + 2 * S.HALO, False)
        b["x"].normal_()
        net.forward(b, n)
    else:
        raise SystemExit(f"unknown workload {what}")
    torch.cuda.synchronize()
    print("ok", what, n)


if __name__ == "__main__":
    mode = sys.argv[1]
    if mode == "drive":
        drive(sys.argv[2], int(sys.argv[3]))
    elif mode == "launches":
        print(launches(sys.argv[2]))
    else:
        print(metrics(sys.argv[2]))

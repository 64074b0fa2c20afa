"""Summaries of Nsight Compute output for the profiles/ notes.

    python -m lare3d_b200.profiling launches <launch-list.csv>
        per-kernel launches, total device time and share, from a
        `ncu --metrics gpu__time_duration.sum --csv` launch list
    python -m lare3d_b200.profiling metrics <raw.csv>
        the roofline-relevant counters of a `ncu -i <rep> --page raw --csv`
        export, one row per captured launch
"""
from __future__ import annotations

import collections
import csv
import re
import sys


def _short(name: str) -> str:
    m = re.search(r"k_box<void (\w+)<\w+>\(.*?\)::\[lambda\(int, int, int\) \(instance (\d+)\)\]>", name)
    if m:
        return f"{m.group(1)}#{m.group(2)}"
    m = re.search(r"k_box_(sum|min)<\d+, void (\w+)<\w+>", name)
    if m:
        return f"{m.group(2)}:box_{m.group(1)}"
    m = re.search(r"void (?:lare::)?(\w+)", name)
    return m.group(1) if m else name[:60]


def launches(path: str) -> str:
    rows = [r for r in csv.reader(open(path)) if len(r) > 14 and r[0].isdigit()]
    agg = collections.OrderedDict()
    for r in rows:
        if r[12] != "gpu__time_duration.sum":
            continue
        k = _short(r[4])
        t = float(r[14]) * (1e-3 if r[13] == "ns" else 1.0)  # -> us
        a = agg.setdefault(k, [0, 0.0])
        a[0] += 1
        a[1] += t
    total = sum(v[1] for v in agg.values())
    lines = [f"{'kernel':48s} {'launches':>8s} {'total us':>12s} {'share':>7s}"]
    for k, (n, t) in sorted(agg.items(), key=lambda kv: -kv[1][1]):
        lines.append(f"{k:48s} {n:8d} {t:12.1f} {100 * t / total:6.1f}%")
    lines.append(f"{'TOTAL':48s} {sum(v[0] for v in agg.values()):8d} {total:12.1f}")
    return "\n".join(lines)


WANT = ["gpu__time_duration.sum", "dram__bytes_read.sum", "dram__bytes_write.sum",
        "gpu__dram_throughput.avg.pct_of_peak_sustained_elapsed", "sm__throughput.avg.pct_of_peak_sustained_elapsed",
        "launch__registers_per_thread", "sm__warps_active.avg.pct_of_peak_sustained_active",
        "smsp__inst_executed_pipe_fp64.avg.pct_of_peak_sustained_active"]


def metrics(path: str) -> str:
    rows = list(csv.reader(open(path)))
    hdr_i = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    hdr = rows[hdr_i]
    out = []
    for r in rows[hdr_i + 2:]:
        if len(r) != len(hdr):
            continue
        d = dict(zip(hdr, r))
        vals = {k: d.get(k, "") for k in WANT if k in d}
        out.append(_short(d["Kernel Name"]) + "\n" + "\n".join(f"  {k} = {v}" for k, v in vals.items()))
    return "\n".join(out)


if __name__ == "__main__":
    mode, path = sys.argv[1], sys.argv[2]
    print(launches(path) if mode == "launches" else metrics(path))

"""Summaries of Nsight Compute output for the profile notes.

    python -m adatm_b200.ncu_summary launches LAUNCHES.csv [--top 25]
    python -m adatm_b200.ncu_summary kernel REPORT.ncu-rep

`launches` reads a launch list made with
`ncu --metrics gpu__time_duration.sum --csv --log-file LAUNCHES.csv <cmd>` and
prints, per kernel, its launches, total device time and share of the total
(per-launch times under ncu are cold-cache and serialised: compare shares).
`kernel` runs `ncu -i REPORT --page raw --csv` and prints the metrics the
notes use for every captured launch.
"""
from __future__ import annotations

import argparse
import csv
import io
import re
import subprocess
import sys
from collections import OrderedDict


def _short(name):
    """Kernel name without the anonymous namespace and argument list."""
    name = re.sub(r"\(.*\)$", "", name.strip())
    for ns in ("(anonymous namespace)::", "<unnamed>::", "unnamed>::"):
        name = name.replace(ns, "")
    return re.sub(r"^void ", "", name)


def launches(path, top):
    rows = []
    with open(path, newline="") as f:
        lines = [l for l in f if l.startswith('"')]
    for r in csv.DictReader(io.StringIO("".join(lines))):
        if r.get("Metric Name") == "gpu__time_duration.sum":
            v = float(r["Metric Value"].replace(",", ""))
            unit = r.get("Metric Unit", "ns")
            us = v / 1000.0 if unit in ("nsecond", "ns") else (v * 1000.0 if unit in ("msecond", "ms") else v)
            rows.append((_short(r["Kernel Name"]), us))
    per = OrderedDict()
    for k, us in rows:
        n, t = per.get(k, (0, 0.0))
        per[k] = (n + 1, t + us)
    total = sum(t for _, t in per.values())
    print(f"Total {total:.1f} us over {len(rows)} launches.\n")
    print("| kernel | launches | total us | share |")
    print("|---|---|---|---|")
    for k, (n, t) in sorted(per.items(), key=lambda kv: -kv[1][1])[:top]:
        print(f"| `{k}` | {n} | {t:.1f} | {100.0 * t / total:.1f}% |")


METRICS = [
    "gpu__time_duration.sum", "dram__bytes_read.sum", "dram__bytes_write.sum",
    "dram__throughput.avg.pct_of_peak_sustained_elapsed", "lts__t_sector_hit_rate.pct",
    "lts__throughput.avg.pct_of_peak_sustained_elapsed", "l1tex__t_sector_hit_rate.pct",
    "launch__registers_per_thread", "launch__grid_size", "sm__warps_active.avg.per_cycle_active",
    "smsp__issue_active.avg.pct_of_peak_sustained_active", "smsp__inst_executed.sum",
    "sm__pipe_tensor_cycles_active.avg.pct_of_peak_sustained_active",
    "smsp__average_warps_issue_stalled_long_scoreboard_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_wait_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_short_scoreboard_per_issue_active.ratio",
    "smsp__average_warps_issue_stalled_not_selected_per_issue_active.ratio",
]


def kernel(report):
    out = subprocess.run(["ncu", "-i", report, "--page", "raw", "--csv"], capture_output=True,
                         text=True, check=True).stdout
    rows = list(csv.reader(io.StringIO(out)))
    hdr, units = rows[0], rows[1]
    for r in rows[2:]:
        print(f"### `{_short(r[hdr.index('Kernel Name')])}`\n")
        print("| metric | value |")
        print("|---|---|")
        for m in METRICS:
            if m in hdr:
                i = hdr.index(m)
                print(f"| {m} | {r[i]} {units[i]} |")
        print()


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("launches")
    a.add_argument("csv")
    a.add_argument("--top", type=int, default=25)
    b = sub.add_parser("kernel")
    b.add_argument("report")
    args = ap.parse_args()
    if args.cmd == "launches":
        launches(args.csv, args.top)
    else:
        kernel(args.report)


if __name__ == "__main__":
    sys.exit(main())

"""Summarise an ncu launch list (``--metrics gpu__time_duration.sum --csv``):
launches, total time and share per kernel.

    python -m pyto_b200.ncu_summary launches.csv
"""
import csv
import sys
from collections import defaultdict


def summarise(path):
    rows = list(csv.reader(open(path)))
    hdr = None
    for i, r in enumerate(rows):
        if "Kernel Name" in r and "Metric Value" in r:
            hdr, start = r, i + 1
            break
    if hdr is None:
        raise SystemExit("no ncu csv header found")
    kn, mn, mv, mu = (hdr.index(k) for k in ("Kernel Name", "Metric Name", "Metric Value", "Metric Unit"))
    tot, cnt = defaultdict(float), defaultdict(int)
    for r in rows[start:]:
        if len(r) <= mv or r[mn] != "gpu__time_duration.sum":
            continue
        v = float(r[mv].replace(",", ""))
        scale = {"nsecond": 1e-3, "ns": 1e-3, "usecond": 1.0, "us": 1.0, "msecond": 1e3, "ms": 1e3,
                 "second": 1e6, "s": 1e6}[r[mu]]
        name = r[kn].split("(")[0].split("<")[0].replace("void ", "").strip()
        tot[name] += v * scale
        cnt[name] += 1
    T = sum(tot.values())
    print(f"{'kernel':40s} {'launches':>9s} {'total_us':>12s} {'share':>7s} {'avg_us':>9s}")
    for k in sorted(tot, key=lambda k: -tot[k]):
        print(f"{k:40s} {cnt[k]:9d} {tot[k]:12.1f} {100 * tot[k] / T:6.1f}% {tot[k] / cnt[k]:9.2f}")
    print(f"{'TOTAL':40s} {sum(cnt.values()):9d} {T:12.1f}")


if __name__ == "__main__":
    summarise(sys.argv[1])

"""Compare a run's diagnostics CSV against a reference time series.

The reference compares its CSV with an external 512^3 DNS curve (``spectral_Re1600_512.dat``:
whitespace columns t, E, epsilon, enstrophy) by plotting both
(``compare_taylor_green.py``).  This module does the same comparison numerically: the
reference series is interpolated at the run's output times and the report gives the largest
absolute and relative gaps in E, epsilon and enstrophy, and the time and value of peak
dissipation in each series.  With --aligned the two series are also written side by side
as CSV (for plotting elsewhere).

    python -m spectral_solver_b200.compare --ours out/taylor_green_diagnostics.csv \\
        --reference spectral_Re1600_512.dat [--re 1600] [--aligned out/compare.csv]
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

KEYS = ("kinetic_energy", "dissipation", "enstrophy")


def load_reference(path):
    data = np.loadtxt(path)
    if data.ndim != 2 or data.shape[1] < 4:
        raise ValueError(f"{path} must have at least four columns: t E epsilon enstrophy")
    return {"t": data[:, 0], "kinetic_energy": data[:, 1], "dissipation": data[:, 2], "enstrophy": data[:, 3]}


def load_ours(path, reynolds):
    data = np.genfromtxt(path, delimiter=",", names=True)
    names = set(data.dtype.names or ())
    missing = {"t", "kinetic_energy", "dissipation"} - names
    if missing:
        raise ValueError(f"{path} is missing columns: {', '.join(sorted(missing))}")
    out = {k: np.atleast_1d(np.asarray(data[k], dtype=np.float64)) for k in ("t", "kinetic_energy", "dissipation")}
    # older CSVs without enstrophy: eps = 2 nu * enstrophy
    out["enstrophy"] = (np.atleast_1d(np.asarray(data["enstrophy"], dtype=np.float64)) if "enstrophy" in names
                        else out["dissipation"] * reynolds / 2.0)
    return out


def peak(t, eps):
    i = int(np.argmax(eps))
    return float(t[i]), float(eps[i])


def compare(ours, ref):
    t = ours["t"]
    inside = (t >= ref["t"][0]) & (t <= ref["t"][-1])
    if not np.any(inside):
        raise ValueError("the two series do not overlap in time")
    t = t[inside]
    report = {"t_range": [float(t[0]), float(t[-1])], "points": int(t.size)}
    aligned = {"t": t}
    for k in KEYS:
        a = ours[k][inside]
        b = np.interp(t, ref["t"], ref[k])
        aligned[k] = a
        aligned["reference_" + k] = b
        gap = np.abs(a - b)
        report[k] = {"max_abs": float(np.max(gap)), "max_rel": float(np.max(gap / np.maximum(np.abs(b), 1e-300))),
                     "at_t": float(t[int(np.argmax(gap))])}
    report["peak_dissipation"] = {"ours": peak(ours["t"], ours["dissipation"]),
                                  "reference": peak(ref["t"], ref["dissipation"])}
    return report, aligned


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--ours", required=True)
    ap.add_argument("--reference", required=True)
    ap.add_argument("--re", type=float, default=1600.0)
    ap.add_argument("--aligned", default=None, help="write the aligned series to this CSV")
    a = ap.parse_args(argv)
    report, aligned = compare(load_ours(a.ours, a.re), load_reference(a.reference))
    if a.aligned:
        cols = list(aligned)
        np.savetxt(a.aligned, np.column_stack([aligned[c] for c in cols]), delimiter=",", header=",".join(cols),
                   comments="")
    print(json.dumps(report, indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Regenerates the golden fixtures from the reference's own CSV outputs.

Run where the reference project is checked out, giving its root (or set
FE_REFERENCE_ROOT):
    python tests/golden/make_golden.py <reference project root>
Writes:
  rest_density.npy     float32[4800]: scripts/rest_density.csv, the densities
                       after one neighbour search (bitonic) + density_alpha
                       of the zero-jitter 20x20x12 scene
                       (convergence_benchmark.rs:420-542), in sorted order.
  reference_csv.json   scripts/sort_benchmark.csv (radix/bitonic ms per N),
                       scripts/convergence.csv (error vs Jacobi iterations)
                       and a summary of scripts/cfl_comparison.csv.
"""
import csv
import json
import os
import sys

import numpy as np


def main(ref_root: str) -> None:
    here = os.path.dirname(os.path.abspath(__file__))
    scripts = os.path.join(ref_root, "scripts")
    rho = np.loadtxt(os.path.join(scripts, "rest_density.csv"), skiprows=1,
                     dtype=np.float32)
    np.save(os.path.join(here, "rest_density.npy"), rho)

    out = {"sort_benchmark": [], "convergence": [], "cfl_comparison": {}}
    with open(os.path.join(scripts, "sort_benchmark.csv")) as f:
        for row in csv.DictReader(f):
            out["sort_benchmark"].append({"n": int(row["n"]), "algorithm": row["algorithm"],
                                          "time_ms": float(row["time_ms"])})
    with open(os.path.join(scripts, "convergence.csv")) as f:
        for row in csv.DictReader(f):
            out["convergence"].append({"iters": int(row["iters"]),
                                       "density_error": float(row["density_error"]),
                                       "divergence_error": float(row["divergence_error"])})
    rows = list(csv.DictReader(open(os.path.join(scripts, "cfl_comparison.csv"))))
    for mode in ("static", "adaptive"):
        r = [x for x in rows if x["mode"] == mode]
        sp = [float(x["max_speed"]) for x in r]
        out["cfl_comparison"][mode] = {
            "frames": len(r), "first_max_speed": sp[:5],
            "max_speed_frames_0_50_median": float(np.median(sp[:50])),
            "dt_last": float(r[-1]["dt"]), "iters": int(r[0]["iters"])}
    with open(os.path.join(here, "reference_csv.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FE_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference project root> "
                 "(or set FE_REFERENCE_ROOT)")
    main(root)

"""The harnesses' CSV writers reproduce the reference's files byte for byte
when given the reference's own values (the golden fixture of its CSVs)."""
import json
import os

import numpy as np

from conftest import GOLDEN
from fluid_step import harness


def _golden():
    with open(os.path.join(GOLDEN, "reference_csv.json")) as f:
        return json.load(f)


def test_convergence_csv_format(tmp_path):
    rows = [(r["iters"], np.float32(r["density_error"]), np.float32(r["divergence_error"]))
            for r in _golden()["convergence"]]
    p = tmp_path / "convergence.csv"
    harness.write_convergence_csv(str(p), rows)
    lines = p.read_text().splitlines()
    assert lines[0] == "iters,density_error,divergence_error"
    # the reference file's first rows, as written by its write_csv
    assert lines[1] == "1,1304.851318,418.425354"
    assert lines[2] == "2,178.012680,854.307617"
    assert len(lines) == len(rows) + 1


def test_sort_csv_format(tmp_path):
    rows = [(r["n"], r["algorithm"], r["time_ms"]) for r in _golden()["sort_benchmark"]]
    p = tmp_path / "sort.csv"
    harness.write_sort_csv(str(p), rows)
    lines = p.read_text().splitlines()
    assert lines[:3] == ["n,algorithm,time_ms", "1024,Bitonic,0.2249", "1024,Radix,1.0585"]


def test_cfl_csv_format(tmp_path):
    g = _golden()["cfl_comparison"]["static"]
    rows = [(k, "static", np.float32(0.005), np.float32(v), 4)
            for k, v in enumerate(g["first_max_speed"])]
    p = tmp_path / "cfl.csv"
    harness.write_cfl_csv(str(p), rows)
    lines = p.read_text().splitlines()
    assert lines[:3] == ["frame,mode,dt,max_speed,iters", "0,static,0.005000,0.8102,4",
                         "1,static,0.005000,0.6511,4"]


def test_rest_density_csv_format(tmp_path):
    d = np.load(os.path.join(GOLDEN, "rest_density.npy"))
    p = tmp_path / "rest.csv"
    harness.write_rest_density_csv(str(p), d)
    lines = p.read_text().splitlines()
    assert lines[0] == "density" and len(lines) == d.size + 1
    assert lines[1] == f"{float(d[0]):.6f}"


def test_f32_mean_is_sequential_single_precision():
    xs = [np.float32(1e8), np.float32(1.0), np.float32(-1e8), np.float32(1.0)]
    # a float32 running sum loses the first 1.0 against 1e8
    assert harness._f32_mean(xs) == float(np.float32(1.0) / np.float32(4.0))

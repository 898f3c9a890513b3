"""The reference's harnesses on this library: files in the reference's
formats, and results inside the bands of the reference's own published runs
(its jitter is unseeded, so only bands compare)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from fluid_step import harness

pytestmark = pytest.mark.gpu


def _golden():
    with open(os.path.join(GOLDEN, "reference_csv.json")) as f:
        return json.load(f)


def test_convergence_plateau_matches_reference_band(tmp_path):
    p = tmp_path / "convergence.csv"
    rows = harness.convergence(str(p), iter_values=(1, 2, 4))
    lines = p.read_text().splitlines()
    assert lines[0] == "iters,density_error,divergence_error" and len(lines) == 4
    ref = {r["iters"]: r for r in _golden()["convergence"]}
    d = {k: de for k, de, _ in rows}
    # one iteration leaves a large error; from two on the free-surface plateau
    assert d[1] > 3 * d[2]
    for k in (2, 4):
        assert 0.75 * ref[k]["density_error"] <= d[k] <= 1.25 * ref[k]["density_error"], (k, d[k])


def test_cfl_comparison_static_speeds_match_reference_band(tmp_path):
    p = tmp_path / "cfl.csv"
    rows = harness.cfl_comparison(str(p), frames=30)
    lines = p.read_text().splitlines()
    assert lines[0] == "frame,mode,dt,max_speed,iters" and len(lines) == 61
    static = [r for r in rows if r[1] == "static"]
    adaptive = [r for r in rows if r[1] == "adaptive"]
    assert all(abs(r[2] - 0.005) < 1e-9 and r[4] == 4 for r in static)
    assert all(r[4] == 100 for r in adaptive)
    assert len({round(r[2], 6) for r in adaptive}) > 1          # dt adapts
    ref = _golden()["cfl_comparison"]["static"]["first_max_speed"]
    for ours, theirs in zip([r[3] for r in static[:5]], ref):
        assert 0.6 * theirs <= ours <= 1.4 * theirs


def test_rest_density_matches_golden(tmp_path):
    p = tmp_path / "rest.csv"
    d = harness.rest_density(str(p))
    golden = np.load(os.path.join(GOLDEN, "rest_density.npy"))
    assert d.shape == golden.shape
    rel = np.abs(np.sort(d) - np.sort(golden)) / np.sort(golden)
    assert rel.max() < 1e-6
    assert p.read_text().splitlines()[0] == "density"


def test_sort_benchmark_file(tmp_path):
    p = tmp_path / "sort.csv"
    rows = harness.sort_benchmark(str(p), n_values=(1024, 65536), warmup=1, timed=3)
    assert [(r[0], r[1]) for r in rows] == [(1024, "Bitonic"), (1024, "Radix"),
                                            (65536, "Bitonic"), (65536, "Radix")]
    assert all(r[2] > 0 for r in rows)
    assert p.read_text().splitlines()[0] == "n,algorithm,time_ms"

"""The configuration-size fixtures describe the workloads the benchmark runs (CPU)."""

import json
from pathlib import Path

import numpy as np

FIXTURES = json.loads((Path(__file__).resolve().parent / "golden" / "config_fixtures.json").read_text())


def test_xxz_fixture_is_the_benchmark_workload():
    xxz = FIXTURES["xxz"]
    # the XXZ benchmark line draws Delta from the seed L + rank (rank 0)
    assert xxz["delta"] == float(np.random.default_rng(xxz["sites"]).uniform(0.5, 1.5))
    assert xxz["seed"] == xxz["sites"] == 28
    assert np.all(np.diff(xxz["eigenvalues"]) >= 0)
    assert np.all(np.asarray(xxz["residuals"]) <= 1e-10 * np.maximum(np.abs(xxz["eigenvalues"]), 1.0))


def test_sector_fixtures_cover_the_scan_and_count_right(oracle):
    sectors = FIXTURES["sectors"]
    assert sorted(s["momentum"] for s in sectors if s["sites"] == 26) == list(range(26))
    for s in sectors:
        assert s["dimension"] == oracle.sector_dimension(s["sites"], s["up"], s["momentum"], s["parity"])

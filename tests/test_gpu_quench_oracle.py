"""The transverse-field Ising quench against the oracle at 22 sites.

Workload of the quench benchmark line at a size the oracle can propagate:
open chain, J = 1, g = 1, h_i ~ U[-2, 2] (seed 2024), |up...up> to t = 10 in
100 steps of 0.1. The oracle's Taylor plan (complex128) is summarised in
tests/golden/quench_fixture.json at t = 1..10 by 64 seeded +-1 projections,
32 amplitudes, the norm and the return amplitude. The 2-norm distance of the
GPU state is estimated from the projections (||G e|| / sqrt(64), within a
factor ~1.5 of ||e|| with overwhelming probability): complex128 working
vectors must stay within 1e-9; complex64 working vectors are reported and
bounded by 1e-4.
"""

import importlib.util
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
FIXTURE_PATH = GOLDEN / "quench_fixture.json"
FIXTURE = json.loads(FIXTURE_PATH.read_text()) if FIXTURE_PATH.exists() else None


def _sketcher():
    spec = importlib.util.spec_from_file_location("make_quench_fixture", GOLDEN / "make_quench_fixture.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


@pytest.mark.skipif(FIXTURE is None, reason="tests/golden/quench_fixture.json not generated")
@pytest.mark.parametrize("precision,bound", [(64, 1e-9), (32, 1e-4)])
def test_tfim_quench_matches_the_oracle_taylor_plan(precision, bound):
    import torch
    from qmbed_b200 import learned
    sk = _sketcher()
    sites, g = FIXTURE["sites"], FIXTURE["g"]
    fields = np.asarray(FIXTURE["fields"])
    assert np.array_equal(fields, learned.tfim_instance(sites, g, FIXTURE["width"], FIXTURE["seed"]))
    op = learned.tfim_operator(sites, g, fields)
    n = op.dim
    interval = learned.lanczos_interval(op)
    state = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    state[-2] = 1.0
    probes = np.asarray(FIXTURE["probe_indices"])
    steps = [FIXTURE["dt"] * (k + 1) for k in range(10)]
    signs = None
    estimates = []
    for record in FIXTURE["records"]:
        learned.propagate_device(op, state, steps, interval, precision=precision)
        psi = state.cpu().numpy().view(np.complex128)
        if signs is None:
            signs = np.stack([sk.sketch_signs(r, n) for r in range(FIXTURE["sketch_rows"])])
        sketch = signs @ psi
        expected = np.array([complex(*v) for v in record["sketch"]])
        estimate = np.linalg.norm(sketch - expected) / np.sqrt(FIXTURE["sketch_rows"])
        estimates.append(estimate)
        probe_err = np.max(np.abs(psi[probes] - np.array([complex(*v) for v in record["probes"]])))
        norm_err = abs(np.linalg.norm(psi) - record["norm"])
        ret_err = abs(psi[-1] - complex(*record["return_amplitude"]))
        print(f"precision {precision} t={record['t']:.0f}: sketch estimate {estimate:.2e}, probes {probe_err:.2e}, "
              f"norm {norm_err:.2e}, return amplitude {ret_err:.2e}")
        # the estimate is within a factor ~1.5 of the distance; require a margin of 2
        assert estimate <= bound / 2
        assert probe_err <= bound and ret_err <= bound and norm_err <= bound

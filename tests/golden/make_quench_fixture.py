"""Oracle answer for the transverse-field Ising quench at 22 sites.

The quench workload (open chain, J = 1, g = 1, longitudinal fields
h_i ~ U[-2, 2] from numpy's default_rng(2024), Pauli normalisation,
|up...up> evolved to t = 10 in 100 steps of 0.1) is propagated by the oracle's
Taylor exponential-action plan (ExpmActionPlan, src/solve/mod.rs:116-248) in
complex128. The states (2^22 amplitudes each) are too large to commit, so the
fixture keeps, at t = 1, 2, ..., 10: the norm, the return amplitude
<up...up|psi(t)>, 64 seeded random projections of psi(t) (rows of +-1 from
sketch_signs below), from which the 2-norm distance to another state is
estimated, and 32 amplitudes at seeded indices.

    python tests/golden/make_quench_fixture.py

writes tests/golden/quench_fixture.json (about 6 minutes on one core).
"""

from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent / "quench_fixture.json"
SITES, G, WIDTH, SEED = 22, 1.0, 2.0, 2024
SKETCH_ROWS, SKETCH_SEED, PROBES = 64, 97, 32


def sketch_signs(row: int, n: int) -> np.ndarray:
    """+-1 entries of sketch row `row` over n amplitudes (SplitMix64 of (seed, row, index))."""
    z = (np.arange(n, dtype=np.uint64) + np.uint64(((SKETCH_SEED << 20) + row) << 32)) * np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    z ^= z >> np.uint64(31)
    return np.where((z >> np.uint64(63)) == 0, 1.0, -1.0)


def sketch(psi: np.ndarray) -> np.ndarray:
    return np.array([sketch_signs(r, len(psi)) @ psi for r in range(SKETCH_ROWS)])


def probe_indices(n: int) -> np.ndarray:
    return np.sort(np.random.default_rng(SKETCH_SEED).choice(n, PROBES, replace=False))


def terms(fields):
    bonds = [(i, i + 1) for i in range(SITES - 1)]
    return [("zz", [(-1.0, b) for b in bonds]), ("x", [(-G, (i,)) for i in range(SITES)]),
            ("z", [(float(h), (i,)) for i, h in enumerate(fields)])]


def main() -> None:
    sys.path.insert(0, str(ROOT))
    from oracle import oracle
    fields = np.random.default_rng(SEED).uniform(-WIDTH, WIDTH, SITES)
    t0 = time.time()
    op = oracle.Operator.build(oracle.Basis(SITES, normalization="pauli"), terms(fields), check_particles=False)
    n = op.dim
    psi = np.zeros(n, complex)
    psi[-1] = 1.0
    probes = probe_indices(n)
    records = []
    for step in range(1, 101):
        psi = op.expm_apply(-0.1j, psi)
        if step % 10 == 0:
            s = sketch(psi)
            records.append({"t": step / 10, "norm": float(np.linalg.norm(psi)),
                            "return_amplitude": [psi[-1].real, psi[-1].imag],
                            "sketch": [[v.real, v.imag] for v in s],
                            "probes": [[psi[i].real, psi[i].imag] for i in probes]})
            print(f"t={step / 10:.1f} norm={records[-1]['norm']:.15f} {time.time() - t0:.0f}s", flush=True)
    OUT.write_text(json.dumps({"sites": SITES, "g": G, "width": WIDTH, "seed": SEED, "fields": fields.tolist(),
                               "dt": 0.1, "steps": 100, "sketch_rows": SKETCH_ROWS, "sketch_seed": SKETCH_SEED,
                               "probe_indices": probe_indices(n).tolist(), "records": records,
                               "oracle_seconds": round(time.time() - t0)}, indent=0) + "\n")
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()

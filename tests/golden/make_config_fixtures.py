"""Oracle answers at the benchmark configurations' own sizes.

Writes tests/golden/config_fixtures.json (checked by
tests/test_golden_config.py on the CPU for its generator inputs and by
tests/test_gpu_config_parity.py on the GPU):

* every momentum sector of the L=26, up=13 chain (the batched scan's 26
  sectors) and the L=28 up=14 k=0 p=+1 sector: dimension, SHA-256 of the
  representatives (u64 little-endian) and of the orbit sizes (u16
  little-endian), and the first and last representatives;
* the L=28 XXZ chain of the XXZ benchmark line (periodic, J = 1, Delta drawn
  U[0.5, 1.5] from numpy's default_rng(28), Sz = 0, k = 0, p = +1): the
  oracle's 6 lowest eigenvalues at tolerance 1e-10 and their residuals.

Run from the repository root (the oracle library is built on demand):

    python tests/golden/make_config_fixtures.py [processes]
"""

from __future__ import annotations

import hashlib
import json
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent / "config_fixtures.json"


def sector_digest(args):
    sites, up, momentum, parity = args
    sys.path.insert(0, str(ROOT))
    from oracle import oracle
    t0 = time.time()
    basis = oracle.Basis(sites, up=up, momentum=momentum, parity=parity)
    states, orbits = basis.states()
    states = np.asarray(states, dtype="<u8")
    orbits = np.asarray(orbits, dtype="<u2")
    return {"sites": sites, "up": up, "momentum": momentum, "parity": parity, "dimension": int(len(states)),
            "states_sha256": hashlib.sha256(states.tobytes()).hexdigest(),
            "orbits_sha256": hashlib.sha256(orbits.tobytes()).hexdigest(),
            "head": [int(s) for s in states[:3]], "tail": [int(s) for s in states[-3:]],
            "oracle_seconds": round(time.time() - t0, 1)}


def xxz_eigenvalues(_):
    sys.path.insert(0, str(ROOT))
    from oracle import oracle
    sites = 28
    delta = float(np.random.default_rng(sites).uniform(0.5, 1.5))
    t0 = time.time()
    basis = oracle.Basis(sites, up=14, momentum=0, parity=1)
    op = oracle.Operator.build(basis, oracle.heisenberg_terms(sites, delta=delta))
    result = op.eigsh(6, tolerance=1e-10, seed=sites)
    return {"sites": sites, "up": 14, "momentum": 0, "parity": 1, "delta": delta, "seed": sites,
            "eigenpairs": 6, "tolerance": 1e-10, "dimension": len(basis),
            "eigenvalues": [float(v) for v in result.eigenvalues],
            "residuals": [float(v) for v in result.residuals], "iterations": int(result.iterations),
            "oracle_seconds": round(time.time() - t0, 1)}


def main() -> None:
    processes = int(sys.argv[1]) if len(sys.argv) > 1 else 8
    sectors = [(26, 13, k, None) for k in range(26)] + [(28, 14, 0, 1)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(processes) as pool:
        xxz = pool.apply_async(xxz_eigenvalues, (None,))
        digests = pool.map(sector_digest, sectors)
        xxz = xxz.get()
    OUT.write_text(json.dumps({"sectors": digests, "xxz": xxz}, indent=1) + "\n")
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()

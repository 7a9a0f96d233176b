"""Generate tests/golden/oracle_fixtures.npz from the CPU oracle.

The oracle restates the reference algorithms in C++ and is pinned by the
reference's own known answers (tests/golden/reference_anchors.json and
tests/test_oracle_anchors.py). This script records its outputs on small,
seeded inputs so that the GPU parity tests (tests/test_gpu_golden.py) compare
against committed numbers, and tests/test_golden_fixtures.py checks that the
oracle still reproduces them.

    python tests/golden/make_fixtures.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402

OUT = Path(__file__).resolve().parent / "oracle_fixtures.npz"


def tfim_terms(sites, j=1.0, g=1.0, fields=None, periodic=False):
    bonds = [(i, (i + 1) % sites) for i in range(sites if periodic else sites - 1)]
    terms = [("zz", [(-j, b) for b in bonds]), ("x", [(-g, (i,)) for i in range(sites)])]
    if fields is not None:
        terms.append(("z", [(float(h), (i,)) for i, h in enumerate(fields)]))
    return terms


def fixtures() -> dict:
    f = {}
    rng = np.random.default_rng(20261203)

    # Heisenberg (Delta = 0.85) on the real sector L=16, up=8, k=0, p=+1
    b = oracle.Basis(16, up=8, momentum=0, parity=1)
    op = oracle.Operator.build(b, oracle.heisenberg_terms(16, delta=0.85))
    reps, orbit = b.states()
    f["real_sector_states"] = reps.astype(np.uint64)
    f["real_sector_orbits"] = orbit.astype(np.uint16)
    x = oracle.deterministic_start(op.dim, 3)
    f["real_sector_x"] = x
    f["real_sector_hx"] = op.apply(x).real
    f["real_sector_eigenvalues"] = op.eigsh(4, tolerance=1e-12, seed=3).eigenvalues

    # the complex sector L=15, up=7, k=3 with a complex seeded vector
    b = oracle.Basis(15, up=7, momentum=3)
    op = oracle.Operator.build(b, oracle.heisenberg_terms(15, delta=1.1))
    reps, orbit = b.states()
    f["complex_sector_states"] = reps.astype(np.uint64)
    f["complex_sector_orbits"] = orbit.astype(np.uint16)
    z = rng.standard_normal(op.dim) + 1j * rng.standard_normal(op.dim)
    f["complex_sector_x"] = z
    f["complex_sector_hx"] = op.apply(z)
    f["complex_sector_eigenvalues"] = op.eigsh(3, tolerance=1e-12, seed=5).eigenvalues

    # XXZ L=20, k=0, p=+1, six lowest (the cfg-2 model at a CPU-feasible size)
    b = oracle.Basis(20, up=10, momentum=0, parity=1)
    op = oracle.Operator.build(b, oracle.heisenberg_terms(20, delta=1.3518))
    f["xxz20_eigenvalues"] = op.eigsh(6, tolerance=1e-12, seed=20).eigenvalues

    # transverse-field Ising chain with random fields, full space of 12 sites (Pauli)
    fields = np.random.default_rng(12).uniform(-2.0, 2.0, 12)
    b = oracle.Basis(12, normalization="pauli")
    op = oracle.Operator.build(b, tfim_terms(12, g=0.9, fields=fields))
    f["tfim12_fields"] = fields
    y = rng.standard_normal(op.dim) + 1j * rng.standard_normal(op.dim)
    f["tfim12_x"] = y
    f["tfim12_hx"] = op.apply(y)

    # thermal Lanczos on L=14, up=7, k=0, p=+1 from the deterministic start of seed 7
    b = oracle.Basis(14, up=7, momentum=0, parity=1)
    op = oracle.Operator.build(b, oracle.heisenberg_terms(14))
    v = oracle.deterministic_start(op.dim, 7)
    betas = np.array([0.0, 0.2, 1.0, 3.0])
    lz, e, m = op.thermal_iteration(v, betas, 40)
    f["ftlm14_betas"] = betas
    f["ftlm14_log_partition"] = lz
    f["ftlm14_energy"] = e
    f["ftlm14_krylov"] = np.array([m])

    # cross-sector shift: sum_j exp(-2 pi i 3 j / 12) S-_j from (up 6, k 1) to (up 5, k 4)
    src = oracle.Basis(12, up=6, momentum=1)
    tgt = oracle.Basis(12, up=5, momentum=4)
    terms = [("-", [(np.exp(-2j * np.pi * 3 * j / 12), (j,)) for j in range(12)])]
    w = rng.standard_normal(len(src)) + 1j * rng.standard_normal(len(src))
    f["shift12_x"] = w
    f["shift12_y"] = oracle.sector_shift(src, tgt, terms, w)
    return f


def main() -> None:
    f = fixtures()
    np.savez_compressed(OUT, **f)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(f)} arrays)")


if __name__ == "__main__":
    main()

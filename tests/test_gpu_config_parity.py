"""GPU sectors and solves against the oracle at the benchmark configurations' sizes.

* the 26 momentum sectors of the L=26 scan and the L=28 k=0 p=+1 sector:
  representatives and orbit sizes bit-exact (SHA-256 of the oracle's arrays,
  tests/golden/config_fixtures.json, written by make_config_fixtures.py);
* the L=28 XXZ chain: eigenvalues within 1e-10 relative of the oracle's;
* the L=34 k=0 p=+1 sector (the headline size, beyond the oracle's full
  lookup): the dimension equals the character-formula count, and random
  parent states map to the representative, phase and orbit size that the
  reference's per-orbit rule gives (oracle.orbit_images), through both the
  image table and the representative search.
"""

import hashlib
import json
import math
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIXTURES = json.loads((Path(__file__).resolve().parent / "golden" / "config_fixtures.json").read_text())


@pytest.fixture(scope="module")
def engine():
    import qmbed_b200.engine as module
    return module


def _digest(array, dtype):
    return hashlib.sha256(np.ascontiguousarray(array, dtype=dtype).tobytes()).hexdigest()


@pytest.mark.parametrize("entry", FIXTURES["sectors"], ids=lambda e: f"L{e['sites']}-k{e['momentum']}-p{e['parity']}")
def test_config_sector_bit_exact(engine, entry):
    basis = engine.GpuBasis(entry["sites"], up=entry["up"], momentum=entry["momentum"], parity=entry["parity"])
    assert len(basis) == entry["dimension"]
    lo, hi, orbit = basis.states()
    assert not hi.any()
    assert _digest(lo, "<u8") == entry["states_sha256"]
    assert _digest(orbit, "<u2") == entry["orbits_sha256"]
    assert lo[:3].tolist() == entry["head"] and lo[-3:].tolist() == entry["tail"]


@pytest.mark.parametrize("storage,mode", [("matrix_free", "fp64"), ("packed", "filtered"), ("matrix_free", "filtered"),
                                          ("packed", "mixed")])
def test_xxz_l28_eigenvalues_match_oracle(engine, storage, mode):
    ref = FIXTURES["xxz"]
    terms = engine.heisenberg_terms(ref["sites"], delta=ref["delta"])
    basis = engine.GpuBasis(ref["sites"], up=ref["up"], momentum=ref["momentum"], parity=ref["parity"])
    op = engine.GpuOperator(basis, terms, storage=storage)
    r = op.eigsh(ref["eigenpairs"], tolerance=ref["tolerance"], seed=ref["seed"], mode=mode)
    expected = np.asarray(ref["eigenvalues"])
    assert r.converged
    assert np.max(np.abs(r.eigenvalues - expected) / np.abs(expected)) <= 1e-10
    assert np.all(r.residuals <= ref["tolerance"] * np.maximum(np.abs(r.eigenvalues), 1.0))


def _random_weight_states(sites, weight, n, seed):
    rng = np.random.default_rng(seed)
    keys = rng.random((n, sites))
    positions = np.argsort(keys, axis=1)[:, :weight]
    return np.bitwise_or.reduce(np.left_shift(np.uint64(1), positions.astype(np.uint64)), axis=1)


@pytest.mark.parametrize("momentum,parity,samples", [(0, 1, 200_000), (5, None, 50_000)])
def test_l34_sector_dimension_and_images_follow_the_oracle_rule(engine, oracle, momentum, parity, samples):
    sites, up = 34, 17
    basis = engine.GpuBasis(sites, up=up, momentum=momentum, parity=parity)
    assert len(basis) == oracle.sector_dimension(sites, up, momentum, parity)
    states = _random_weight_states(sites, up, samples, seed=momentum)
    rep, phase, orbit = oracle.orbit_images(sites, states, momentum=momentum, parity=parity)
    lo, _, orbits = basis.states()
    for resolve in (basis.table_images, lambda s: basis.images(s)):
        index, gphase, gorbit = resolve(states)
        kept = orbit > 0
        assert np.array_equal(index >= 0, kept)
        assert np.array_equal(lo[index[kept]], rep[kept])
        assert np.array_equal(gorbit[kept].astype(np.uint64), orbit[kept])
        assert np.array_equal(orbits[index[kept]].astype(np.uint64), orbit[kept])
        assert np.max(np.abs(gphase[kept] - phase[kept])) <= 1e-12

"""The committed oracle fixtures (tests/golden/oracle_fixtures.npz, written by
tests/golden/make_fixtures.py) are what the oracle computes today: integer
arrays bit-identical, floating-point values within 1e-13 relative."""

import importlib.util
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_oracle_reproduces_the_committed_fixtures():
    spec = importlib.util.spec_from_file_location("make_fixtures", GOLDEN / "make_fixtures.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    fresh = module.fixtures()
    committed = np.load(GOLDEN / "oracle_fixtures.npz")
    assert sorted(fresh) == sorted(committed.files)
    for name, value in fresh.items():
        stored = committed[name]
        assert stored.shape == np.shape(value), name
        if np.issubdtype(stored.dtype, np.integer):
            np.testing.assert_array_equal(stored, value, err_msg=name)
        else:
            scale = max(1.0, float(np.max(np.abs(stored))))
            np.testing.assert_allclose(value, stored, rtol=0, atol=1e-13 * scale, err_msg=name)

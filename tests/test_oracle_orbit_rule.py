"""The oracle's per-orbit image rule and sector-dimension count (CPU).

Both serve the GPU checks at sizes where the oracle cannot build the full
sector lookup (L=34): they must agree with the full construction
(spin_symmetry_sector restated in oracle/qmbed_oracle.cpp) wherever that is
feasible.
"""

import numpy as np
import pytest


@pytest.mark.parametrize("sites,up,momentum,parity", [(14, 7, 0, 1), (14, 7, 3, None), (16, 8, 8, -1),
                                                       (12, None, 0, -1), (15, 7, None, 1), (13, 6, 5, None)])
def test_orbit_images_equal_the_full_lookup(oracle, sites, up, momentum, parity):
    basis = oracle.Basis(sites, up=up, momentum=momentum, parity=parity)
    rng = np.random.default_rng(sites)
    states = rng.integers(0, 1 << sites, size=3000, dtype=np.uint64)
    if up is not None:
        states = states[[bin(int(s)).count("1") == up for s in states]]
    rep, phase, orbit = oracle.orbit_images(sites, states, momentum=momentum, parity=parity)
    for s, r, ph, o in zip(states.tolist(), rep.tolist(), phase, orbit.tolist()):
        image = basis.image(int(s))
        if image is None:
            assert o == 0
            continue
        assert (r, o) == (image[0], image[2])
        assert ph == image[1]  # the same per-orbit code: identical doubles


@pytest.mark.parametrize("sites,up,momentum,parity", [(20, 10, 0, None), (20, 10, 0, 1), (16, 8, 8, -1),
                                                       (15, 7, 3, None), (18, 9, 6, None), (12, 6, 0, -1),
                                                       (14, None, 0, 1), (13, None, 4, None)])
def test_sector_dimension_counts_the_enumerated_sector(oracle, sites, up, momentum, parity):
    weights = [up] if up is not None else range(sites + 1)
    count = sum(oracle.sector_dimension(sites, w, momentum, parity) for w in weights)
    assert count == len(oracle.Basis(sites, up=up, momentum=momentum, parity=parity))

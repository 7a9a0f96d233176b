"""Host logic of the learned eigsh hint, without a GPU.

The network is replaced by a stand-in with fixed outputs, so the features,
the padding of the predicted interval and the restart-size rule are checked
on their own: the interval is [E0, E_max] widened by the margin on both
sides, the gap is returned in energy units, and the restart keeps the wanted
pairs and two more only when the predicted relative gap is small.
"""

import numpy as np
import pytest

from qmbed_b200 import learned


class _FixedNetwork:
    def __init__(self, e0_per_site, emax_per_site, gap_times_sites):
        self.out = np.array([[e0_per_site, emax_per_site, gap_times_sites]], np.float32)

    def predict(self, x):
        assert np.asarray(x).shape[-1] == len(learned.CHAIN_FEATURES)
        return self.out


def test_chain_features():
    f = learned.chain_features(28, 0.25, 1.1, 0)
    assert f.dtype == np.float32 and f.shape == (len(learned.CHAIN_FEATURES),)
    assert np.allclose(f, [1 / 28, 0.25, 1.1, 1.0, 1.0, 1.0])
    g = learned.chain_features(26, 0.0, 0.9, 13)
    assert np.allclose(g, [1 / 26, 0.0, 0.9, -1.0, 0.0, 0.0])


@pytest.mark.parametrize("gap_times_sites,expected_keep", [(4.0, 6), (40.0, 0)])
def test_hint_interval_and_restart_rule(gap_times_sites, expected_keep):
    model = learned.ChainSpectrum(mlp=_FixedNetwork(-0.44, 0.25, gap_times_sites), margin=0.03)
    hint = model.hint(34, 0.0, 1.0, 0, eigenpairs=4, krylov_dimension=40)
    e0, emax, width = -0.44 * 34, 0.25 * 34, (0.25 + 0.44) * 34
    assert hint["lower"] == pytest.approx(e0 - 0.03 * width, rel=1e-6)
    assert hint["upper"] == pytest.approx(emax + 0.03 * width, rel=1e-6)
    assert hint["gap"] == pytest.approx(gap_times_sites / 34, rel=1e-6)
    assert hint["restart_keep"] == expected_keep
    assert hint["check_steps"] == 8


def test_negative_gap_predictions_are_clipped():
    model = learned.ChainSpectrum(mlp=_FixedNetwork(-0.44, 0.25, -1.0))
    assert model.predict(20, 0.1, 1.0, 0)[2] == 0.0


@pytest.mark.parametrize("e0,emax,gap", [(float("nan"), 0.25, 4.0), (-0.44, float("inf"), 4.0),
                                         (-0.44, 0.25, float("nan")), (0.3, 0.25, 4.0)])
def test_unusable_predictions_give_the_empty_hint(e0, emax, gap):
    """A non-finite prediction or an inverted interval must not reach the solver
    as an interval: the hint is empty (lower = upper = 0), so the solver takes
    its own Lanczos bounds and the reference restart size."""
    import json
    model = learned.ChainSpectrum(mlp=_FixedNetwork(e0, emax, gap))
    hint = model.hint(28, 0.0, 1.0, 0, eigenpairs=6, krylov_dimension=40)
    assert hint["usable"] is False
    assert hint["lower"] == hint["upper"] == 0.0 and hint["gap"] == 0.0 and hint["restart_keep"] == 0
    json.dumps(hint, allow_nan=False)  # reported values stay valid JSON


def test_usable_prediction_is_marked():
    model = learned.ChainSpectrum(mlp=_FixedNetwork(-0.44, 0.25, 4.0))
    assert model.hint(28, 0.0, 1.0, 0, eigenpairs=6)["usable"] is True


class _FixedBoundsNetwork:
    def __init__(self, lo_per_site, hi_per_site):
        self.out = np.array([[lo_per_site, hi_per_site]], np.float32)

    def predict(self, x):
        assert np.asarray(x).shape[-1] == len(learned.FEATURES)
        return self.out


@pytest.mark.parametrize("lo,hi,source", [(-1.9, 1.9, "learned"), (-1.0, 1.0, "lanczos"),
                                          (float("-inf"), float("inf"), "lanczos"),
                                          (float("nan"), 1.9, "lanczos"), (1.9, -1.9, "lanczos")])
def test_quench_interval_check(monkeypatch, lo, hi, source):
    """The Chebyshev interval is the network's only when it is finite, ordered
    and holds the short Lanczos run's Ritz extremes; otherwise the plain
    Lanczos estimate replaces it."""
    sites = 10
    monkeypatch.setattr(learned, "lanczos_extremes", lambda op, steps, seed=0: np.array([-15.0, 15.0, 0.1, 0.1]))
    monkeypatch.setattr(learned, "lanczos_interval",
                        lambda op, seed=0: learned.Interval(-16.0, 16.0, "lanczos", 40))
    bounds = learned.LearnedBounds(mlp=_FixedBoundsNetwork(lo, hi), margin=0.03, check_steps=8)
    interval = bounds.interval(None, sites, 1.0, 1.0, np.zeros(sites))
    assert interval.source == source
    assert np.isfinite(interval.e_min) and np.isfinite(interval.e_max) and interval.e_min < interval.e_max
    if source == "learned":
        assert interval.e_min <= -15.0 and interval.e_max >= 15.0 and interval.applications == 8
    else:
        assert (interval.e_min, interval.e_max, interval.applications) == (-16.0, 16.0, 48)


def test_network_calls_check_shapes_before_the_library():
    """The library reads rows x width floats from the arrays it is given, so a
    wrong width is refused in Python before any call (a network shell without
    a device handle is enough to show it)."""
    net = object.__new__(learned.GpuMlp)
    net.inputs, net.outputs, net.handle = 6, 3, None
    good_x, good_y = np.zeros((4, 6), np.float32), np.zeros((4, 3), np.float32)
    with pytest.raises(ValueError):
        net.predict(np.zeros((4, 5)))
    with pytest.raises(ValueError):
        net.train(np.zeros((4, 7)), good_y)
    with pytest.raises(ValueError):
        net.train(good_x, np.zeros((4, 2)))
    with pytest.raises(ValueError):
        net.gradients(good_x, np.zeros((5, 3)))
    x, y = net._samples(good_x[0], good_y[0])  # one sample as 1-D rows
    assert x.shape == (1, 6) and y.shape == (1, 3)

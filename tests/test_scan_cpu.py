"""Host side of the batched scan, without a GPU: the J1-J2 workload's
components and scan points, and the argument checks that run before the
library is called."""

import numpy as np
import pytest

from qmbed_b200 import scan


class _Component:
    """Stands in for a GpuOperator; the checks under test fail before its handle is used."""
    handle = None


def test_j1j2_components_and_points():
    terms = scan.j1j2_component_terms(8)
    assert len(terms) == 4
    assert [t[0] for t in terms[0]] == ["zz"] and [t[0] for t in terms[1]] == ["+-", "-+"]
    assert all(len(couplings) == 8 for component in terms for _, couplings in component)
    assert terms[2][0][1][7][1] == (7, 1)  # next-nearest bonds wrap around the ring
    points = scan.j1j2_scan_points(64, seed=3)
    assert points.shape == (64, 4)
    delta, ones, j2_delta, j2 = points.T
    assert np.all(ones == 1.0) and np.allclose(j2, np.linspace(0.0, 0.5, 64))
    assert np.allclose(j2_delta, j2 * delta) and np.all((0.8 <= delta) & (delta <= 1.2))
    assert np.array_equal(points, scan.j1j2_scan_points(64, seed=3))


@pytest.mark.parametrize("components,coefficients,eigenpairs", [
    ([], np.ones((2, 4)), 2),
    ([[_Component()] * 4, [_Component()] * 3], np.ones((2, 4)), 2),
    ([[_Component()] * 4], np.ones(4), 2),
    ([[_Component()] * 4], np.ones((2, 3)), 2),
    ([[_Component()] * 4], np.ones((0, 4)), 2),
    ([[_Component()] * 4], np.ones((2, 4)), 0),
])
def test_scan_arguments_are_checked_before_the_library(components, coefficients, eigenpairs):
    with pytest.raises(ValueError):
        scan.scan_lowest(components, coefficients, eigenpairs=eigenpairs)

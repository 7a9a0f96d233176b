"""Host-side argument checks of the engine's host-buffer entries, without a GPU.

The C entries behind GpuOperator.apply / eigsh / evolve / expm_lanczos /
chebyshev_evolve / expm_apply read the sector dimension's worth of values
from the buffers they are given, so vectors of another length must be
refused in Python with the library's dimension-mismatch error (status 9)
before any call. An operator shell with a fixed dimension and no device
handle shows it.
"""

import numpy as np
import pytest

from qmbed_b200 import QmbedError, engine


class _Operator(engine.GpuOperator):
    dim = 6
    is_real = True

    def __init__(self):
        self.handle = None


@pytest.mark.parametrize("call", [
    lambda op: op.apply(np.zeros(5)),
    lambda op: op.apply(np.zeros((2, 6))),
    lambda op: op.eigsh(1, initial=np.zeros((2, 5))),
    lambda op: op.evolve(np.zeros(7, complex), [1.0]),
    lambda op: op.expm_lanczos(np.zeros(5), 1.0),
    lambda op: op.chebyshev_evolve(np.zeros(5, complex), [1.0]),
    lambda op: op.expm_apply(-1j, np.zeros((3, 5))),
])
def test_wrong_length_vectors_are_dimension_mismatches(call):
    with pytest.raises(QmbedError) as e:
        call(_Operator())
    assert e.value.code == 9 and str(e.value).startswith("dimension mismatch")


def test_sector_vectors_shapes():
    one = engine._sector_vectors([1, 2, 3], 3, np.complex128, "x")
    assert one.shape == (3,) and one.dtype == np.complex128 and one.flags.c_contiguous
    rows = engine._sector_vectors(np.arange(3.0), 3, np.complex128, "x", batch=True)
    assert rows.shape == (1, 3)
    rows = engine._sector_vectors(np.ones((4, 3)), 3, np.float64, "x", batch=True)
    assert rows.shape == (4, 3)

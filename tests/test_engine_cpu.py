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


@pytest.mark.parametrize("call,code", [
    (lambda op, t: op.apply_device(t.zeros(5, dtype=t.float64), t.zeros(6, dtype=t.float64)), 9),
    (lambda op, t: op.apply_device(t.zeros(6, dtype=t.float32), t.zeros(6, dtype=t.float32), precision=64), 9),
    (lambda op, t: op.apply_device(t.zeros(6, dtype=t.float64), t.zeros(6, dtype=t.float64),
                                   complex_vectors=True), 9),
    (lambda op, t: op.apply_device(t.zeros(24, dtype=t.float64)[::2], t.zeros(6, dtype=t.float64)), 8),
    (lambda op, t: op.apply_device_noalloc(t.zeros(6, dtype=t.float64), t.zeros(5, dtype=t.float64)), 9),
    (lambda op, t: op.apply_block_device(t.zeros(48), t.zeros(47), nb=8, precision=32), 9),
    (lambda op, t: op.apply_block_device(t.zeros(48), t.zeros(48), nb=8, precision=32, p=t.zeros(40)), 9),
    (lambda op, t: op.chebyshev_evolve_device(t.zeros(6, dtype=t.complex64), [1.0]), 9),
])
def test_device_operands_are_checked_before_the_library(call, code):
    """Device entries refuse tensors smaller than the action's span (status 9)
    and strided views (status 8) before looking at the device, so CPU tensors
    show both checks here."""
    import torch
    with pytest.raises(QmbedError) as e:
        call(_Operator(), torch)
    assert e.value.code == code, str(e.value)
    assert "CUDA tensor" not in str(e.value)


def test_host_tensors_are_refused_by_device_entries():
    import torch
    with pytest.raises(QmbedError) as e:
        _Operator().apply_device(torch.zeros(6, dtype=torch.float64), torch.zeros(6, dtype=torch.float64))
    assert e.value.code == 8 and "CUDA tensor" in str(e.value)


def test_lanczos_entries_check_the_vector_length():
    from qmbed_b200 import lanczos
    for call in (lambda: lanczos.LanczosBasis(_Operator(), np.zeros(5), 4),
                 lambda: lanczos.thermal_iteration(_Operator(), np.zeros(7), [1.0], 4)):
        with pytest.raises(QmbedError) as e:
            call()
        assert e.value.code == 9


def test_sector_shift_and_row_slab_device_operands():
    import torch
    from qmbed_b200 import spectrum
    from qmbed_b200.distributed import RowPartition, gpu_slab
    shift = object.__new__(spectrum.SectorShift)
    shift.handle, shift.source, shift.target = None, [0] * 6, [0] * 4
    with pytest.raises(QmbedError) as e:
        shift.apply_device(torch.zeros(5, dtype=torch.complex128), torch.zeros(4, dtype=torch.complex128))
    assert e.value.code == 9 and "source-sector" in str(e.value)
    with pytest.raises(QmbedError) as e:
        shift.apply_device(torch.zeros(6, dtype=torch.complex128), torch.zeros(3, dtype=torch.complex128))
    assert e.value.code == 9 and "target-sector" in str(e.value)
    part = RowPartition(10, 3)  # blocks of 4: rank 1 owns rows 4..7
    slab = gpu_slab(_Operator(), part, 1, precision=64)
    with pytest.raises(QmbedError) as e:
        slab(torch.zeros(9, dtype=torch.float64), torch.zeros(4, dtype=torch.float64))
    assert e.value.code == 9 and "gathered" in str(e.value)
    with pytest.raises(QmbedError) as e:
        slab(torch.zeros(12, dtype=torch.float64), torch.zeros(3, dtype=torch.float64))
    assert e.value.code == 9 and "slab output" in str(e.value)


def test_images_need_matching_state_words():
    basis = object.__new__(engine.GpuBasis)
    basis.handle = None
    with pytest.raises(QmbedError) as e:
        basis.images(np.arange(4), np.zeros(3))
    assert e.value.code == 9


class _FakeCudaTensor:
    """A CUDA tensor's size, layout and device attributes, for the host checks."""

    def __init__(self, numel, element_size, index):
        self._numel, self._element_size = numel, element_size
        self.is_cuda = True
        self.device = type("Device", (), {"index": index})()

    def numel(self):
        return self._numel

    def element_size(self):
        return self._element_size

    def is_contiguous(self):
        return True

    def data_ptr(self):
        return 0


def test_tensors_on_another_gpu_are_refused():
    op = _Operator()
    op.basis = type("Basis", (), {"device": 0})()
    with pytest.raises(QmbedError) as e:
        op.apply_device(_FakeCudaTensor(6, 8, 0), _FakeCudaTensor(6, 8, 1))
    assert e.value.code == 8 and "cuda:1" in str(e.value)

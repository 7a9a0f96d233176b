"""The allocation-free H.v entry point against the regular one.

qmbed_gpu_operator_apply_device_noalloc serves callers that cannot let the
library allocate device memory (they own all GPU memory through their own
pool or budget, or cannot take the device synchronisation of cudaMalloc in
their loop). It must give the same result as qmbed_gpu_operator_apply_device,
call after call, and refuse vectors above its fixed 32 MiB scratch. This file
is collected last so a failure here leaves every other test already run.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _operator(sites, momentum, parity, storage="packed"):
    from oracle import oracle
    from qmbed_b200 import GpuBasis, GpuOperator
    return GpuOperator(GpuBasis(sites, up=sites // 2, momentum=momentum, parity=parity),
                       oracle.heisenberg_terms(sites, delta=0.85), storage=storage)


def _free_device_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _compare(op, n, precision, complex_vectors, seed):
    import torch
    dtype = torch.float64 if precision == 64 else torch.float32
    width = 2 * n if complex_vectors else n
    tol = 1e-13 if precision == 64 else 1e-6
    generator = torch.Generator(device="cuda").manual_seed(seed)
    for call in range(2):
        x = torch.randn(width, dtype=dtype, device="cuda", generator=generator)
        y_regular = torch.empty_like(x)
        y_noalloc = torch.full_like(x, float("nan"))
        op.apply_device(x, y_regular, precision=precision, complex_vectors=complex_vectors)
        op.apply_device_noalloc(x, y_noalloc, precision=precision, complex_vectors=complex_vectors)
        torch.cuda.synchronize()
        scale = max(float(torch.linalg.vector_norm(y_regular.double())), 1.0)
        error = float(torch.linalg.vector_norm((y_noalloc - y_regular).double()))
        assert error <= tol * scale, (call, error, scale)


@pytest.mark.parametrize("sites,momentum,parity,precision,complex_vectors", [
    (24, 0, 1, 64, False),   # real sector, packed rows, FP64
    (24, 0, 1, 32, False),   # real sector, packed rows, FP32
    (22, 3, None, 64, True),  # complex sector, explicit-value rows
    (22, 11, -1, 64, False),  # k = pi sector
])
def test_noalloc_matches_regular_apply_on_consecutive_calls(sites, momentum, parity, precision, complex_vectors):
    import torch
    op = _operator(sites, momentum, parity)
    n = op.dim
    dtype = torch.float64 if precision == 64 else torch.float32
    width = 2 * n if complex_vectors else n
    tol = 1e-13 if precision == 64 else 1e-6
    generator = torch.Generator(device="cuda").manual_seed(11)
    for call in range(2):  # two calls in a row share the scratch array
        x = torch.randn(width, dtype=dtype, device="cuda", generator=generator)
        y_regular = torch.empty_like(x)
        y_noalloc = torch.full_like(x, float("nan"))
        op.apply_device(x, y_regular, precision=precision, complex_vectors=complex_vectors)
        op.apply_device_noalloc(x, y_noalloc, precision=precision, complex_vectors=complex_vectors)
        torch.cuda.synchronize()
        scale = max(float(torch.linalg.vector_norm(y_regular.double())), 1.0)
        error = float(torch.linalg.vector_norm((y_noalloc - y_regular).double()))
        assert error <= tol * scale, (call, error, scale)


def test_noalloc_refuses_vectors_above_its_scratch():
    import torch
    from qmbed_b200 import QmbedError
    op = _operator(30, 0, 1)  # 2.6M rows: complex FP64 vectors need 42 MB > 32 MiB
    n = op.dim
    assert n * 16 > (1 << 25)
    x = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    with pytest.raises(QmbedError) as error:
        op.apply_device_noalloc(x, y, precision=64, complex_vectors=True)
    assert error.value.code == 9 and "at most 33554432 bytes" in str(error.value)
    # a real FP64 vector of the same operator fits (21 MB) and agrees with the regular path
    xr = torch.rand(n, dtype=torch.float64, device="cuda")
    y1, y2 = torch.empty_like(xr), torch.empty_like(xr)
    op.apply_device(xr, y1, precision=64)
    op.apply_device_noalloc(xr, y2, precision=64)
    torch.cuda.synchronize()
    assert float(torch.linalg.vector_norm(y1 - y2)) <= 1e-13 * float(torch.linalg.vector_norm(y1))


def test_noalloc_paths_without_scratch():
    """Operators whose action needs no scaled vector: wide rows of a real
    operator applied to complex vectors (they run on the fly), a full-space
    flip chain (the tile kernel instead of the flip-chain kernels, which
    allocate tables) and stored rows without symmetry. None has a size limit."""
    from oracle import oracle
    from qmbed_b200 import GpuBasis, GpuOperator
    from qmbed_b200.engine import tfim_terms
    wide = _operator(22, 0, 1, storage="explicit")
    _compare(wide, wide.dim, 64, True, 1)
    _compare(wide, wide.dim, 32, True, 2)
    chain = GpuOperator(GpuBasis(18, normalization="pauli_cartesian"),
                        tfim_terms(18, g=0.8, fields=np.linspace(-1, 1, 18)), storage="matrix_free",
                        check_particles=False)
    _compare(chain, chain.dim, 64, True, 3)
    _compare(chain, chain.dim, 32, False, 4)
    plain = GpuOperator(GpuBasis(18, up=9), oracle.heisenberg_terms(18, delta=1.2), storage="packed")
    _compare(plain, plain.dim, 64, False, 5)
    # above the scratch size: 2^22 complex FP64 elements = 64 MiB, no scratch involved
    big = GpuOperator(GpuBasis(22, normalization="pauli_cartesian"), tfim_terms(22, g=1.1), storage="matrix_free",
                      check_particles=False)
    _compare(big, big.dim, 64, True, 6)


def test_noalloc_takes_no_device_memory():
    """Free device memory is unchanged across calls on a fresh operator whose
    regular path once allocated (wide real rows with complex vectors)."""
    import torch
    warm = _operator(28, 0, 1, storage="explicit")
    n = warm.dim
    x = torch.randn(2 * n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    warm.apply_device_noalloc(x, y, precision=64, complex_vectors=True)  # loads the kernels
    op = _operator(28, 0, 1, storage="explicit")
    before = _free_device_bytes()
    for _ in range(2):
        op.apply_device_noalloc(x, y, precision=64, complex_vectors=True)
    assert _free_device_bytes() == before

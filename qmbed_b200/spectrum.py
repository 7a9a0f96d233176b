"""Cross-sector actions and broadened spectral functions on the GPU.

``SectorShift`` is the reference's apply_sector_shift
(src/operator/mod.rs:2305-2351): local terms applied to vectors of one
sector and reduced into another (momentum, parity and particle number may
differ). ``spectral_function`` is src/dynamics/mod.rs:964-1021: the probe
applied to a source state, then the Lehmann sum over every eigenpair of the
target Hamiltonian (at most 128 states) or over the Lanczos spectral measure,
broadened by Lorentzians.
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib
from .engine import GpuBasis, GpuOperator, _device_operands, _ptr, encode_terms


class SectorShift:
    """Terms acting from `source` into `target` (same sites and normalisation)."""

    def __init__(self, source: GpuBasis, target: GpuBasis, terms):
        arity, symbols, n_couplings, coefficients, sites = encode_terms(terms)
        handle = ctypes.c_void_p()
        check(lib().qmbed_gpu_shift_create(source.handle, target.handle, len(arity), _ptr(arity), symbols,
                                           _ptr(n_couplings), _ptr(coefficients), _ptr(sites), ctypes.byref(handle)))
        self.handle = handle
        self.source, self.target = source, target

    def close(self):
        if getattr(self, "handle", None):
            lib().qmbed_gpu_shift_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass

    def apply(self, x) -> np.ndarray:
        xin = np.ascontiguousarray(np.asarray(x, np.complex128))
        y = np.zeros(len(self.target), np.complex128)
        check(lib().qmbed_gpu_shift_apply_host(self.handle, xin.size, _ptr(xin), y.size, _ptr(y)))
        return y

    def apply_device(self, x, y, stream=None) -> None:
        """y = shift(x) on device tensors (complex128 ``data_ptr()``)."""
        _device_operands(("the source-sector vector", x, 16 * len(self.source)),
                         ("the target-sector vector", y, 16 * len(self.target)),
                         device=getattr(self.source, "device", None))
        check(lib().qmbed_gpu_shift_apply_device(self.handle, _ptr(x), _ptr(y),
                                                 None if stream is None else ctypes.c_void_p(stream)))


def spectral_function(target: GpuOperator, probe: SectorShift, source, frequencies, reference_energy: float,
                      broadening: float, krylov_dimension: int = 64, tolerance: float = 1e-10) -> np.ndarray:
    """S(omega) = sum_e w_e eta / (pi ((omega + E_ref - E_e)^2 + eta^2)) for the
    weights w_e = |<e|probe|source>|^2 of the target Hamiltonian."""
    x = np.ascontiguousarray(np.asarray(source, np.complex128))
    f = np.ascontiguousarray(np.atleast_1d(np.asarray(frequencies, np.float64)))
    out = np.zeros(max(f.size, 1))
    check(lib().qmbed_gpu_spectral_function(target.handle, probe.handle, x.size, _ptr(x), f.size, _ptr(f),
                                            float(reference_energy), float(broadening), int(krylov_dimension),
                                            float(tolerance), _ptr(out)))
    return out[:f.size]

"""Batched parameter scans: lowest eigenvalues of every sector x point.

A family H(p) = sum_k c_k(p) A_k is given by its components A_k, assembled
once per sector with explicit-value rows; qmbed_gpu_scan_lowest then runs
one batched Lanczos over every (sector, point) pair. The J1-J2 chain scan
(all momentum sectors at half filling, J2 on a uniform grid, Delta drawn per
point on both zz terms) is provided as the standard workload.
"""

from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib
from .engine import GpuBasis, GpuOperator


def scan_lowest(components, coefficients, eigenpairs: int = 2, tolerance: float = 1e-10, max_steps: int = 600,
                seed: int = 0):
    """components[s][k]: GpuOperator A_k of sector s (explicit storage, one basis per sector);
    coefficients: points x components. Returns (eigenvalues[s, p, eigenpairs], steps[s, p], info);
    info also holds the FP64 residual of every reported pair and the top Ritz value of every pair."""
    sectors = len(components)
    k = len(components[0]) if sectors else 0
    if sectors < 1 or k < 1 or any(len(row) != k for row in components):
        raise ValueError("a scan needs at least one sector, each with the same (nonzero) number of components")
    coef = np.ascontiguousarray(coefficients, np.float64)
    if coef.ndim != 2 or coef.shape[0] < 1 or coef.shape[1] != k:
        raise ValueError(f"coefficients must be a (points x {k}) array; got shape {coef.shape}")
    if eigenpairs < 1:
        raise ValueError("eigenpairs must be at least 1")
    points = coef.shape[0]
    handles = (ctypes.c_void_p * (sectors * k))(*[op.handle.value for row in components for op in row])
    values = np.full((sectors, points, eigenpairs), np.nan)
    residuals = np.full((sectors, points, eigenpairs), np.nan)
    e_max = np.full((sectors, points), np.nan)
    steps = np.zeros((sectors, points), np.int32)
    info = np.zeros(11)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    check(lib().qmbed_gpu_scan_solve(sectors, k, ctypes.cast(handles, ctypes.c_void_p), points, ptr(coef),
                                     eigenpairs, tolerance, max_steps, seed, ptr(values), ptr(residuals), ptr(e_max),
                                     ptr(steps), ptr(info)))
    return values, steps, {"total_steps": int(info[0]), "applications": int(info[1]),
                           "verification_applications": int(info[2]), "graph": bool(info[3]),
                           "pass1_seconds": float(info[4]), "seconds": float(info[5]),
                           "max_relative_residual": float(info[6]), "merged_copies": int(info[7]),
                           "tuned_blocks_per_sm": int(info[8]), "tuning_chunk_ms": float(info[9]),
                           "tuned_rows_per_warp": int(info[10]),
                           "residuals": residuals, "e_max": e_max}


def barrier_selftest(device: int = 0) -> int:
    """Status of the persistent scan kernel's barrier run one block short (1: timed out as designed)."""
    status = ctypes.c_int(-1)
    check(lib().qmbed_gpu_scan_barrier_selftest(device, ctypes.byref(status)))
    return status.value


def j1j2_component_terms(sites: int):
    """The four components of the J1-J2 chain: zz and flips on nearest and next-nearest bonds."""
    nn = [(i, (i + 1) % sites) for i in range(sites)]
    nnn = [(i, (i + 2) % sites) for i in range(sites)]
    flips = lambda bonds: [("+-", [(0.5, b) for b in bonds]), ("-+", [(0.5, b) for b in bonds])]
    return [[("zz", [(1.0, b) for b in nn])], flips(nn), [("zz", [(1.0, b) for b in nnn])], flips(nnn)]


def j1j2_scan_points(count: int, seed: int = 0, j2_max: float = 0.5, delta_range=(0.8, 1.2)):
    """Coefficients (points x 4) of H = Delta (zz1 + J2 zz2) + flips1 + J2 flips2 (J1 = 1):
    J2 on a uniform grid in [0, j2_max], Delta drawn per point from `seed`."""
    j2 = np.linspace(0.0, j2_max, count)
    delta = np.random.default_rng(seed).uniform(*delta_range, count)
    return np.stack([delta, np.ones(count), j2 * delta, j2], axis=1)


def j1j2_sectors(sites: int, momenta=None, device: int = 0):
    """Component operators of every momentum sector at half filling (explicit storage)."""
    momenta = range(sites) if momenta is None else momenta
    out = []
    for k in momenta:
        basis = GpuBasis(sites, up=sites // 2, momentum=k, device=device)
        out.append([GpuOperator(basis, terms, storage="explicit") for terms in j1j2_component_terms(sites)])
    return out

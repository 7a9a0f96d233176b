"""Learned spectral bounds: the Chebyshev propagator and the eigsh hint.

A small ReLU network (4 hidden layers of 128 by default) maps the parameters
of a transverse-field Ising chain with random longitudinal fields (size L,
transverse field g, disorder width W, and statistics of the drawn fields) to
its spectral extremes per site, E_min / L and E_max / L. Its training set is
produced by this library's own GPU eigensolver on small chains, and it is
trained and evaluated by the library's GPU kernels (qmbed_gpu_mlp_*).

A prediction is only used after a short Lanczos check on the actual operator:
the Ritz extremes of a few-step run lie inside the spectrum, so an interval
that fails to contain them is wrong and the plain Lanczos bound estimate is
used instead. The norm of the propagated state is the second check: if it
drifts, the interval missed part of the spectrum and the propagation is
repeated with the guaranteed bound +-sum|coefficients|.

The second network (ChainSpectrum) maps the couplings, size and momentum of a
J1-J2 / XXZ chain sector to its lowest eigenvalue, its largest eigenvalue and
the gap above the lowest one. Its training set is what the batched scan
solver (qmbed_gpu_scan_solve) returns for every sector and scan point. Its
prediction becomes an eigsh hint: the padded interval replaces the filtered
solver's own Lanczos bound estimate once a short Lanczos check finds the
interval holding its Ritz values, and the predicted relative gap sets how
many Ritz vectors the plain thick restart keeps per cycle.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._lib import check, lib
from .engine import GpuBasis, GpuOperator, _ptr, tfim_terms

FEATURES = ("inverse_sites", "g", "W", "mean_h", "std_h", "mean_abs_h", "mean_site_energy", "mean_half_step",
            "mean_half_pair")
TARGETS = ("e_min_per_site", "e_max_per_site")


class GpuMlp:
    """Fully connected ReLU network trained and evaluated on the GPU."""

    def __init__(self, inputs: int, outputs: int, width: int = 128, hidden_layers: int = 4, seed: int = 0,
                 device: int = 0):
        handle = ctypes.c_void_p()
        check(lib().qmbed_gpu_mlp_create(device, inputs, outputs, width, hidden_layers, seed, ctypes.byref(handle)))
        self.handle = handle
        self.inputs, self.outputs, self.width, self.hidden_layers = inputs, outputs, width, hidden_layers

    def __del__(self):
        handle = getattr(self, "handle", None)
        if handle:
            try:
                lib().qmbed_gpu_mlp_destroy(handle)
            except Exception:  # interpreter shutdown
                pass
            self.handle = None

    @property
    def parameter_count(self) -> int:
        count = ctypes.c_uint64()
        check(lib().qmbed_gpu_mlp_parameter_count(self.handle, ctypes.byref(count)))
        return count.value

    def parameters(self) -> np.ndarray:
        out = np.zeros(self.parameter_count, np.float32)
        check(lib().qmbed_gpu_mlp_get_parameters(self.handle, _ptr(out)))
        return out

    def set_parameters(self, params) -> None:
        p = np.ascontiguousarray(params, np.float32).ravel()
        if p.size != self.parameter_count:
            raise ValueError(f"expected {self.parameter_count} parameters, got {p.size}")
        check(lib().qmbed_gpu_mlp_set_parameters(self.handle, _ptr(p)))

    def scaling(self):
        arrays = [np.zeros(self.inputs, np.float32), np.zeros(self.inputs, np.float32),
                  np.zeros(self.outputs, np.float32), np.zeros(self.outputs, np.float32)]
        check(lib().qmbed_gpu_mlp_get_scaling(self.handle, *[_ptr(a) for a in arrays]))
        return arrays

    def _inputs(self, x) -> np.ndarray:
        x = np.ascontiguousarray(np.atleast_2d(x), np.float32)
        if x.ndim != 2 or x.shape[1] != self.inputs:
            raise ValueError(f"inputs must be (rows x {self.inputs}); got shape {x.shape}")
        return x

    def _samples(self, x, y):
        """(x, y) as contiguous float32 rows whose widths match the network (the library reads rows x width)."""
        x = self._inputs(x)
        y = np.ascontiguousarray(np.atleast_2d(y), np.float32)
        if y.shape != (x.shape[0], self.outputs):
            raise ValueError(f"targets must be ({x.shape[0]} x {self.outputs}); got shape {y.shape}")
        return x, y

    def gradients(self, x, y):
        """Loss and parameter gradient of the unscaled network on (x, y)."""
        x, y = self._samples(x, y)
        grads = np.zeros(self.parameter_count, np.float32)
        loss = ctypes.c_float()
        check(lib().qmbed_gpu_mlp_gradients(self.handle, _ptr(x), _ptr(y), x.shape[0], _ptr(grads),
                                            ctypes.byref(loss)))
        return loss.value, grads

    def train(self, x, y, epochs: int = 400, batch: int = 32, learning_rate: float = 2e-3, seed: int = 0) -> float:
        x, y = self._samples(x, y)
        loss = ctypes.c_float()
        check(lib().qmbed_gpu_mlp_train(self.handle, _ptr(x), _ptr(y), x.shape[0], epochs, batch, learning_rate,
                                        seed, ctypes.byref(loss)))
        return loss.value

    def predict(self, x) -> np.ndarray:
        x = self._inputs(x)
        y = np.zeros((x.shape[0], self.outputs), np.float32)
        check(lib().qmbed_gpu_mlp_predict(self.handle, _ptr(x), x.shape[0], _ptr(y)))
        return y


def tfim_instance(sites: int, g: float, width: float, seed: int) -> np.ndarray:
    """Longitudinal fields h_i ~ U[-W, W] of one disorder instance."""
    return np.random.default_rng(seed).uniform(-width, width, sites)


def tfim_features(sites: int, g: float, width: float, fields) -> np.ndarray:
    """Network inputs: 1/L (per-site extremes move like 1/L with open ends), g, W,
    moments of the fields, the mean single-site energy sqrt(h^2 + g^2), and the
    mean half difference and half sum of neighbouring fields (what aligned and
    anti-aligned neighbour pairs gain from the fields)."""
    h = np.asarray(fields, float)
    site = np.sqrt(h * h + g * g)
    step = np.abs(np.diff(h)).mean() / 2 if sites > 1 else 0.0
    pair = np.abs(h[:-1] + h[1:]).mean() / 2 if sites > 1 else 0.0
    return np.array([1.0 / sites, g, width, h.mean(), h.std(), np.abs(h).mean(), site.mean(), step, pair],
                    np.float32)


def tfim_operator(sites: int, g: float, fields, j: float = 1.0, periodic: bool = False, device: int = 0):
    """Ising chain J zz + g x + h z in Pauli normalisation, with the flip-chain action."""
    return GpuOperator(GpuBasis(sites, normalization="pauli", device=device),
                       tfim_terms(sites, j=j, g=g, fields=fields, periodic=periodic), storage="matrix_free")


def lanczos_extremes(op: GpuOperator, steps: int, seed: int = 0):
    out = np.zeros(4)
    check(lib().qmbed_gpu_lanczos_extremes(op.handle, steps, seed, _ptr(out)))
    return out  # theta_min, theta_max, residual at theta_min, residual at theta_max


def generate_tfim_bounds(count: int, sizes=(6, 8, 10, 12), seed: int = 0, g_range=(0.5, 1.5),
                         width_range=(0.5, 3.0), steps: int = 200, tolerance: float = 1e-8):
    """Training set from the GPU solver: features and spectral extremes per site.

    Each instance draws g, W and the fields from `seed`; E_min and E_max are
    the extreme Ritz values of one FP64 Lanczos run on the GPU, accepted when
    the residuals of both Ritz pairs are below tolerance * max(|E|, 1)
    (otherwise the run is repeated with twice the steps)."""
    rng = np.random.default_rng(seed)
    xs, ys = [], []
    for index in range(count):
        sites = int(sizes[index % len(sizes)])
        g = rng.uniform(*g_range)
        width = rng.uniform(*width_range)
        fields = tfim_instance(sites, g, width, int(rng.integers(1 << 31)))
        op = tfim_operator(sites, g, fields)
        run = steps
        while True:
            lo, hi, r_lo, r_hi = lanczos_extremes(op, min(run, op.dim), seed=index)
            if (r_lo <= tolerance * max(abs(lo), 1.0) and r_hi <= tolerance * max(abs(hi), 1.0)) or run >= op.dim:
                break
            run *= 2
        xs.append(tfim_features(sites, g, width, fields))
        ys.append([lo / sites, hi / sites])
    return np.array(xs, np.float32), np.array(ys, np.float32)


@dataclass
class Interval:
    e_min: float
    e_max: float
    source: str            # "learned" or "lanczos"
    applications: int      # H applications spent to obtain it


class LearnedBounds:
    """Spectral intervals from the network, checked by a short Lanczos run."""

    def __init__(self, mlp: GpuMlp | None = None, margin: float = 0.03, check_steps: int = 8):
        self.mlp = mlp or GpuMlp(len(FEATURES), len(TARGETS))
        self.margin = margin
        self.check_steps = check_steps

    def fit(self, x, y, epochs: int = 400, batch: int = 32, learning_rate: float = 2e-3, seed: int = 0) -> float:
        return self.mlp.train(x, y, epochs=epochs, batch=batch, learning_rate=learning_rate, seed=seed)

    def predict(self, sites: int, g: float, width: float, fields):
        per_site = self.mlp.predict(tfim_features(sites, g, width, fields))[0]
        return float(per_site[0]) * sites, float(per_site[1]) * sites

    def interval(self, op: GpuOperator, sites: int, g: float, width: float, fields, seed: int = 0) -> Interval:
        lo, hi = self.predict(sites, g, width, fields)
        pad = self.margin * (hi - lo)
        lo, hi = lo - pad, hi + pad
        ritz = lanczos_extremes(op, self.check_steps, seed)
        if np.isfinite(lo) and np.isfinite(hi) and hi > lo and lo <= ritz[0] and hi >= ritz[1]:
            return Interval(lo, hi, "learned", self.check_steps)
        fallback = lanczos_interval(op, seed=seed)
        return Interval(fallback.e_min, fallback.e_max, "lanczos", fallback.applications + self.check_steps)


def lanczos_interval(op: GpuOperator, steps: int = 40, seed: int = 0, margin: float = 0.01) -> Interval:
    """Plain Lanczos bound estimate: Ritz extremes widened by their residuals and a margin."""
    ritz = lanczos_extremes(op, steps, seed)
    lo, hi = ritz[0] - ritz[2], ritz[1] + ritz[3]
    pad = margin * (hi - lo)
    return Interval(lo - pad, hi + pad, "lanczos", steps)


def propagate_device(op: GpuOperator, state, times, interval: Interval, precision: int = 64,
                     tolerance: float = 1e-10, drift_limit: float | None = None) -> dict:
    """propagate() in place on a device complex128 tensor (no host copies of the state)."""
    import torch
    if drift_limit is None:
        drift_limit = 1e-8 if precision == 64 else 1e-4
    initial = state.clone()
    info = op.chebyshev_evolve_device(state, times, interval.e_min, interval.e_max, tolerance=tolerance,
                                      precision=precision)
    info["source"] = interval.source
    norm0 = max(1.0, float(torch.linalg.vector_norm(initial)))
    if info["max_norm_drift"] > drift_limit * norm0:
        state.copy_(initial)
        info = op.chebyshev_evolve_device(state, times, tolerance=tolerance, precision=precision)
        info["source"] = "norm bound (after drift)"
    return info


def propagate(op: GpuOperator, psi0, times, interval: Interval, precision: int = 64, tolerance: float = 1e-10,
              final_only: bool = False, drift_limit: float | None = None):
    """Chebyshev propagation on `interval`; repeats on the guaranteed bound if the norm drifts.

    A spectrum that leaves the interval makes the norm grow exponentially with
    the expansion degree, far beyond rounding: the default limit is 1e-8 of the
    norm with complex128 vectors and 1e-4 with complex64 (whose rounding over a
    long trajectory reaches 1e-6)."""
    if drift_limit is None:
        drift_limit = 1e-8 if precision == 64 else 1e-4
    states, info = op.chebyshev_evolve(psi0, times, interval.e_min, interval.e_max, tolerance=tolerance,
                                       precision=precision, final_only=final_only)
    info["source"] = interval.source
    info["bound_applications"] = interval.applications
    if info["max_norm_drift"] > drift_limit * max(1.0, float(np.linalg.norm(psi0))):
        states, info = op.chebyshev_evolve(psi0, times, tolerance=tolerance, precision=precision,
                                           final_only=final_only)
        info["source"] = "norm bound (after drift)"
        info["bound_applications"] = interval.applications
    return states, info


# ---------------------------------------------------------------------------
# Chain spectra for the eigsh hint
# ---------------------------------------------------------------------------

CHAIN_FEATURES = ("inverse_sites", "j2", "delta", "cos_momentum", "momentum_zero", "sites_mod_4")
CHAIN_TARGETS = ("e0_per_site", "e_max_per_site", "gap_times_sites")


def chain_features(sites: int, j2: float, delta: float, momentum: int) -> np.ndarray:
    """Network inputs of a momentum sector of H = Delta (zz1 + J2 zz2) + flips1 + J2 flips2
    at half filling: 1/L, J2, Delta, cos(2 pi k / L), [k = 0] and [L = 0 mod 4] (the
    sector holding the ground state alternates with L mod 4 by the Marshall sign rule)."""
    return np.array([1.0 / sites, j2, delta, np.cos(2.0 * np.pi * momentum / sites), 1.0 if momentum == 0 else 0.0,
                     1.0 if sites % 4 == 0 else 0.0], np.float32)


def scan_training_set(sizes=(12, 14, 16, 18, 20), points: int = 16, seed: int = 0, j2_max: float = 0.5,
                      delta_range=(0.5, 1.5), device: int = 0, tolerance: float = 1e-10):
    """Training set from the batched scan solver: for every size, every momentum
    sector at half filling times `points` scan points (J2 on a grid, Delta drawn),
    the scan's lowest two eigenvalues and largest Ritz value give the targets
    (E0 / L, E_max / L, (E1 - E0) L). Returns (x, y, info)."""
    from . import scan
    xs, ys = [], []
    solves = 0
    for sites in sizes:
        components = scan.j1j2_sectors(sites, device=device)
        coef = scan.j1j2_scan_points(points, seed=seed + sites, j2_max=j2_max, delta_range=delta_range)
        values, steps, info = scan.scan_lowest(components, coef, eigenpairs=2, tolerance=tolerance, seed=seed)
        e_max = info["e_max"]
        for k in range(sites):
            for p in range(points):
                delta, j2 = float(coef[p, 0]), float(coef[p, 3])
                e0, e1 = float(values[k, p, 0]), float(values[k, p, 1])
                xs.append(chain_features(sites, j2, delta, k))
                ys.append([e0 / sites, float(e_max[k, p]) / sites, (e1 - e0) * sites])
        solves += sites * points
        del components
    return np.array(xs, np.float32), np.array(ys, np.float32), {"solves": solves, "sizes": list(sizes)}


class ChainSpectrum:
    """Lowest and largest eigenvalue and the gap of chain sectors from a GPU network."""

    def __init__(self, mlp: GpuMlp | None = None, margin: float = 0.03, check_steps: int = 8, device: int = 0):
        self.mlp = mlp or GpuMlp(len(CHAIN_FEATURES), len(CHAIN_TARGETS), device=device)
        self.margin = margin
        self.check_steps = check_steps

    def fit(self, x, y, epochs: int = 400, batch: int = 64, learning_rate: float = 2e-3, seed: int = 0) -> float:
        return self.mlp.train(x, y, epochs=epochs, batch=batch, learning_rate=learning_rate, seed=seed)

    def predict(self, sites: int, j2: float, delta: float, momentum: int):
        """(E0, E_max, gap) of the momentum sector (half filling)."""
        e0, emax, gap = self.mlp.predict(chain_features(sites, j2, delta, momentum))[0]
        return float(e0) * sites, float(emax) * sites, max(float(gap), 0.0) / sites

    def hint(self, sites: int, j2: float, delta: float, momentum: int, eigenpairs: int,
             krylov_dimension: int = 40) -> dict:
        """eigsh hint for a sector of these couplings (a parity subsector of momentum
        sector k has its spectrum inside sector k's, so the interval still holds it).

        Interval: [E0, E_max] padded by `margin` of its width on both sides.
        Restart size: with a small predicted relative gap (E1 - E0) / (E_max - E0),
        where the thick restart converges slowly, it keeps two Ritz vectors beyond
        the wanted ones (measured at 28 sites, 6 wanted, Krylov 40: 466 -> 173
        steps; keeping more cost time), otherwise the reference's size.

        A prediction that is not finite, or whose E_max is not above E0, gives
        the empty hint (lower = upper = 0, no restart change, "usable" False):
        the solver then takes its own Lanczos bounds and the reference's
        restart size instead of failing on the prediction."""
        e0, emax, gap = self.predict(sites, j2, delta, momentum)
        if not (np.isfinite(e0) and np.isfinite(emax) and np.isfinite(gap)) or not emax > e0:
            return {"lower": 0.0, "upper": 0.0, "gap": 0.0, "restart_keep": 0, "check_steps": self.check_steps,
                    "relative_gap": None, "e0": e0 if np.isfinite(e0) else None,
                    "e_max": emax if np.isfinite(emax) else None, "usable": False}
        width = max(emax - e0, 1e-12)
        relative_gap = gap / width
        keep = min(krylov_dimension // 2, eigenpairs + 2) if relative_gap < 0.05 else 0
        return {"lower": e0 - self.margin * width, "upper": emax + self.margin * width, "gap": gap,
                "restart_keep": keep, "check_steps": self.check_steps, "relative_gap": relative_gap,
                "e0": e0, "e_max": emax, "usable": True}

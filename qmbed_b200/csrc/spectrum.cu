// Broadened spectral functions on the GPU.
//
// Reference behaviour (matrixlab-research/QMBED):
//   SpectrumOptions / validate          src/dynamics/mod.rs:903-962
//   spectral_function                   src/dynamics/mod.rs:964-1021
//   lanczos_spectral_measure            src/solve/mod.rs:2886-2907
//   hermitian_eigenpairs_all            src/solve/mod.rs:558-583
// The probe's action (a sector shift or an operator) and the Lanczos
// projection run on the device; the Lorentzian sums over at most a few
// hundred poles run on the host in FP64.
#include <cmath>

#include "evolve.cuh"
#include "spectrum.cuh"

namespace qmbed {

void validate_spectrum(const SpectrumOptions& o) {
  bool ok = !o.frequencies.empty() && std::isfinite(o.reference_energy) && std::isfinite(o.broadening) &&
            o.broadening > 0.0 && o.krylov_dimension > 0 && std::isfinite(o.tolerance) && o.tolerance > 0.0;
  for (double f : o.frequencies) ok = ok && std::isfinite(f);
  if (!ok) raise(QMBED_INVALID_OPTIONS, "invalid spectrum frequency grid or numerical controls");
}

std::vector<double> spectral_function(const LinearOperatorView& view, const double* created,
                                      const SpectrumOptions& o, BlockOps& ops) {
  validate_spectrum(o);
  const uint64_t n = view.dim;
  std::vector<double> energies, weights;
  if (n <= 128) {
    // hermitian_eigenpairs_all: dense matrix (columns H e_c from the device
    // action, whatever the storage), Hermiticity at 1e-12, every eigenpair
    std::vector<C64> dense(static_cast<size_t>(n * n), C64(0.0, 0.0));
    {
      DeviceBuffer x(n * 16), y(n * 16);
      std::vector<C64> column(static_cast<size_t>(n));
      const C64 one(1.0, 0.0);
      for (uint64_t c = 0; c < n; ++c) {
        QMBED_CUDA(cudaMemsetAsync(x.get(), 0, n * 16, ops.stream()));
        QMBED_CUDA(cudaMemcpyAsync(static_cast<char*>(x.get()) + c * 16, &one, 16, cudaMemcpyHostToDevice, ops.stream()));
        view.apply(64, true, x.get(), y.get());
        QMBED_CUDA(cudaMemcpyAsync(column.data(), y.get(), n * 16, cudaMemcpyDeviceToHost, ops.stream()));
        ops.sync();
        for (uint64_t r = 0; r < n; ++r) dense[r * n + c] = column[r];
      }
    }
    for (uint64_t r = 0; r < n; ++r)
      for (uint64_t c = 0; c < n; ++c)
        if (std::abs(dense[r * n + c] - std::conj(dense[c * n + r])) > 1.0e-12) raise(QMBED_NON_HERMITIAN, "");
    std::vector<C64> vectors;
    device_hermitian_eigen(static_cast<int>(n), dense, energies, vectors, ops.stream());
    std::vector<C64> v(static_cast<size_t>(n));
    QMBED_CUDA(cudaMemcpyAsync(v.data(), created, n * 16, cudaMemcpyDeviceToHost, ops.stream()));
    ops.sync();
    for (uint64_t e = 0; e < n; ++e) {
      C64 overlap(0.0, 0.0);
      for (uint64_t i = 0; i < n; ++i) overlap += std::conj(vectors[i + n * e]) * v[i];
      weights.push_back(std::norm(overlap));
    }
  } else {
    std::vector<C64> host(static_cast<size_t>(n));
    QMBED_CUDA(cudaMemcpyAsync(host.data(), created, n * 16, cudaMemcpyDeviceToHost, ops.stream()));
    ops.sync();
    bool real = true;
    for (const C64& x : host) real = real && x.imag() == 0.0;
    lanczos_spectral_measure(view, created, real, o.krylov_dimension, energies, weights, ops);
  }
  std::vector<double> out;
  out.reserve(o.frequencies.size());
  const double pi = 3.14159265358979323846;
  for (double frequency : o.frequencies) {
    double sum = 0.0;
    for (size_t e = 0; e < energies.size(); ++e) {
      const double detuning = frequency + o.reference_energy - energies[e];
      sum += weights[e] * o.broadening / (pi * (detuning * detuning + o.broadening * o.broadening));
    }
    out.push_back(sum);
  }
  return out;
}

}  // namespace qmbed

// Broadened spectral functions of a probed state in the same or another
// sector (the response step after eigsh).
#pragma once

#include <vector>

#include "eigsh.cuh"
#include "krylov.cuh"

namespace qmbed {

// SpectrumOptions (src/dynamics/mod.rs:903-962): frequency grid, reference
// energy, Lorentzian broadening, Krylov dimension (default 64) and the
// continued-fraction tolerance (validated; default 1e-10).
struct SpectrumOptions {
  std::vector<double> frequencies;
  double reference_energy = 0.0;
  double broadening = 0.0;
  size_t krylov_dimension = 64;
  double tolerance = 1.0e-10;
};

void validate_spectrum(const SpectrumOptions& o);

// spectral_function (src/dynamics/mod.rs:964-1021) of `created` = probe |source>
// (device, interleaved complex FP64, target dimension): every eigenpair of
// the target Hamiltonian when it has at most 128 states, else the Lanczos
// spectral measure; sum_e w_e eta / (pi ((omega + E_ref - E_e)^2 + eta^2)).
std::vector<double> spectral_function(const LinearOperatorView& target, const double* created,
                                      const SpectrumOptions& o, BlockOps& ops);

}  // namespace qmbed

"""Runtime-symmetry spin bases and site conventions (test infrastructure only).

Only the tests and the fixture scripts under ``tests/golden/`` import this
module. It restates, in pure Python for small chains, how the reference builds
a spin basis from explicit lattice maps -- the form its QuSpin-compatible
frontend sends -- and how a model applies a frontend site permutation:

* ``LatticeSymmetryMap::mapped_state`` (src/basis/mod.rs:3100-3130): the digit
  at source site ``i`` moves to ``destinations[i]`` after the local
  permutation of site ``i``; distinguishable statistics carry phase 1.
* ``trace_symmetry_orbit`` (src/basis/mod.rs:3455-3538): breadth-first orbit
  from a seed; each generator step multiplies the coefficient by
  ``exp(-2 pi i sector / period)``; a state reached twice with different
  coefficients marks the orbit incompatible.
* ``GeneralBasis::from_reducer_impl`` with orbit seeds
  (src/basis/mod.rs:4163-4306): representative = minimum (or maximum) orbit
  state, gauge by the representative's coefficient, phase = coefficient /
  gauge, orbit size = number of orbit states, representatives ordered by the
  parent's row (colex = numeric for a fixed-weight spin basis).
* ``ordered_basis`` / ``representative_ordering``
  (bindings/capi/src/lib.rs:3412-3423) and ``build_spin_basis`` (2849-2905):
  ``reverse`` selects maximum representatives for general maps and reverses
  the public row order.
* ``OperatorSpec::with_site_permutation`` (src/operator/mod.rs:264-300):
  coupling site ``s`` becomes ``permutation[s]``.

The reduced operator follows the reference's transition rule
(``GeneralBasis::reduce_transition``, src/basis/mod.rs:4466-4479): column ``j``
takes the parent operator's column at the representative ``r_j`` (assembled by
the C++ oracle) and adds each parent target ``t`` of a compatible orbit at the
row of its representative with the factor ``sqrt(R_j / R_t) conj(phase(t))``.
"""

from __future__ import annotations

import cmath
import math
from collections import deque
from itertools import combinations

import numpy as np

from . import oracle as _oracle


def map_state(state: int, destinations, local_permutations=None) -> int:
    """``LatticeSymmetryMap::mapped_state`` for spin one half (base 2)."""
    out = 0
    for source, dest in enumerate(destinations):
        digit = (state >> source) & 1
        if local_permutations is not None:
            digit = local_permutations[source][digit]
        out |= digit << dest
    return out


def permutation_period(destinations, local_permutations=None) -> int:
    """Smallest n > 0 with map^n = identity on every site and digit."""
    sites = len(destinations)
    n = 1
    while True:
        ok = True
        for site in range(sites):
            s, digits = site, [0, 1]
            for _ in range(n):
                if local_permutations is not None:
                    digits = [local_permutations[s][d] for d in digits]
                s = destinations[s]
            if s != site or digits != [0, 1]:
                ok = False
                break
        if ok:
            return n
        n += 1


class GeneralSpinBasis:
    """A spin-1/2 chain basis reduced by explicit lattice maps.

    ``symmetries`` is a list of dicts with ``destinations``, ``sector`` and
    optional ``local_permutations`` -- the reference's ``SymmetryRequest``
    (bindings/capi/src/lib.rs:600-611).
    """

    def __init__(self, sites: int, up: int | None = None, symmetries=(), reverse: bool = False):
        self.sites = sites
        self.up = up
        if up is None:
            parent = list(range(1 << sites))
        else:
            parent = sorted(sum(1 << b for b in bits) for bits in combinations(range(sites), up))
        self.parent = parent
        gens = []
        for sym in symmetries:
            dest = list(sym["destinations"])
            local = sym.get("local_permutations")
            period = permutation_period(dest, local)
            sector = int(sym["sector"]) % period
            step = cmath.exp(-2j * math.pi * sector / period)
            gens.append((dest, local, step))
        self.images = {}
        reps = []
        if not gens:
            reps = [(s, 1) for s in parent]
            self.images = {s: (s, 1.0 + 0j, 1) for s in parent}
        else:
            visited = set()
            for seed in parent:
                if seed in visited:
                    continue
                coeff = {seed: 1.0 + 0j}
                queue = deque([seed])
                compatible = True
                while queue:
                    src = queue.popleft()
                    for dest, local, step in gens:
                        tgt = map_state(src, dest, local)
                        c = coeff[src] * step
                        if tgt in coeff:
                            if abs(coeff[tgt] - c) > 1e-10:
                                compatible = False
                        else:
                            coeff[tgt] = c
                            queue.append(tgt)
                visited.update(coeff)
                if not compatible:
                    continue
                rep = max(coeff) if reverse else min(coeff)
                gauge = coeff[rep] / abs(coeff[rep])
                size = len(coeff)
                for s, c in coeff.items():
                    self.images[s] = (rep, c / gauge, size)
                reps.append((rep, size))
            reps.sort()
        if reverse:
            reps.reverse()
        self.states = np.array([r for r, _ in reps], dtype=np.uint64)
        self.orbits = np.array([n for _, n in reps], dtype=np.int64)
        self.index = {int(r): i for i, (r, _) in enumerate(reps)}

    def __len__(self) -> int:
        return len(self.states)

    def vectors(self) -> np.ndarray:
        """Columns: the normalised orbit vectors in the parent space (rows in ``parent`` order)."""
        row = {s: i for i, s in enumerate(self.parent)}
        out = np.zeros((len(self.parent), len(self)), dtype=complex)
        for s, (rep, phase, size) in self.images.items():
            if s not in row:
                raise NotImplementedError("an orbit leaves the parent magnetisation sector")
            out[row[s], self.index[rep]] = phase / math.sqrt(size)
        return out


def permute_terms(terms, permutation):
    """``OperatorSpec::with_site_permutation``: site s becomes permutation[s]."""
    if permutation is None:
        return terms
    return [(symbols, [(c, tuple(permutation[s] for s in sites)) for c, sites in couplings])
            for symbols, couplings in terms]


def reduced_dense(basis: GeneralSpinBasis, terms, normalization: str = "angular_momentum",
                  site_permutation=None) -> np.ndarray:
    """Dense reduced operator by the reference's transition rule, from the oracle's parent operator."""
    parent = _oracle.Basis(basis.sites, up=basis.up, normalization=normalization)
    h = _oracle.Operator.build(parent, permute_terms(terms, site_permutation),
                               check_hermitian=False, check_particles=False).dense()
    row = {s: i for i, s in enumerate(basis.parent)}
    out = np.zeros((len(basis), len(basis)), dtype=complex)
    for j, rep in enumerate(basis.states):
        column = h[:, row[int(rep)]]
        r_j = basis.orbits[j]
        for t in np.flatnonzero(column):
            image = basis.images.get(basis.parent[t])
            if image is None:
                continue
            rep_t, phase, r_t = image
            out[basis.index[rep_t], j] += column[t] * math.sqrt(r_j / r_t) * phase.conjugate()
    return out

"""The spectral-bound network on the GPU: gradients against the CPU oracle,
training, and what the learned bounds gain over plain Lanczos bounds.

Gradients of the GPU kernels must match the numpy oracle (oracle/mlp_oracle.py,
itself pinned by finite differences) to 1e-4 relative (FP32 kernels against an
FP64 oracle). The learned interval is only used after a short Lanczos check;
states propagated on it must match the oracle within 1e-9 while costing fewer
operator applications than the plain Lanczos bound route.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def learned():
    import qmbed_b200.learned as module
    return module


def test_mlp_gradients_match_oracle(learned):
    from oracle import mlp_oracle
    net = learned.GpuMlp(6, 2, width=128, hidden_layers=4, seed=1)
    dims = mlp_oracle.layer_dims(6, 2, 128, 4)
    params = net.parameters().astype(np.float64)
    assert params.size == sum(a * b + b for a, b in zip(dims[:-1], dims[1:]))
    rng = np.random.default_rng(2)
    x = rng.standard_normal((37, 6)).astype(np.float32)
    y = rng.standard_normal((37, 2)).astype(np.float32)
    loss, grads = net.gradients(x, y)
    ref_loss, ref = mlp_oracle.loss_and_gradients(params, dims, x.astype(np.float64), y.astype(np.float64))
    assert abs(loss - ref_loss) <= 1e-5 * abs(ref_loss)
    assert np.linalg.norm(grads - ref) <= 1e-4 * np.linalg.norm(ref)
    # the forward pass of the trained-units network
    out = net.predict(x)
    assert np.allclose(out, mlp_oracle.forward(params, dims, x.astype(np.float64))[-1], rtol=1e-4, atol=1e-5)


def test_mlp_training_fits_and_is_reproducible(learned):
    from oracle import mlp_oracle
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, (256, 3)).astype(np.float32)
    y = np.stack([np.sin(2 * x[:, 0]) + x[:, 1] ** 2, x[:, 2] * x[:, 0]], axis=1).astype(np.float32)
    a = learned.GpuMlp(3, 2, width=64, hidden_layers=4, seed=5)
    b = learned.GpuMlp(3, 2, width=64, hidden_layers=4, seed=5)
    loss = a.train(x, y, epochs=300, batch=32, learning_rate=3e-3, seed=9)
    b.train(x, y, epochs=300, batch=32, learning_rate=3e-3, seed=9)
    assert loss < 1e-2
    assert np.array_equal(a.parameters(), b.parameters())  # fixed-order sums: bitwise reproducible
    in_mean, in_std, out_mean, out_std = a.scaling()
    dims = mlp_oracle.layer_dims(3, 2, 64, 4)
    net_out = mlp_oracle.forward(a.parameters().astype(np.float64), dims, (x - in_mean) / in_std)[-1]
    assert np.allclose(a.predict(x), net_out * out_std + out_mean, rtol=1e-4, atol=1e-4)
    assert np.mean((a.predict(x) - y) ** 2) < 2e-2 * np.var(y)


def test_lanczos_extremes_lie_inside_the_spectrum(learned):
    fields = learned.tfim_instance(12, 1.0, 2.0, 4)
    op = learned.tfim_operator(12, 1.0, fields)
    lo = op.eigsh(1, target="smallest_algebraic", tolerance=1e-10).eigenvalues[0]
    hi = op.eigsh(1, target="largest_algebraic", tolerance=1e-10).eigenvalues[0]
    for steps in (4, 8, 40):
        t_min, t_max, r_min, r_max = learned.lanczos_extremes(op, steps)
        assert lo - 1e-9 <= t_min <= t_max <= hi + 1e-9
    assert abs(t_min - lo) < 1e-3 * abs(lo) and abs(t_max - hi) < 1e-3 * abs(hi)
    # the training labels: a 200-step run resolves both extremes to the eigensolver's accuracy
    t_min, t_max, r_min, r_max = learned.lanczos_extremes(op, 200)
    assert abs(t_min - lo) <= 1e-8 * abs(lo) and abs(t_max - hi) <= 1e-8 * abs(hi)
    assert r_min <= 1e-8 * abs(lo) and r_max <= 1e-8 * abs(hi)


def test_learned_bounds_gain_over_lanczos_bounds(learned, oracle):
    x, y = learned.generate_tfim_bounds(240, sizes=(6, 8, 10, 12), seed=11)
    bounds = learned.LearnedBounds()
    loss = bounds.fit(x, y, epochs=400, seed=1)
    assert loss < 0.05

    # held-out chains, larger than any in the training set
    rng = np.random.default_rng(12)
    errors, used_learned = [], 0
    for k in range(6):
        sites, g, width = 14, rng.uniform(0.5, 1.5), rng.uniform(0.5, 3.0)
        fields = learned.tfim_instance(sites, g, width, 100 + k)
        op = learned.tfim_operator(sites, g, fields)
        lo = op.eigsh(1, target="smallest_algebraic", tolerance=1e-10).eigenvalues[0]
        hi = op.eigsh(1, target="largest_algebraic", tolerance=1e-10).eigenvalues[0]
        plo, phi = bounds.predict(sites, g, width, fields)
        errors.append(max(abs(plo - lo), abs(phi - hi)) / sites)
        used_learned += bounds.interval(op, sites, g, width, fields).source == "learned"
    assert np.mean(errors) < 0.15  # per site, extrapolated from chains of at most 12 sites
    assert used_learned >= 3
    # one quench step at 16 sites: same state, fewer operator applications
    sites, g, width = 16, 1.0, 2.0
    fields = learned.tfim_instance(sites, g, width, 7)
    op = learned.tfim_operator(sites, g, fields)
    o = oracle.Operator.build(oracle.Basis(sites, normalization="pauli"),
                              learned.tfim_terms(sites, j=1.0, g=g, fields=fields))
    psi0 = np.zeros(op.dim, complex)
    psi0[-1] = 1.0
    times = [0.2]
    ref, _ = o.evolve(psi0, times, krylov_dimension=40, tolerance=1e-12)
    interval = bounds.interval(op, sites, g, width, fields)
    assert interval.source == "learned"
    fast, fast_info = learned.propagate(op, psi0, times, interval)
    slow_interval = learned.lanczos_interval(op)
    slow, slow_info = learned.propagate(op, psi0, times, slow_interval)
    assert np.linalg.norm(fast[0] - ref[0]) <= 1e-9 and np.linalg.norm(slow[0] - ref[0]) <= 1e-9
    fast_cost = fast_info["applications"] + fast_info["bound_applications"]
    slow_cost = slow_info["applications"] + slow_info["bound_applications"]
    assert fast_cost < slow_cost, (fast_cost, slow_cost)

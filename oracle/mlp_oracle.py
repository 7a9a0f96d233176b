"""CPU oracle for the spectral-bound network (TEST INFRASTRUCTURE ONLY).

A plain numpy restatement, in FP64, of the fully connected ReLU network that
the library trains on the GPU: forward pass, mean-squared-error loss and its
gradient by backpropagation, with the library's parameter layout (per linear
map: W as in x out row-major, then b). Only the tests load it; the library
never calls it. The network has no counterpart in the reference, so this
oracle is pinned by finite differences (tests/test_mlp_oracle.py).
"""

import numpy as np


def layer_dims(inputs, outputs, width, hidden_layers):
    return [inputs] + [width] * hidden_layers + [outputs]


def unpack(params, dims):
    """Split the flat parameter vector into [(W, b), ...]."""
    out, off = [], 0
    for din, dout in zip(dims[:-1], dims[1:]):
        w = params[off:off + din * dout].reshape(din, dout)
        off += din * dout
        b = params[off:off + dout]
        off += dout
        out.append((w, b))
    assert off == len(params)
    return out


def forward(params, dims, x):
    acts = [np.asarray(x, np.float64)]
    layers = unpack(np.asarray(params, np.float64), dims)
    for i, (w, b) in enumerate(layers):
        z = acts[-1] @ w + b
        acts.append(np.maximum(z, 0.0) if i + 1 < len(layers) else z)
    return acts


def loss_and_gradients(params, dims, x, y):
    """Mean squared error over samples x outputs and its parameter gradient."""
    acts = forward(params, dims, x)
    layers = unpack(np.asarray(params, np.float64), dims)
    y = np.asarray(y, np.float64)
    diff = acts[-1] - y
    loss = float(np.mean(diff * diff))
    delta = 2.0 * diff / diff.size
    grads = [None] * len(layers)
    for i in range(len(layers) - 1, -1, -1):
        w, _ = layers[i]
        grads[i] = (acts[i].T @ delta, delta.sum(axis=0))
        if i > 0:
            delta = (delta @ w.T) * (acts[i] > 0.0)
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat

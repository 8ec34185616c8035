"""FP64 numpy reference of the plan model's network (same parameter layout as
the library: per layer W (out x in, row-major) then b (out); ReLU hidden
layers, linear output; loss = mean squared error). Test infrastructure: the
checker for the GPU forward/backward kernels."""
import numpy as np


def unpack(params, widths):
    params = np.asarray(params, dtype=np.float64)
    out, off = [], 0
    for l in range(len(widths) - 1):
        i, o = widths[l], widths[l + 1]
        W = params[off:off + o * i].reshape(o, i)
        off += o * i
        b = params[off:off + o]
        off += o
        out.append((W, b))
    assert off == params.size
    return out


def forward(params, widths, X):
    layers = unpack(params, widths)
    A = np.asarray(X, dtype=np.float64)
    acts, pres = [A], [None]
    for l, (W, b) in enumerate(layers):
        Z = A @ W.T + b
        A = np.maximum(Z, 0.0) if l + 1 < len(layers) else Z
        pres.append(Z)
        acts.append(A)
    return acts[-1][:, 0], acts, pres


def loss_and_grad(params, widths, X, T):
    layers = unpack(params, widths)
    y, acts, pres = forward(params, widths, X)
    T = np.asarray(T, dtype=np.float64)
    B = len(T)
    loss = np.mean((y - T) ** 2)
    d = (2.0 * (y - T) / B)[:, None]
    grads = []
    for l in range(len(layers) - 1, -1, -1):
        if l + 1 < len(layers):
            d = d * (pres[l + 1] > 0)
        W, _ = layers[l]
        grads.append((d.T @ acts[l], d.sum(axis=0)))
        d = d @ W
    g = []
    for dW, db in reversed(grads):
        g.append(dW.ravel())
        g.append(db)
    return loss, np.concatenate(g)

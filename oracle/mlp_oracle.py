"""CPU oracle of the learned-preconditioner network (TEST INFRASTRUCTURE ONLY).

A numpy restatement of hp-multiphysics_b200/csrc/hp_mlp.cu: affine layers with
ReLU between them, inputs standardised, parameters and hidden activations
rounded to BF16 (round to nearest even), masked MSE loss 0.5/n sum mask (y-t)^2,
backward pass with the straight-through rule for the roundings. Used by the
tests to check the GPU kernels' gradients.
"""
import numpy as np


def bf16(x):
    """Round float values to BF16 (nearest even), returned as float64."""
    a = np.asarray(x, dtype=np.float32).copy()
    u = a.view(np.uint32)
    lsb = (u >> 16) & 1
    u += 0x7FFF + lsb
    u &= 0xFFFF0000
    return a.astype(np.float64)


def unpack(params, widths):
    out, off = [], 0
    for l in range(len(widths) - 1):
        ni, no = widths[l], widths[l + 1]
        W = params[off:off + ni * no].reshape(no, ni)
        off += ni * no
        b = params[off:off + no]
        off += no
        out.append((W, b))
    return out


def forward(params, widths, mean, std, X, round_bf16=True):
    r = bf16 if round_bf16 else (lambda z: np.asarray(z, np.float64))
    p = r(params)
    layers = unpack(p, widths)
    istd = np.where(std > 0, 1.0 / np.asarray(std, np.float32), 1.0).astype(np.float32)
    a = r(((np.asarray(X, np.float32) - np.asarray(mean, np.float32)) * istd))
    acts = [a]
    for l, (W, b) in enumerate(layers):
        z = a @ W.T + b
        if l < len(layers) - 1:
            a = r(np.maximum(z, 0.0))
        else:
            a = z
        acts.append(a)
    return acts


def grad(params, widths, mean, std, X, T, mask, round_bf16=True):
    """Gradient of 0.5/n sum_s sum_o mask_o (y - t)^2 (straight-through)."""
    acts = forward(params, widths, mean, std, X, round_bf16)
    r = bf16 if round_bf16 else (lambda z: np.asarray(z, np.float64))
    layers = unpack(r(params), widths)
    n = X.shape[0]
    e = acts[-1] - T
    loss = 0.5 * np.sum(mask * e * e) / n
    delta = mask * e / n
    g = []
    for l in range(len(layers) - 1, -1, -1):
        W, b = layers[l]
        gW = delta.T @ acts[l]
        gb = delta.sum(axis=0)
        g.append((gW, gb))
        if l > 0:
            delta = (delta @ W) * (acts[l] > 0)
    g.reverse()
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in g])
    return flat, loss

"""FP64 numpy restatement of libytf's node-placement MLP (ytf_mlp_*): forward pass, loss and
gradient. Test infrastructure only: the checker of the GPU training kernels' gradients.

Same parameter layout (per layer W [out x in] row-major, then b [out]), GELU
0.5 z (1 + erf(z/√2)) between layers, products with the weights rounded to BF16
(round-to-nearest-even, as __float2bfloat16_rn), biases FP32, loss
mean_b (o0 - t0)^2 + mean_b [softplus(o1) - t1 o1]. The gradient is the one the kernels
form: dW = dZ^T H and dH = dZ · bf16(W) (the rounding passes the gradient straight through).
"""
import numpy as np
from scipy.special import erf


def bf16_round(x):
    """FP32 values rounded to BF16 (nearest even), returned as float64."""
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(params, sizes):
    p = np.asarray(params, np.float64)
    out, o = [], 0
    for l in range(1, len(sizes)):
        n_in, n_out = sizes[l - 1], sizes[l]
        W = p[o:o + n_out * n_in].reshape(n_out, n_in)
        o += n_out * n_in
        b = p[o:o + n_out]
        o += n_out
        out.append((W, b))
    return out


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(params, sizes, X, round_weights=True):
    layers = unpack(params, sizes)
    H = [np.asarray(X, np.float64)]
    Z = [None]
    for l, (W, b) in enumerate(layers, start=1):
        Wq = bf16_round(W) if round_weights else W
        z = H[-1] @ Wq.T + b
        Z.append(z)
        H.append(gelu(z) if l < len(layers) else z)
    return Z, H


def loss_and_grad(params, sizes, X, T, round_weights=True):
    T = np.asarray(T, np.float64)
    Z, H = forward(params, sizes, X, round_weights)
    out = H[-1]
    B = out.shape[0]
    e = out[:, 0] - T[:, 0]
    o1 = out[:, 1]
    sp = np.where(o1 > 0, o1 + np.log1p(np.exp(-np.abs(o1))), np.log1p(np.exp(o1)))
    loss = float(np.mean(e * e + sp - T[:, 1] * o1))
    dZ = np.stack([2 * e / B, (1 / (1 + np.exp(-o1)) - T[:, 1]) / B], axis=1)
    layers = unpack(params, sizes)
    grads = [None] * len(layers)
    for l in range(len(layers), 0, -1):
        W, _ = layers[l - 1]
        Wq = bf16_round(W) if round_weights else W
        if l < len(layers):
            dZ = dZ * gelu_grad(Z[l])
        grads[l - 1] = (dZ.T @ H[l - 1], dZ.sum(axis=0))
        dZ = dZ @ Wq
    g = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, g

"""TEST INFRASTRUCTURE ONLY — FP64 numpy oracle of the degree selector's MLP.

Mirrors the parameter layout and arithmetic of the library's BF16 MLP kernels
(16 -> 64 -> 64 -> 9, ReLU) in FP64 on the BF16-rounded weights, with the
masked mean-squared-error loss L = sum mask (y - t)^2 / (9 n), its gradient
by backpropagation, and one Adam step (beta 0.9 / 0.999, eps 1e-8).
"""
import numpy as np

F, H, O = 16, 64, 9
SHAPES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (O, H)), ("b3", (O,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16_round(x):
    """Round FP32 values to BF16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def unpack(p):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def pack(d):
    return np.concatenate([d[name].ravel() for name, _ in SHAPES])


def forward(p, x):
    w = unpack(p)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = np.maximum(z2, 0)
    y = h2 @ w["W3"].T + w["b3"]
    return y, (x, z1, h1, z2, h2)


def forward_bf16_activations(p, x):
    """forward() with the inputs and both hidden activations rounded to BF16
    (round to nearest even) before each layer, as the tensor-core inference
    kernel feeds its BF16 operands; products and sums in FP64."""
    w = unpack(p)
    xb = bf16_round(x)
    h1 = bf16_round(np.maximum(xb @ w["W1"].T + w["b1"], 0))
    h2 = bf16_round(np.maximum(h1 @ w["W2"].T + w["b2"], 0))
    return h2 @ w["W3"].T + w["b3"]


def loss_and_grad(p, x, t, mask):
    n = len(x)
    y, (x, z1, h1, z2, h2) = forward(p, x)
    w = unpack(p)
    e = y - t
    loss = float(np.sum(mask * e * e) / (O * n))
    d3 = 2 * mask * e / (O * n)
    d2 = (d3 @ w["W3"]) * (z2 > 0)
    d1 = (d2 @ w["W2"]) * (z1 > 0)
    g = {"W3": d3.T @ h2, "b3": d3.sum(0), "W2": d2.T @ h1, "b2": d2.sum(0), "W1": d1.T @ x, "b1": d1.sum(0)}
    return loss, pack(g)


def adam(master, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    upd = lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return master - upd, m, v

"""CPU oracle of the MLP surrogate (forward pass and MSE gradients).

TEST INFRASTRUCTURE ONLY: used by tests/ to check the tensor-core kernels
of alsvinn_b200/csrc/mlp_*.  The reference has no learned component; this
file restates the network's mathematics in NumPy FP64:

    H_0 = x,  Z_l = H_{l-1} W_l^T + b_l,  H_l = gelu(Z_l)  (l = 1..hidden),
    y = H_hidden w + b,  loss = (1/B) sum_r (y_r - t_r)^2,
    gelu(z) = z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))  (tanh form),

with back-propagation written out by hand.  ``bf16=True`` rounds at the
same points as the GPU path (inputs, hidden weight matrices, activations
H_l and back-propagated dZ_l to BF16; the 1-wide head stays FP32), so the
remaining differences are the GPU's FP32 accumulation order.  The flat
parameter layout is the one of include/als_surrogate.h: per layer the
weight matrix (out x in, row-major) then the bias.
"""
import numpy as np


def bf16(a):
    """Round to BF16 (nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


K_GELU = 0.79788456080286536   # sqrt(2/pi)
A_GELU = 0.044715


def gelu(z):
    """GELU, tanh form (Hendrycks and Gimpel 2016)."""
    return 0.5 * z * (1.0 + np.tanh(K_GELU * (z + A_GELU * z ** 3)))


def gelu_grad(z):
    t = np.tanh(K_GELU * (z + A_GELU * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * K_GELU * (1.0 + 3.0 * A_GELU * z * z)


def layer_shapes(inputs, width, hidden):
    shapes = []
    for l in range(hidden + 1):
        shapes.append((1 if l == hidden else width, inputs if l == 0 else width))
    return shapes


def unpack(params, inputs, width, hidden):
    """Flat vector -> [(W, b)] per layer (float64 copies)."""
    p = np.asarray(params, dtype=np.float64)
    out = []
    off = 0
    for o, i in layer_shapes(inputs, width, hidden):
        W = p[off:off + o * i].reshape(o, i)
        off += o * i
        b = p[off:off + o]
        off += o
        out.append((W, b))
    if off != p.size:
        raise ValueError("parameter vector has %d entries, the network %d" % (p.size, off))
    return out


def param_count(inputs, width, hidden):
    return sum(o * i + o for o, i in layer_shapes(inputs, width, hidden))


def forward(params, x, inputs, width, hidden, bf16_path=True):
    """Returns (y, cache) for rows of x."""
    layers = unpack(params, inputs, width, hidden)
    rnd = bf16 if bf16_path else (lambda a: np.asarray(a, dtype=np.float64))
    h = rnd(x)
    cache = {"h": [h], "z": [], "w": []}
    for l in range(hidden):
        W, b = layers[l]
        Wr = rnd(W)
        z = h @ Wr.T + b
        if bf16_path:
            z = z.astype(np.float32).astype(np.float64)
        h = rnd(gelu(z))
        cache["z"].append(z)
        cache["h"].append(h)
        cache["w"].append(Wr)
    w, b = layers[hidden]
    y = h @ w[0] + b[0]
    return y, cache


def gradients(params, x, t, inputs, width, hidden, bf16_path=True):
    """Flat gradient of the mean squared error and the loss."""
    layers = unpack(params, inputs, width, hidden)
    rnd = bf16 if bf16_path else (lambda a: np.asarray(a, dtype=np.float64))
    y, c = forward(params, x, inputs, width, hidden, bf16_path)
    B = y.shape[0]
    r = y - np.asarray(t, dtype=np.float64)
    loss = float(np.mean(r * r))
    dy = 2.0 * r / B
    grads = [None] * (hidden + 1)
    w_head = layers[hidden][0][0]
    h_last = c["h"][hidden]
    grads[hidden] = (dy @ h_last, np.array([dy.sum()]))
    dz = rnd(np.outer(dy, w_head) * gelu_grad(c["z"][hidden - 1]))
    for l in range(hidden - 1, -1, -1):
        h_in = c["h"][l]
        gW = dz.T @ h_in
        gb = dz.sum(axis=0)
        grads[l] = (gW, gb)
        if l > 0:
            dz = rnd((dz @ c["w"][l]) * gelu_grad(c["z"][l - 1]))
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return flat, loss

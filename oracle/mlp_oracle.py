"""ORACLE -- test infrastructure only.  FP64 numpy restatement of the learned
preconditioner's network (dmrgpp_b200/csrc/mlp.cu): the same feature map,
parameter layout [W1 (256x4), b1, W2 (256x256), b2, w3 (256), b3], forward
pass and mean-squared-error gradients, used to check the GPU kernels'
gradients.  The network has no counterpart in the reference."""
import numpy as np

F, H = 4, 256
DELTA = 0.05
SIZES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("w3", (H,)), ("b3", (1,))]


def unpack(flat):
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def num_params():
    return sum(int(np.prod(s)) for _, s in SIZES)


def features(d, r, theta, rnorm):
    s = max(1.0, abs(theta))
    rms = rnorm / np.sqrt(max(len(d), 1))
    f0 = (d - theta) / s
    f1 = r / rms if rms > 0 else np.zeros_like(r)
    x = np.stack([f0, f1, f1 * f0 / (f0 * f0 + DELTA ** 2), 1.0 / (1.0 + (f0 / DELTA) ** 2)],
                 axis=1)
    return x


def to_bf16(a):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(flat, x, bf16_hidden=False):
    """Network output; bf16_hidden rounds the first hidden layer to BF16
    before the second layer (the operand format of the tensor-core
    inference, mlp.cu)."""
    p = unpack(flat)
    h1 = np.tanh(x @ p["W1"].T + p["b1"])
    if bf16_hidden:
        h1 = to_bf16(h1)
    h2 = np.tanh(h1 @ p["W2"].T + p["b2"])
    o = h2 @ p["w3"] + p["b3"][0]
    return o, (h1, h2)


def loss_and_grads(flat, x, y, w=None):
    p = unpack(flat)
    rows = len(x)
    o, (h1, h2) = forward(flat, x)
    w = np.ones(rows) if w is None else w
    d = o - y
    loss = float(np.sum(w * d * d) / rows)
    g = 2.0 * w * d / rows
    grads = {"w3": h2.T @ g, "b3": np.array([g.sum()])}
    dz2 = np.outer(g, p["w3"]) * (1 - h2 * h2)
    grads["W2"] = dz2.T @ h1
    grads["b2"] = dz2.sum(0)
    dz1 = (dz2 @ p["W2"]) * (1 - h1 * h1)
    grads["W1"] = dz1.T @ x
    grads["b1"] = dz1.sum(0)
    flat_g = np.concatenate([grads[name].ravel() for name, _ in SIZES])
    return loss, flat_g

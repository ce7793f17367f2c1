"""numpy reference of the surrogate MLP (7 -> 64 -> 64 -> 4, SiLU), forward
and backward, with the same bf16 rounding points as the tensor-core kernels:
inputs, hidden activations and weights are rounded to bf16 (round to nearest
even), products accumulate in f32 / f64.

TEST INFRASTRUCTURE ONLY: the checker for adaptive-gimp_b200/csrc/mlp.cu.
"""
import numpy as np

IN, H, OUT = 7, 64, 4
SIZES = [("W1", (IN, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, OUT)), ("b3", (OUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(P):
    out, o = {}, 0
    for k, s in SIZES:
        n = int(np.prod(s))
        out[k] = np.asarray(P[o:o + n]).reshape(s)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[k], np.float32).ravel() for k, _ in SIZES]).astype(np.float32)


def bf16(a):
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(P, X, emulate_bf16=True):
    """Returns (y, cache).  f64 arithmetic on (optionally) bf16-rounded values."""
    p = unpack(np.asarray(P, np.float32))
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float32))
    x = r(X).astype(np.float64)
    W1, W2, W3 = (r(p[k]).astype(np.float64) for k in ("W1", "W2", "W3"))
    z1 = x @ W1 + p["b1"]
    a1 = r(silu(z1)).astype(np.float64)
    z2 = a1 @ W2 + p["b2"]
    a2 = r(silu(z2)).astype(np.float64)
    y = a2 @ W3 + p["b3"]
    return y, dict(x=x, z1=z1, a1=a1, z2=z2, a2=a2, W1=W1, W2=W2, W3=W3)


def loss_and_grad(P, X, T, emulate_bf16=True):
    """Mean squared error over the batch (sum over outputs, mean over samples)
    and its gradient with respect to the f32 parameters.  With emulate_bf16 the
    backward pass rounds dy, dz2 and dz1 to bf16 where the kernels feed them to
    the tensor cores (the bias gradients are column sums of the rounded values,
    as the kernels obtain them from a row of ones in the transposed operands)."""
    y, c = forward(P, X, emulate_bf16)
    n = len(X)
    r = bf16 if emulate_bf16 else (lambda a: np.asarray(a, np.float32))
    dy = 2.0 * (y - T) / n
    dyr = r(dy).astype(np.float64)
    g = {}
    g["W3"] = c["a2"].T @ dyr
    g["b3"] = dyr.sum(0)
    da2 = dyr @ c["W3"].T
    dz2 = r(da2 * dsilu(c["z2"])).astype(np.float64)
    g["W2"] = c["a1"].T @ dz2
    g["b2"] = dz2.sum(0)
    da1 = dz2 @ c["W2"].T
    dz1 = r(da1 * dsilu(c["z1"])).astype(np.float64)
    g["W1"] = c["x"].T @ dz1
    g["b1"] = dz1.sum(0)
    loss = float(((y - T) ** 2).sum() / n)
    return loss, pack(g)


def init_params(rng, scale=1.0):
    d = {}
    for k, s in SIZES:
        if k.startswith("W"):
            d[k] = rng.normal(0, scale * np.sqrt(1.0 / s[0]), s)
        else:
            d[k] = rng.normal(0, 0.1 * scale, s)
    return pack(d)

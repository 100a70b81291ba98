"""CPU oracle of the surrogate MLP's forward and backward passes.

TEST INFRASTRUCTURE ONLY: the checker for the tcgen05 training kernels.
NumPy float64 arithmetic with BF16 rounding applied where the GPU stores BF16
(weights of layers 2-4, activations h, pre-activations z, gradients dO and
dZ), so the GPU's gradients must agree to BF16 precision.  Parameter layout
as cl_mlp: W1[256][3] b1 W2t[256][256] b2 W3t b3 W4t[192][256] b4.
"""
import numpy as np

D_IN, D_H, D_OUT = 3, 256, 192
SHAPES = [("W1", (D_H, D_IN)), ("b1", (D_H,)), ("W2", (D_H, D_H)), ("b2", (D_H,)),
          ("W3", (D_H, D_H)), ("b3", (D_H,)), ("W4", (D_OUT, D_H)), ("b4", (D_OUT,))]


def split(p):
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = p[o:o + n].reshape(shp)
        o += n
    return out


def bf16(x):
    """Round to bfloat16 (round to nearest even) and back, as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x):
    P = split(p)
    x = np.asarray(x, np.float64)
    z1 = x @ P["W1"].T.astype(np.float64) + P["b1"]
    h1 = bf16(silu(z1)); z1b = bf16(z1)
    z2 = h1 @ bf16(P["W2"]).T + P["b2"]
    h2 = bf16(silu(z2)); z2b = bf16(z2)
    z3 = h2 @ bf16(P["W3"]).T + P["b3"]
    h3 = bf16(silu(z3)); z3b = bf16(z3)
    o = h3 @ bf16(P["W4"]).T + P["b4"]
    return o, dict(x=x, h1=h1, z1=z1b, h2=h2, z2=z2b, h3=h3, z3=z3b)


def gradient(p, x, t):
    """Loss mean((o - t)^2) over all B*192 outputs and its gradient."""
    P = split(p)
    o, c = forward(p, x)
    B = o.shape[0]
    scale = 1.0 / (B * D_OUT)
    d = o - np.asarray(t, np.float64)
    loss = float((d * d).sum() * scale)
    dO = bf16(2.0 * d * scale)
    dz3 = bf16((dO @ bf16(P["W4"])) * dsilu(c["z3"]))
    dz2 = bf16((dz3 @ bf16(P["W3"])) * dsilu(c["z2"]))
    dz1 = bf16((dz2 @ bf16(P["W2"])) * dsilu(c["z1"]))
    g = {"W4": dO.T @ c["h3"], "b4": dO.sum(0), "W3": dz3.T @ c["h2"], "b3": dz3.sum(0),
         "W2": dz2.T @ c["h1"], "b2": dz2.sum(0), "W1": dz1.T @ c["x"], "b1": dz1.sum(0)}
    flat = np.concatenate([g[name].reshape(-1) for name, _ in SHAPES])
    return loss, flat

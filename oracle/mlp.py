"""CPU oracle of the learned-microphysics MLP — TEST INFRASTRUCTURE ONLY.

A float64 numpy restatement of the network the library trains on the
tensor cores (16 -> 256 -> 256 -> 256 -> 9, SiLU), with BF16 rounding
applied at the same points as the device path: inputs, weights, hidden
activations and the back-propagated gradients that enter a GEMM are
rounded to BF16 (round to nearest even); accumulations, biases, the loss
and the bias gradients stay in high precision.  Used by the tests to check
the device forward pass and the hand-written backward pass (gradient
check), never by the product.

Parameter layout (as cress_mlp_get_params): W1 [256][64], b1 [256],
W2 [256][256], b2, W3 [256][256], b3 (stored [out][in]), W4 [256][64]
([in][out]), b4 [64]; inputs padded to 64, outputs to 64.
"""
import numpy as np

H, K1, N4, NIN, NOUT = 256, 64, 64, 16, 9
SIZES = [("W1", H * K1), ("b1", H), ("W2", H * H), ("b2", H), ("W3", H * H), ("b3", H),
         ("W4", H * N4), ("b4", N4)]


def count():
    return sum(n for _, n in SIZES)


def unpack(p):
    out, o = {}, 0
    for name, n in SIZES:
        out[name] = np.asarray(p[o:o + n], np.float64)
        o += n
    out["W1"] = out["W1"].reshape(H, K1)
    out["W2"] = out["W2"].reshape(H, H)
    out["W3"] = out["W3"].reshape(H, H)
    out["W4"] = out["W4"].reshape(H, N4)
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SIZES])


ROUND = True   # False: exact float64 network (for finite-difference checks)


def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    if not ROUND:
        return np.asarray(a, np.float64)
    x = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((x + 0x7FFF + ((x >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x):
    """x [n][16] standardized -> (y [n][9], cache)."""
    w = unpack(p)
    n = x.shape[0]
    xp = np.zeros((n, K1))
    xp[:, :NIN] = x
    a = bf16(xp)
    cache = {"a0": a}
    for l, (wn, bn) in enumerate((("W1", "b1"), ("W2", "b2"), ("W3", "b3")), start=1):
        z = a @ bf16(w[wn]).T + w[bn]
        cache[f"z{l}"] = z
        a = bf16(silu(z))
        cache[f"a{l}"] = a
    y = a @ bf16(w["W4"]) + w["b4"]
    return y[:, :NOUT], cache


def loss_grad(p, x, t):
    """Mean-square loss over the batch and the 9 outputs and its gradient
    (same layout as the parameters), following the device's rounding."""
    w = unpack(p)
    n = x.shape[0]
    y, c = forward(p, x)
    d = y - t
    loss = float(np.mean(d * d))
    dy = np.zeros((n, N4))
    dy[:, :NOUT] = 2.0 * d / (NOUT * n)
    dyb = bf16(dy)
    g = {}
    g["W4"] = c["a3"].T @ dyb
    g["b4"] = dy.sum(0)
    dh = dyb @ bf16(w["W4"]).T
    for l, wn in ((3, "W3"), (2, "W2"), (1, "W1")):
        dz = dh * dsilu(c[f"z{l}"])
        dzb = bf16(dz)
        g[wn] = dzb.T @ c[f"a{l - 1}"]
        g[f"b{l}"] = dz.sum(0)
        if l > 1:
            dh = dzb @ bf16(w[wn])
    return loss, pack(g)

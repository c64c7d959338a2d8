"""CPU restatement (numpy) of the learned Newton initial guess: the network's
forward pass and the gradient of its mean squared error, with the BF16
roundings of the device kernels at the same places (inputs of every
tensor-core product rounded to BF16, FP32 accumulation and activations).

Test infrastructure only: the oracle for the device kernels of
dynela-v.-4.0_b200/csrc/mlp.cu and csrc/dnl_mlp.cuh.  The network has no
counterpart in the reference (DynELA's return starts from the previous
increment's gamma, Sources/dnlElements/Element.C:507-515); its inputs are
the trial state of that return (Element.C:440-470).
"""
import numpy as np

KIN, H, NIN = 16, 64, 5


def bf16(a):
    """Round float32 values to the nearest BF16 value (ties to even), as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    nan = np.isnan(a)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    out = u.astype(np.uint32).view(np.float32).copy()
    out[nan] = np.nan
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def normalise(net, x, dt=np.float32):
    xin = np.zeros((x.shape[0], KIN), dtype=dt)
    xin[:, :NIN] = (x.astype(dt) - np.asarray(net["in_mean"], dt)) * np.asarray(net["in_scale"], dt)
    clip = float(net.get("in_clip", 0.0))
    if clip > 0.0:  # inputs past the training range held at its edge (dnl_mlp.in_clip)
        xin[:, :NIN] = np.clip(xin[:, :NIN], -clip, clip)
    return xin


def forward(net, x, rounding=True):
    """Outputs and the cached intermediates of the forward pass.
    rounding=False: the same function in FP64 without roundings (for the
    finite-difference check of the backward pass)."""
    r = bf16 if rounding else (lambda a: a)
    dt = np.float32 if rounding else np.float64
    xin = r(normalise(net, x, dt))
    W1, W2, W3 = (r(np.asarray(net[k], dtype=dt)) for k in ("w1", "w2", "w3"))
    b1, b2, b3, w4 = (np.asarray(net[k], dtype=dt) for k in ("b1", "b2", "b3", "w4"))
    z1 = xin @ W1.T + b1
    h1 = r(silu(z1).astype(dt))
    z2 = h1 @ W2.T + b2
    h2 = r(silu(z2).astype(dt))
    z3 = h2 @ W3.T + b3
    y = silu(z3) @ w4 + dt(net["b4"])
    return y, dict(xin=xin, z1=z1, h1=h1, z2=z2, h2=h2, z3=z3, W2=W2, W3=W3, w4=w4)


def gradients(net, x, t, rounding=True):
    """Gradient of (1/n) sum (y - t)^2 with respect to every weight and bias,
    and the loss, in the order of the device backward pass."""
    r = bf16 if rounding else (lambda a: a)
    dt = np.float32 if rounding else np.float64
    y, c = forward(net, x, rounding)
    n = x.shape[0]
    dy = (2.0 / n) * (y - t.astype(dt))
    g = {}
    g["w4"] = silu(c["z3"]).T @ dy
    g["b4"] = dy.sum()
    dz3 = dy[:, None] * c["w4"][None, :] * silu_grad(c["z3"])
    dh2 = r(dz3.astype(dt)) @ c["W3"]
    dz2 = dh2 * silu_grad(c["z2"])
    dh1 = r(dz2.astype(dt)) @ c["W2"]
    dz1 = dh1 * silu_grad(c["z1"])
    g["w3"] = dz3.T @ c["h2"]
    g["b3"] = dz3.sum(0)
    g["w2"] = dz2.T @ c["h1"]
    g["b2"] = dz2.sum(0)
    w1 = dz1.T @ c["xin"]
    w1[:, NIN:] = 0.0
    g["w1"] = w1
    g["b1"] = dz1.sum(0)
    loss = float(np.mean((y - t) ** 2))
    return g, loss


def random_net(seed, scale=1.0):
    """A seeded network with He-like initial weights (and identity input normalisation)."""
    rng = np.random.default_rng(seed)
    w1 = np.zeros((H, KIN), np.float32)
    w1[:, :NIN] = rng.normal(0, scale * np.sqrt(2.0 / NIN), (H, NIN))
    return dict(w1=w1, b1=rng.normal(0, 0.1 * scale, H).astype(np.float32),
                w2=rng.normal(0, scale * np.sqrt(2.0 / H), (H, H)).astype(np.float32),
                b2=rng.normal(0, 0.1 * scale, H).astype(np.float32),
                w3=rng.normal(0, scale * np.sqrt(2.0 / H), (H, H)).astype(np.float32),
                b3=rng.normal(0, 0.1 * scale, H).astype(np.float32),
                w4=rng.normal(0, scale * np.sqrt(1.0 / H), H).astype(np.float32),
                b4=np.float32(0.1), in_mean=np.zeros(NIN, np.float32), in_scale=np.ones(NIN, np.float32))

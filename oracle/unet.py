"""CPU oracle of the brick-local learned preconditioner (test infrastructure only).

The reference has no learned preconditioner; this file DEFINES the network that
paracfd_b200/csrc/learned.cu implements, in plain numpy, so that the GPU forward pass, the
backward pass and the optimiser step can be checked against it:

* one 8^3 brick is one sample; the network never looks outside its brick (zero padding at the
  brick boundary in every 3x3x3 convolution);
* levels 8^3 (16 channels), 4^3 (32), 2^3 (64); 2x2x2 average pooling down, nearest-neighbour
  upsampling up, skip connections by channel concatenation (a concatenated convolution is the
  sum of one convolution per source);
* no biases, ReLU after every convolution, a 1x1x1 head (16 -> 1);
* inputs: channel 0 = D^-1 r / s, channel 1 = active mask, channels 2..15 = 0, where s is the
  RMS of D^-1 r over the brick's active cells; output z = s * head(...) * mask;
* BF16 rounding (round to nearest even) of every tensor the GPU stores in BF16: the network
  input, every post-ReLU activation, the pooled / upsampled staging copies, the weights, and the
  pre-activation gradients fed to the transposed convolutions and weight gradients.

Voxel order inside a brick is (z*n + y)*n + x, channels innermost: arrays are [B, n, n, n, C]
indexed [b, z, y, x, c].  Taps are t = (dz+1)*9 + (dy+1)*3 + (dx+1); weights are [27, Cout, Cin].
"""
from __future__ import annotations

import numpy as np

LAYERS = (  # name, level n, Cout, Cin (per source, concatenation order)
    ("enc0", 8, 16, (16,)),
    ("enc1", 4, 32, (16,)),
    ("bott", 2, 64, (32,)),
    ("dec1", 4, 32, (64, 32)),
    ("dec0", 8, 16, (32, 16)),
)
HEAD = 16
TAPS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def param_shapes():
    """Parameter tensors in the flat order the library uses (weights then the head)."""
    shapes = []
    for name, _n, cout, cins in LAYERS:
        for k, cin in enumerate(cins):
            shapes.append((f"{name}.{k}", (27, cout, cin)))
    shapes.append(("head", (HEAD,)))
    return shapes


def param_count():
    return int(sum(np.prod(s) for _, s in param_shapes()))


def unflatten(flat):
    out, o = {}, 0
    for name, shape in param_shapes():
        size = int(np.prod(shape))
        out[name] = np.asarray(flat[o:o + size], np.float64).reshape(shape)
        o += size
    return out


def flatten(params):
    return np.concatenate([np.asarray(params[name], np.float64).ravel() for name, _ in param_shapes()])


def init_params(seed):
    """He-normal weights (fan-in 27*Cin) from numpy's PCG64, the head N(0, 1/16)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p = {}
    for name, shape in param_shapes():
        fan_in = shape[0] * shape[2] if len(shape) == 3 else shape[0]
        p[name] = rng.standard_normal(shape) * np.sqrt(2.0 / fan_in)
    return p


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(np.isnan(f), np.nan, out)


def conv(x, w):
    """Zero-padded 3x3x3 convolution per brick: y[b,v,co] = sum_t sum_ci w[t,co,ci] x[b,v+shift_t,ci]."""
    B, n = x.shape[0], x.shape[1]
    xp = np.zeros((B, n + 2, n + 2, n + 2, x.shape[4]))
    xp[:, 1:-1, 1:-1, 1:-1] = x
    y = np.zeros((B, n, n, n, w.shape[1]))
    for t, (dz, dy, dx) in enumerate(TAPS):
        y += xp[:, 1 + dz:1 + dz + n, 1 + dy:1 + dy + n, 1 + dx:1 + dx + n] @ w[t].T
    return y


def conv_weight_grad(g, x):
    """dW[t,co,ci] = sum_b sum_v g[b,v,co] x[b,v+shift_t,ci] (the adjoint of conv in w)."""
    B, n = x.shape[0], x.shape[1]
    xp = np.zeros((B, n + 2, n + 2, n + 2, x.shape[4]))
    xp[:, 1:-1, 1:-1, 1:-1] = x
    gw = np.zeros((27, g.shape[4], x.shape[4]))
    gf = g.reshape(-1, g.shape[4])
    for t, (dz, dy, dx) in enumerate(TAPS):
        gw[t] = gf.T @ xp[:, 1 + dz:1 + dz + n, 1 + dy:1 + dy + n, 1 + dx:1 + dx + n].reshape(-1, x.shape[4])
    return gw


def conv_transpose(g, w):
    """The adjoint of conv in x: the convolution with flipped taps and transposed channels."""
    wt = np.transpose(w[::-1], (0, 2, 1))
    return conv(g, wt)


def pool(x):
    B, n, C = x.shape[0], x.shape[1], x.shape[4]
    return x.reshape(B, n // 2, 2, n // 2, 2, n // 2, 2, C).mean(axis=(2, 4, 6))


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)


def sum_children(x):
    B, n, C = x.shape[0], x.shape[1], x.shape[4]
    return x.reshape(B, n // 2, 2, n // 2, 2, n // 2, 2, C).sum(axis=(2, 4, 6))


def prepare(r, dinv, mask):
    """Network input and brick scale from one brick's residual: r, dinv, mask are [B, 512]."""
    q = r * dinv * mask
    active = np.maximum(mask.sum(1), 1.0)
    s = np.sqrt((q * q).sum(1) / active)
    s = np.where(s > 0, s, 1.0)
    x = np.zeros((r.shape[0], 8, 8, 8, 16))
    x[..., 0] = (q / s[:, None]).reshape(-1, 8, 8, 8)
    x[..., 1] = mask.reshape(-1, 8, 8, 8)
    return bf16(x), s


def forward(params, x, rounding=True):
    """All activations of the network on input x [B,8,8,8,16]; returns (zhat [B,512], acts)."""
    R = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    W = {k: R(v) for k, v in params.items()}
    a = {"x": R(x)}
    a["e0"] = R(np.maximum(conv(a["x"], W["enc0.0"]), 0))
    a["p0"] = R(pool(a["e0"]))
    a["e1"] = R(np.maximum(conv(a["p0"], W["enc1.0"]), 0))
    a["p1"] = R(pool(a["e1"]))
    a["b"] = R(np.maximum(conv(a["p1"], W["bott.0"]), 0))
    a["ub"] = up(a["b"])
    a["d1"] = R(np.maximum(conv(a["ub"], W["dec1.0"]) + conv(a["e1"], W["dec1.1"]), 0))
    a["ud1"] = up(a["d1"])
    a["d0"] = R(np.maximum(conv(a["ud1"], W["dec0.0"]) + conv(a["e0"], W["dec0.1"]), 0))
    zhat = a["d0"].reshape(x.shape[0], 512, HEAD) @ W["head"]
    return zhat, a


def loss_and_grads(params, x, target, mask, rounding=True):
    """Masked mean-square loss  sum m (zhat - t)^2 / sum m  and its parameter gradients."""
    R = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    W = {k: R(v) for k, v in params.items()}
    zhat, a = forward(params, x, rounding)
    count = max(float(mask.sum()), 1.0)
    diff = (zhat - target) * mask
    loss = float((diff * diff).sum() / count)
    dz = 2.0 * diff / count                                            # [B,512]
    g = {}
    B = x.shape[0]
    d0 = a["d0"].reshape(B, 512, HEAD)
    g["head"] = np.einsum("bvc,bv->c", d0, dz)
    G4 = R((dz[..., None] * W["head"][None, None, :]) * (d0 > 0)).reshape(B, 8, 8, 8, HEAD)
    g["dec0.0"] = conv_weight_grad(G4, a["ud1"])
    g["dec0.1"] = conv_weight_grad(G4, a["e0"])
    dd1 = sum_children(conv_transpose(G4, W["dec0.0"]))
    de0 = conv_transpose(G4, W["dec0.1"])
    G3 = R(dd1 * (a["d1"] > 0))
    g["dec1.0"] = conv_weight_grad(G3, a["ub"])
    g["dec1.1"] = conv_weight_grad(G3, a["e1"])
    db = sum_children(conv_transpose(G3, W["dec1.0"]))
    de1 = conv_transpose(G3, W["dec1.1"])
    G2 = R(db * (a["b"] > 0))
    g["bott.0"] = conv_weight_grad(G2, a["p1"])
    de1 = de1 + up(conv_transpose(G2, W["bott.0"])) / 8.0
    G1 = R(de1 * (a["e1"] > 0))
    g["enc1.0"] = conv_weight_grad(G1, a["p0"])
    de0 = de0 + up(conv_transpose(G1, W["enc1.0"])) / 8.0
    G0 = R(de0 * (a["e0"] > 0))
    g["enc0.0"] = conv_weight_grad(G0, a["x"])
    return loss, g


def adam_step(params, grads, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update (bias-corrected) of every parameter tensor, in place; step counts from 1."""
    for k in params:
        m[k] = beta1 * m[k] + (1 - beta1) * grads[k]
        v[k] = beta2 * v[k] + (1 - beta2) * grads[k] ** 2
        mh = m[k] / (1 - beta1 ** step)
        vh = v[k] / (1 - beta2 ** step)
        params[k] = params[k] - lr * mh / (np.sqrt(vh) + eps)

"""CPU restatement of the learned initial-guess network: forward, loss and
backward of the 3-D convolutional network, with BF16 rounding at the same
points as the CUDA kernels.

Test infrastructure only: imported by tests/ for the expected values of the
tensor-core kernels (values and gradients), never by the product.

The network (no reference code exists for it; it is defined by the project):
  input  15 channels: the conserved variables Q = U*J of Q^n, Q^(n-1),
         Q^(n-2), each variable normalised as (Q_v - mean_v) / std_v,
         channel = level * 5 + v (level 0 = Q^n);
  layers 3x3x3 convolutions 15 -> 32 -> 32 -> 32 -> 32 -> 5, GELU (erf form)
         after the first four; periodic padding in x and z, zero padding in y
         (the walls);
  output 5 channels: the correction to second-order extrapolation,
         (Q^(n+1) - (3 Q^n - 3 Q^(n-1) + Q^(n-2)))_v / oscale_v.
Weights are kept in float32 (Adam state too) and rounded to BF16 for every
forward and backward product; activations, pre-activations and gradients
flowing between layers are stored in BF16; every sum is accumulated in
float32 (here float64, so the GPU's float32 accumulation is within the
tests' tolerance of this).

Arrays here are (C, nx, ny, nz) float64 holding BF16-representable values
where the GPU holds BF16.  Weights: W[l] of shape (27, cout, cin), tap index
t = (dx * 3 + dy) * 3 + dz with offsets (dx - 1, dy - 1, dz - 1); b[l] (cout,).
"""
from __future__ import annotations

import math

import numpy as np

CIN = (15, 32, 32, 32, 32)
COUT = (32, 32, 32, 32, 5)
NLAYER = 5


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def param_count() -> int:
    return sum(27 * ci * co + co for ci, co in zip(CIN, COUT))


def unpack(theta: np.ndarray):
    """Flat float32 parameter vector -> ([W_l], [b_l]) in the order
    W_0, b_0, W_1, b_1, ... (W_l row-major (27, cout, cin))."""
    W, b, o = [], [], 0
    for ci, co in zip(CIN, COUT):
        n = 27 * co * ci
        W.append(np.asarray(theta[o:o + n], np.float64).reshape(27, co, ci))
        o += n
        b.append(np.asarray(theta[o:o + co], np.float64))
        o += co
    return W, b


def pack(W, b) -> np.ndarray:
    return np.concatenate([np.concatenate([w.ravel(), bb.ravel()]) for w, bb in zip(W, b)]).astype(np.float32)


def init_params(seed: int = 0) -> np.ndarray:
    """He-style uniform initialisation; the last layer starts at zero so the
    untrained network returns plain extrapolation."""
    rng = np.random.default_rng(seed)
    W, b = [], []
    for l, (ci, co) in enumerate(zip(CIN, COUT)):
        lim = math.sqrt(6.0 / (27 * ci)) if l < NLAYER - 1 else 0.0
        W.append(rng.uniform(-lim, lim, size=(27, co, ci)))
        b.append(np.zeros(co))
    return pack(W, b)


def _shift(x, dx, dy, dz):
    """x[c, i+dx, j+dy, k+dz] with periodic i, k and zero outside j."""
    y = np.roll(x, (-dx, -dz), axis=(1, 3))
    if dy == 0:
        return y
    out = np.zeros_like(y)
    if dy > 0:
        out[:, :, :-dy] = y[:, :, dy:]
    else:
        out[:, :, -dy:] = y[:, :, :dy]
    return out


def conv(x, W, bias=None):
    """Correlation out[co] = sum_t W[t, co, :] . x(shifted by tap t) (+ bias)."""
    co = W.shape[1]
    out = np.zeros((co,) + x.shape[1:])
    t = 0
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                xs = _shift(x, dx, dy, dz)
                out += np.einsum("oc,cijk->oijk", W[t], xs)
                t += 1
    if bias is not None:
        out += bias[:, None, None, None]
    return out


def conv_transpose(g, W):
    """Gradient with respect to the input of conv: sum_t W[t]^T g(shifted by -tap)."""
    ci = W.shape[2]
    out = np.zeros((ci,) + g.shape[1:])
    t = 0
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                out += np.einsum("oc,oijk->cijk", W[t], _shift(g, -dx, -dy, -dz))
                t += 1
    return out


def conv_wgrad(x, g):
    """dW[t, co, ci] = sum_cells g[co] * x[ci](shifted by tap t)."""
    dW = np.zeros((27, g.shape[0], x.shape[0]))
    t = 0
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                dW[t] = np.einsum("oijk,cijk->oc", g, _shift(x, dx, dy, dz))
                t += 1
    return dW


def gelu(z):
    from scipy.special import erf
    return 0.5 * z * (1.0 + erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    from scipy.special import erf
    return 0.5 * (1.0 + erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def _identity(a):
    return np.asarray(a, np.float64)


def forward(theta, x0, keep=False, exact=False):
    """x0: (15, nx, ny, nz) input.  Returns the output (5, ...) and, with
    keep=True, the activations and pre-activations the backward pass needs.
    exact=True skips every BF16 rounding (for finite-difference checks)."""
    r = _identity if exact else bf16
    W, b = unpack(theta)
    a = [r(x0)]
    zs = []
    for l in range(NLAYER):
        z = conv(a[-1], r(W[l]), b[l])
        if l < NLAYER - 1:
            zb = r(z)
            zs.append(zb)
            a.append(r(gelu(zb)))
        else:
            out = z
    return (out, a, zs) if keep else out


def loss_and_grad(theta, x0, target, exact=False):
    """Mean squared error over cells and the 5 outputs, and its gradient
    with respect to theta (flat, float64)."""
    r = _identity if exact else bf16
    W, b = unpack(theta)
    out, a, zs = forward(theta, x0, keep=True, exact=exact)
    n = out.size
    diff = out - target
    loss = float(np.mean(diff * diff))
    g = r(2.0 * diff / n)                    # dL/dz of the last layer, stored in BF16
    dW, db = [None] * NLAYER, [None] * NLAYER
    for l in range(NLAYER - 1, -1, -1):
        dW[l] = conv_wgrad(a[l], g)
        db[l] = g.sum(axis=(1, 2, 3))
        if l > 0:
            da = conv_transpose(g, r(W[l]))
            g = r(da * gelu_grad(zs[l - 1]))
    return loss, np.concatenate([np.concatenate([w.ravel(), bb.ravel()]) for w, bb in zip(dW, db)]), out


def adam(theta, grad, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update (Kingma & Ba, 2015) in float32, bias-corrected."""
    m[:] = beta1 * m + (1 - beta1) * grad
    v[:] = beta2 * v + (1 - beta2) * grad * grad
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    theta[:] = theta - lr * mh / (np.sqrt(vh) + eps)

"""CPU oracle of the warm-start MLP (test infrastructure only).

Forward and backward of the 24 -> 64 -> 64 -> 64 -> 3 network with GELU and a
mean-squared-error loss, in FP64. The network's GELU is the FMA-only polynomial form
of the CUDA kernels (libatssim_b200/csrc/ats_gelu.cuh: g(z) = z (1/2 + z S(x)),
x = 2 z^2 / 4.5^2 - 1 for |z| < 4.5, z or 0 beyond), evaluated here in FP64 from the
same FP32 coefficients; it is within 1.2e-4 of z Phi(z). With quantize=True the values are rounded to
BF16 where the CUDA kernels round them (inputs, weights, hidden activations, the
output gradient and the pre-activation gradients that feed the GEMMs), so the
CUDA FP32-accumulated results can be compared tightly. With quantize=False it is
the exact FP64 network used for the finite-difference check of the gradients.
The parameter layout is the library's: W1[24][64] b1 W2[64][64] b2 W3[64][64] b3
W4[64][3] b4, W[in][out] row-major.
"""
import math

import numpy as np

IN, HID, OUT = 24, 64, 3
SHAPES = [("W1", (IN, HID)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, HID)),
          ("b3", (HID,)), ("W4", (HID, OUT)), ("b4", (OUT,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(theta):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(grads):
    return np.concatenate([grads[name].ravel() for name, _ in SHAPES])


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


GELU_CUT = 4.5
GELU_SCALE = float(np.float32(2.0 / 4.5 ** 2))  # 2 / cut^2 as the kernels hold it
GELU_POLY = np.array([
    1.569028050e-01, -7.717044652e-02, 5.479086563e-02, -4.057224095e-02, 2.779665403e-02,
    -1.670240983e-02, 1.189577673e-02, -9.356983006e-03, 3.531820374e-03,
], dtype=np.float32).astype(np.float64)  # S(x), lowest power first

_erf = np.vectorize(math.erf)


def gelu_exact(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def _poly(z):
    z = np.asarray(z, dtype=np.float64)
    x = z * z * GELU_SCALE - 1.0
    s = np.full_like(x, GELU_POLY[-1])
    d = np.zeros_like(x)
    for c in GELU_POLY[-2::-1]:
        d = d * x + s
        s = s * x + c
    return z, s, d


def gelu(z):
    z, s, _ = _poly(z)
    return np.where(z >= GELU_CUT, z, np.where(z <= -GELU_CUT, 0.0, z * (0.5 + z * s)))


def gelu_grad(z):
    z, s, d = _poly(z)
    g = 0.5 + 2.0 * z * s + 2.0 * GELU_SCALE * z ** 3 * d
    return np.where(z >= GELU_CUT, 1.0, np.where(z <= -GELU_CUT, 0.0, g))


def normalize_inputs(x, norm):
    """(f - in_mean) * in_scale with the library's 54-float normalisation vector."""
    norm = np.asarray(norm, dtype=np.float32)
    return ((np.asarray(x, dtype=np.float32) - norm[:IN]) * norm[IN:2 * IN]).astype(np.float64)


def denormalize_outputs(y, norm):
    norm = np.asarray(norm, dtype=np.float64)
    return norm[2 * IN:2 * IN + OUT] + norm[2 * IN + OUT:] * y


def forward(theta, x, quantize=True):
    p = unpack(theta)
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    h = q(x)
    zs, hs = [], [h]
    for l in (1, 2, 3):
        z = h @ q(p[f"W{l}"]) + p[f"b{l}"]
        zs.append(z)
        h = q(gelu(z))
        hs.append(h)
    y = h @ q(p["W4"]) + p["b4"]
    return y, zs, hs


def loss_and_grad(theta, x, t, quantize=True):
    """Mean over samples and outputs of (y - t)^2 and its gradient w.r.t. theta."""
    p = unpack(theta)
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    y, zs, hs = forward(theta, x, quantize)
    n = x.shape[0]
    e = y - t
    loss = float(np.mean(e * e))
    dy = 2.0 * e / (n * OUT)
    g = {}
    dyq = q(dy)
    g["W4"] = hs[3].T @ dyq
    g["b4"] = dy.sum(0)
    dz = (dyq @ q(p["W4"]).T) * gelu_grad(zs[2])
    for l in (3, 2):
        dzq = q(dz)
        g[f"W{l}"] = hs[l - 1].T @ dzq
        g[f"b{l}"] = dz.sum(0)
        dz = (dzq @ q(p[f"W{l}"]).T) * gelu_grad(zs[l - 2])
    dzq = q(dz)
    g["W1"] = hs[0].T @ dzq
    g["b1"] = dz.sum(0)
    return loss, pack(g)


def finite_difference(theta, x, t, idx, eps=1e-6):
    """Central difference of the unquantised loss for the parameters in idx."""
    out = np.zeros(len(idx))
    for j, i in enumerate(idx):
        tp = np.array(theta, dtype=np.float64)
        tm = tp.copy()
        tp[i] += eps
        tm[i] -= eps
        out[j] = (loss_and_grad(tp, x, t, False)[0] - loss_and_grad(tm, x, t, False)[0]) / (2 * eps)
    return out

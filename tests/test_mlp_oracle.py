"""The warm-start MLP oracle checks itself: analytic gradients against central
finite differences of the exact FP64 network (no GPU)."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.RandomState(0)
    theta = rng.uniform(-0.3, 0.3, M.NPARAMS)
    x = rng.standard_normal((7, M.IN))
    t = rng.standard_normal((7, M.OUT))
    _, g = M.loss_and_grad(theta, x, t, quantize=False)
    idx = rng.choice(M.NPARAMS, 40, replace=False)
    idx = np.concatenate([idx, [0, 1535, 1536, 10111, 10112, 10114]])
    fd = M.finite_difference(theta, x, t, idx)
    assert np.allclose(g[idx], fd, rtol=1e-5, atol=1e-9)


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.01171875, 1.001953125, -3.14159], dtype=np.float32)
    r = M.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0          # 1 + 2^-8: a tie, rounds to the even mantissa
    assert r[2] == 1.015625     # 1 + 3 * 2^-8: a tie, rounds up to the even mantissa
    assert r[3] == 1.0          # below half a BF16 ulp
    assert r[4] == -3.140625
    assert M.NPARAMS == 10115


def test_gelu_polynomial_is_the_kernels_and_close_to_exact():
    import os
    import re
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "libatssim_b200", "csrc", "ats_gelu.cuh")).read()
    body = hdr[hdr.index("kGeluPoly[kGeluDeg + 1] = {"):]
    body = body[body.index("{") + 1:body.index("}")]
    coefs = np.array([float(v.rstrip("f")) for v in re.findall(r"[-+0-9.e]+f", body)], dtype=np.float32)
    assert np.array_equal(coefs.astype(np.float64), M.GELU_POLY)
    z = np.linspace(-8, 8, 16001)
    assert np.max(np.abs(M.gelu(z) - M.gelu_exact(z))) < 1.2e-4
    # the derivative is the polynomial's own (central differences away from the cut)
    zz = np.linspace(-4.4, 4.4, 999)
    fd = (M.gelu(zz + 1e-6) - M.gelu(zz - 1e-6)) / 2e-6
    assert np.max(np.abs(fd - M.gelu_grad(zz))) < 1e-7

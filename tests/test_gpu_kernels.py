"""Kernel-level parity of the CUDA path against the oracle, through the C ABI.

Tolerances: the FFT within 1e-5 relative L2 of numpy's FP64 transform and of
the oracle's float transform (the per-kernel bar of this port); the blur,
the Gaussian weights and the max are bit-exact (same operation order as the
reference's CPU code, no contraction into FMA); the Dirac-delta known-answer
test uses the reference's own 30*FLT_EPSILON tolerance
(tests/imresh/algorithms/testGaussian.cpp:53-85).
"""
import numpy as np
import pytest

import imresh_b200 as imr
import oracle

pytestmark = pytest.mark.gpu
FLT_EPS = float(np.finfo(np.float32).eps)

FFT_SHAPES = [(256, 256), (2048, 2048), (128, 384), (384, 192), (512, 128), (64, 64),
              (7, 5), (1, 64), (64, 1), (210, 343), (3, 1536), (4096, 4096), (1024, 768),
              (100, 90),
              # Bluestein lengths (a prime factor > 7)
              (97, 101), (11, 64), (1031, 7), (64, 2039), (257, 300), (13, 13), (2047, 2)]


def _to_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("shape", FFT_SHAPES)
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft2d_matches_fp64_and_oracle(cuda, shape, sign):
    import torch
    rng = np.random.default_rng(hash(shape) % 2**32)
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    d = _to_dev(x)
    imr.fft2d(d, shape[1], shape[0], sign)
    torch.cuda.synchronize()
    y = d.cpu().numpy()
    xd = x.astype(np.complex128)
    ref = np.fft.fft2(xd) if sign < 0 else np.fft.ifft2(xd) * x.size
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-5
    if x.size <= 1 << 22:
        o = oracle.fft2(x, sign)
        assert np.linalg.norm(y - o) / np.linalg.norm(o) < 1e-5


def test_fft2d_roundtrip_is_scaled_identity(cuda):
    import torch
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((2048, 2048)) + 1j * rng.standard_normal((2048, 2048))).astype(np.complex64)
    d = _to_dev(x)
    imr.fft2d(d, 2048, 2048, -1)
    imr.fft2d(d, 2048, 2048, +1)
    torch.cuda.synchronize()
    y = d.cpu().numpy() / x.size
    assert np.linalg.norm(y - x) / np.linalg.norm(x) < 1e-6


@pytest.mark.parametrize("shape", [(1, 1), (3, 5), (37, 234), (256, 256), (1021, 31), (2048, 2048),
                                   (130, 1)])
@pytest.mark.parametrize("sigma", [0.5, 1.5, 3.0, 4.0])
def test_blur_bitexact_vs_oracle(cuda, shape, sigma):
    import torch
    rng = np.random.default_rng(11)
    img = rng.random(shape).astype(np.float32)
    for axes, axis in ((1, "h"), (2, "v"), (3, "hv")):
        d = _to_dev(img)
        tmp = torch.empty_like(d)
        imr.gaussian_blur(d, tmp, shape[1], shape[0], sigma, axes)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(d.cpu().numpy(), oracle.blur(img, sigma, axis))


@pytest.mark.parametrize("sigma", [0.1, 0.5, 1, 1.3, 1.7, 2, 3, 4])
def test_blur_dirac_deltas(cuda, sigma):
    import torch
    w = oracle.gaussian_weights(sigma)
    K = w.size
    half = (K - 1) // 2
    for nx in (31, 37, 234, 512, 1021, 1024):
        if nx < K:
            continue
        img = np.zeros((7, nx), np.float32)
        img[:, half:nx - half:K] = 1
        sol = np.zeros_like(img)
        c = 0
        while c + K - 1 < nx:
            sol[:, c:c + K] = w
            c += K
        for axes, a, s in ((1, img, sol), (2, img.T.copy(), sol.T.copy())):
            d = _to_dev(a)
            tmp = torch.empty_like(d)
            imr.gaussian_blur(d, tmp, a.shape[1], a.shape[0], sigma, axes)
            torch.cuda.synchronize()
            r = d.cpu().numpy()
            m = max(np.abs(r).max(), np.abs(s).max())
            assert np.abs(r - s).max() / m <= 30 * FLT_EPS


@pytest.mark.parametrize("n", [1, 2, 1000, 65537, 1 << 22, 64 * 1024 * 1024])
def test_vector_max_planted(cuda, n):
    import torch
    g = torch.Generator(device="cuda").manual_seed(350471643)
    d = torch.rand(n, device="cuda", generator=g) - 0.5
    if n == 1:
        assert imr.vector_max(d, n) == d.item()
        return
    k = n // 3
    d[k] = 7.37519
    assert imr.vector_max(d, n) == np.float32(7.37519)
    d[k] = -7.37519
    assert imr.vector_max(-d, n) == np.float32(7.37519)

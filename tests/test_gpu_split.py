"""The split-precision tensor-core column stages (IMR_PREC_BF16X3 /
IMR_PREC_FP16X3): radix-16 DFT stages as DFT-16 matrix products on the
tensor cores with hi+lo split operands and FP32 accumulation, everything
else FP32 (FP64 error sums).  They stand in for the column halves of the
cuFFT calls of cudaShrinkWrap.cu:319,343.

Tolerances: the 2D transform within 1e-5 relative L2 of numpy's FP64 FFT at
every supported height up to 4096 (the FP32 transform reaches ~3e-7); one
HIO iteration of the path within 1e-4 of the oracle's FP32 path, as the
FP32 GPU path is held to; longer runs are compared by their per-cycle error,
as for the FP32 path (the iterations are chaotic).
"""
import numpy as np
import pytest

import imresh_b200 as imr
import oracle
from imresh_b200 import data
from imresh_b200.metrics import rel_l2

pytestmark = pytest.mark.gpu
FLT_MIN = imr.FLT_MIN
PRECS = [imr.PREC_BF16X3, imr.PREC_FP16X3]


def _tile(H):
    return {256: 16, 512: 16, 1024: 8, 2048: 4, 4096: 2}[H]


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("H,W", [(256, 64), (512, 48), (1024, 40), (2048, 12), (4096, 6), (4096, 4096)])
def test_split_fft2d_matches_numpy_fp64(cuda, prec, H, W):
    import torch
    rng = np.random.default_rng(H + W)
    x = (rng.standard_normal((H, W)) + 1j * rng.standard_normal((H, W))).astype(np.complex64)
    x[0, 0] += 50.0 * np.sqrt(H * W)   # a strong DC term, as diffraction data has
    for sign in (-1, +1):
        d = torch.from_numpy(x.view(np.float32).copy()).cuda()
        imr.fft2d_split(d, W, H, sign, prec)
        torch.cuda.synchronize()
        got = d.cpu().numpy().view(np.complex64)
        want = np.fft.fft2(x.astype(np.complex128)) if sign < 0 else \
            np.fft.ifft2(x.astype(np.complex128)) * (H * W)
        err = rel_l2(got, want)
        assert err < 1e-5, (prec, H, W, sign, err)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("shape", [(256, 256), (512, 384), (4096, 64), (1024, 1024)])
def test_split_path_one_iteration_matches_oracle(cuda, prec, shape):
    H, W = shape
    spec = data.BlobSpec(W, H, 12, 0.15 * min(W, H), (1.5, 2.5), (0.5, 1.0), 1e9)
    M, _ = data.make_modulus(spec, 1)
    p = oracle.SwParams(1, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 1)
    ref = oracle.shrinkwrap(M, p)
    plan = imr.Plan(W, H, imr.Params(1, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 1))
    plan.set_precision(prec)
    out = plan.execute_host(M)
    n, errs = plan.stats()
    mask = plan.state("mask")
    plan.close()
    assert n == 1
    assert np.mean(mask != ref.mask) <= 1e-3
    assert rel_l2(out, ref.out) < 1e-4
    assert errs[0] == pytest.approx(ref.errors[0], rel=1e-4)


@pytest.mark.parametrize("prec", PRECS)
def test_split_path_error_curve_follows_fp32(cuda, prec):
    """4 cycles x 20 iterations of the 2048^2 Poisson workload: the error of
    cycle 0 within 1 % of the FP32 path's [measured: 0.03 %], those of
    cycles 1-3 within 7 %.  The split path's transforms are 1e-5 (BF16) and
    3e-7 (FP16) from FP64 against the FP32 path's 2e-7, so its run leaves the
    FP32 trajectory about a cycle earlier than FP32 runs leave each other
    (measured at cycle 1: BF16 -2.7 %, FP16 -1.4 %, while 12 FP32 reference
    runs on inputs one ulp apart agree within 0.2 % there); once separated,
    runs differ by the ensemble spread (3.5 % over those 12 runs at cycles
    2-3), and this compares two members of it."""
    M, _ = data.make_modulus(data.cfg1_spec(), 1)
    prm = imr.Params(4, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 20)
    a = imr.Plan(2048, 2048, prm)
    a.execute_host(M)
    _, e32 = a.stats()
    a.set_precision(prec)
    out = a.execute_host(M)
    _, es = a.stats()
    a.close()
    assert np.all(np.isfinite(out))
    np.testing.assert_allclose(es[:1], e32[:1], rtol=0.01)
    np.testing.assert_allclose(es[1:], e32[1:], rtol=0.07)


def test_split_precision_rejects_unsupported_heights(cuda):
    plan = imr.Plan(128, 128, imr.Params(1, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 1))
    with pytest.raises(imr.ImrError) as e:
        plan.set_precision(imr.PREC_BF16X3)
    assert e.value.status == 2
    plan.close()

"""Parity of the fixed-support random-phase HIO (libs::hybridInputOutput,
src/imresh/libs/hybridInputOutput.cpp:126-306) and of the standalone HIO
error (cudaCalculateHioError, src/imresh/algorithms/cuda/cudaVectorReduce.cu:357-403)
on the GPU, through the C ABI, against the oracle (itself bit-exact against
the reference's own CPU code, tests/test_oracle.py).

Tolerances:
* the device rand() field is bit-exact against the C library's rand();
* the standalone error reproduces the reference test's Pythagorean
  known answer exactly (total = 5 * count) and agrees with the oracle's double
  sums to float rounding;
* the reconstruction: within 1e-5 relative L2 of the oracle's float path
  before any update, and after up to five updates within 1e-4 or, where HIO
  already amplifies float rounding (256^2 random phase: the oracle's own
  float and FP64 runs differ by 4e-4 after five), within 10x the oracle's own
  float-vs-FP64 distance; iteration counts equal; the same yardstick at long
  horizons.
"""
import numpy as np
import pytest

import imresh_b200 as imr
import oracle
from imresh_b200 import data

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _assert_close_to_oracle(out, ref_out, M, mask, n, seed=imr.HIO_SEED):
    """Within 1e-4 of the oracle's float path, or within 10x the oracle's own
    float-vs-FP64 distance where HIO already amplifies float rounding."""
    d = _rel(out, ref_out)
    if d >= 1e-4:
        ref64 = oracle.hio(M, mask, n, 1e-30, 0.9, seed=seed, fp64=True)
        assert d <= 10 * _rel(ref_out, ref64.out)


def _case(H, W, seed=3, n_blobs=8):
    spec = data.BlobSpec(W, H, n_blobs, min(W, H) / 6.0, (1.5, 2.0), (0.5, 1.0), None)
    M, _ = data.make_modulus(spec, seed)
    return data.centrosymmetric(M), data.support_mask(spec)


@pytest.mark.parametrize("n,seed", [(1, imr.HIO_SEED), (2, 1), (31, 0), (992, 350471643),
                                    (993, imr.HIO_SEED), (12345, 7), ((1 << 20) + 7, imr.HIO_SEED)])
def test_rand_field_bitexact_vs_c_library(cuda, n, seed):
    import torch
    d = torch.empty(n, dtype=torch.complex64, device="cuda")
    imr.rand_field(d, n, seed)
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    np.testing.assert_array_equal(got.real, oracle.rand_field(n, seed))
    assert not got.imag.any()


@pytest.mark.parametrize("mask_kind", ["f32", "u8"])
@pytest.mark.parametrize("n", [1, 2, 1000, 65537, 1 << 22])
def test_hio_error_pythagorean(cuda, mask_kind, n):
    """tests/imresh/algorithms/testVectorReduce.cu:248-413: masked values are
    (3, 4), so total = 5 * count exactly while total < 2^24."""
    import torch
    rng = np.random.default_rng(350471643)
    mask = (rng.random(n) < 0.5).astype(np.float32)
    z = (rng.random(n) + 1j * rng.random(n)).astype(np.complex64)
    z[mask == 1] = 3 + 4j
    dz = torch.from_numpy(z).cuda()
    dm = torch.from_numpy(mask if mask_kind == "f32" else mask.astype(np.uint8)).cuda()
    total, count, err = imr.calculate_hio_error(dz, dm, n)
    assert count == mask.sum()
    if total < 2 ** 24:
        assert total == 5 * count
    e, t, c = oracle.hio_error(z, mask)
    assert total == pytest.approx(t, rel=1e-6)
    if count:
        assert err == pytest.approx(e, rel=1e-6)
    t2, c2, _ = imr.calculate_hio_error(dz, dm, n, invert_mask=True)   # the complement
    assert c2 == n - count
    _, tt2, _ = oracle.hio_error(z, 1 - mask)
    assert t2 == pytest.approx(tt2, rel=1e-6)


SHAPES = [(64, 64), (48, 64), (96, 256), (256, 256), (192, 384), (30, 42), (97, 101), (2048, 2048)]


@pytest.mark.parametrize("shape", SHAPES)
def test_initial_phase_matches_oracle(cuda, shape):
    """target 1e30: the test at k = 0 stops at once, so the result is
    Re(IFFT2(M e^{i arg FFT2(rand field)})) (addRandomPhase + one transform)."""
    H, W = shape
    M, mask = _case(H, W)
    io = M.copy()
    assert imr.hybrid_input_output(io, mask, 5, 1e30, 0.9) == 0
    ref = oracle.hio(M, mask, 5, 1e30, 0.9)
    assert ref.iterations == 0
    assert _rel(io, ref.out) < 1e-5


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("n", [1, 5])
def test_short_horizon_matches_oracle(cuda, shape, n):
    H, W = shape
    M, mask = _case(H, W)
    plan = imr.HioPlan(W, H, n, 1e-30, 0.9)
    out = plan.execute_host(M, mask)
    iters, last, errs = plan.stats()
    plan.close()
    ref = oracle.hio(M, mask, n, 1e-30, 0.9)
    assert iters == ref.iterations == n
    _assert_close_to_oracle(out, ref.out, M, mask, n)
    np.testing.assert_allclose(errs[:n + 1], ref.errors[:n + 1], rtol=1e-4)


def test_stop_test_matches_oracle(cuda):
    M, mask = _case(64, 64, seed=5)
    errs = oracle.hio(M, mask, 60, 1e-30, 0.9).errors
    k = next(k for k in range(5, 60) if errs[k] < 0.98 * errs[:k].min())
    target = float(0.5 * (errs[k] + errs[:k].min()))
    ref = oracle.hio(M, mask, 60, target, 0.9)
    plan = imr.HioPlan(64, 64, 60, target, 0.9)
    out = plan.execute_host(M, mask)
    iters, last, _ = plan.stats()
    plan.close()
    assert iters == ref.iterations == k
    assert last < target
    assert _rel(out, ref.out) < 1e-3


def test_fixed_count_without_error_test(cuda):
    """targetError <= 0: no test, exactly nCycles updates, then the result."""
    M, mask = _case(128, 128)
    plan = imr.HioPlan(128, 128, 37, 0.0, 0.9)
    out = plan.execute_host(M, mask)
    iters, _, _ = plan.stats()
    plan.close()
    assert iters == 37
    ref = oracle.hio(M, mask, 37, 0.0, 0.9)
    ref64 = oracle.hio(M, mask, 37, 0.0, 0.9, fp64=True)
    assert _rel(out, ref.out) <= max(10 * _rel(ref.out, ref64.out), 1e-4)


@pytest.mark.parametrize("shape", [(256, 256), (384, 192)])
def test_long_horizon_within_yardstick(cuda, shape):
    H, W = shape
    M, mask = _case(H, W, n_blobs=20)
    n = 200
    plan = imr.HioPlan(W, H, n, 1e-30, 0.9)
    out = plan.execute_host(M, mask)
    plan.close()
    f32 = oracle.hio(M, mask, n, 1e-30, 0.9).out
    f64 = oracle.hio(M, mask, n, 1e-30, 0.9, fp64=True).out
    assert _rel(out, f32) <= max(10 * _rel(f32, f64), 1e-4)


def test_drop_in_equals_plan_and_is_deterministic(cuda):
    M, mask = _case(96, 160)
    a = M.copy()
    assert imr.hybrid_input_output(a, mask, 25, 1e-30, 0.9) == 0
    b = M.copy()
    assert imr.hybrid_input_output(b, mask, 25, 1e-30, 0.9) == 0
    plan = imr.HioPlan(160, 96, 25, 1e-30, 0.9)
    c = plan.execute_host(M, mask)
    d = plan.execute_host(M, mask)   # plan reuse
    plan.close()
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)
    np.testing.assert_array_equal(a, d)


def test_device_buffers_and_seed(cuda):
    import torch
    M, mask = _case(128, 96)
    dm = torch.from_numpy(M).cuda()
    dk = torch.from_numpy(mask).cuda()
    out = torch.empty_like(dm)
    plan = imr.HioPlan(96, 128, 8, 1e-30, 0.9)
    plan.execute(dm, dk, out)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), plan.execute_host(M, mask))
    other = plan.execute_host(M, mask, seed=7)
    plan.close()
    _assert_close_to_oracle(other, oracle.hio(M, mask, 8, 1e-30, 0.9, seed=7).out, M, mask, 8, seed=7)


def test_unsupported_size_and_null_arguments(cuda):
    M = np.ones((4, 2500), np.float32)
    mask = np.zeros((4, 2500), np.uint8)
    assert imr.hybrid_input_output(M, mask, 2, 0.0, 0.9) == 2
    L = imr.lib()
    assert L.imr_hybrid_input_output(None, mask.ctypes.data, 4, 4, 1, 0.0, 0.9, None) == 1

"""Path-level parity of the CUDA shrink-wrap engine against the oracle,
through the C ABI.

HIO is chaotic: the reference's own float and FP64 runs separate over long
runs (oracle f32 vs f64 after 64 x 20 iterations at 256^2: > 100 % relative
L2).  Parity is therefore pinned where it is meaningful:
* short horizons (one and two cycles) against the oracle's float path, with
  the support masks compared pixel by pixel (<= 0.1 % differing);
* the per-cycle error metric;
* exact agreement between the drop-in call and the plan API, run-to-run
  determinism, the stop test and the reference's parameter defaults.
"""
import numpy as np
import pytest

import imresh_b200 as imr
import oracle
from imresh_b200 import data

pytestmark = pytest.mark.gpu
FLT_MIN = imr.FLT_MIN


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _spec(W, H, seed_blobs=12):
    return data.BlobSpec(W, H, seed_blobs, 0.15 * min(W, H), (1.5, 2.5), (0.5, 1.0), None)


def _run_gpu(M, p: oracle.SwParams, cuda_defaults=False):
    H, W = M.shape
    prm = imr.Params(p.n_cycles, p.target_error, p.beta, p.cut_auto, p.cut, p.sigma0,
                     p.sigma_change, p.n_hio)
    plan = imr.Plan(W, H, prm)
    out = plan.execute_host(M)
    n, errs = plan.stats()
    mask = plan.state("mask")
    plan.close()
    return out, n, errs, mask


@pytest.mark.parametrize("shape", [(64, 64), (256, 256), (128, 384), (192, 512), (2048, 2048),
                                   (97, 130), (211, 64),
                                   # column-tiled modulus: 2-column tiles at length 4096, and a
                                   # last tile of 4 of 16 columns
                                   (4096, 64), (256, 132),
                                   # half-tile column passes whose last tile's second half lies
                                   # past the width; a Bluestein width over 8-value half tiles
                                   (512, 520), (128, 1000)])
def test_one_cycle_matches_oracle(cuda, shape):
    H, W = shape
    M, _ = data.make_modulus(_spec(W, H), 1)
    p = oracle.SwParams(1, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 1)
    ref = oracle.shrinkwrap(M, p)
    out, n, errs, mask = _run_gpu(M, p)
    assert n == 1
    assert np.mean(mask != ref.mask) <= 1e-3
    assert _rel(out, ref.out) < 1e-4
    assert errs[0] == pytest.approx(ref.errors[0], rel=1e-4)


@pytest.mark.parametrize("shape", [(64, 64), (256, 256), (96, 160), (128, 200)])
def test_five_iterations_match_oracle(cuda, shape):
    """One cycle of five HIO iterations: before HIO's amplification takes
    over (about x2 per iteration on these inputs) the GPU stays within 1e-4
    of the oracle's float path, with identical masks."""
    H, W = shape
    M, _ = data.make_modulus(_spec(W, H), 2)
    p = oracle.SwParams(1, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 5)
    ref = oracle.shrinkwrap(M, p)
    out, n, errs, mask = _run_gpu(M, p)
    assert n == 1
    assert np.mean(mask != ref.mask) <= 1e-3
    assert _rel(out, ref.out) < 1e-4
    np.testing.assert_allclose(errs, ref.errors, rtol=1e-4)


@pytest.mark.parametrize("shape", [(64, 64), (256, 256)])
def test_divergence_no_worse_than_float_rounding(cuda, shape):
    """Two cycles of ten iterations: the GPU's distance from the oracle's
    float path is of the order of the distance between the oracle's own
    float and FP64 runs (the yardstick for rounding-driven divergence)."""
    H, W = shape
    M, _ = data.make_modulus(_spec(W, H), 2)
    p = oracle.SwParams(2, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 10)
    r32 = oracle.shrinkwrap(M, p)
    r64 = oracle.shrinkwrap(M, p, fp64=True)
    out, n, errs, mask = _run_gpu(M, p)
    assert n == 2
    yard = _rel(r32.out, r64.out)
    assert _rel(out, r32.out) <= 10 * yard + 1e-6
    assert _rel(out, r64.out) <= 10 * yard + 1e-6


def test_drop_in_equals_plan_and_is_deterministic(cuda):
    M, _ = data.make_modulus(_spec(256, 256), 3)
    io = M.reshape(-1).copy()
    rc = imr.cuda_shrink_wrap(io, 256, 256, 0, 96, 256, 3, FLT_MIN, 0, 0.04, 0.2, 0, 0, 5)
    assert rc == 0
    out, n, _, _ = _run_gpu(M, oracle.SwParams(3, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 5))
    np.testing.assert_array_equal(io.reshape(256, 256), out)
    io2 = M.reshape(-1).copy()
    assert imr.cuda_shrink_wrap(io2, 256, 256, 0, 96, 256, 3, FLT_MIN, 0, 0.04, 0.2, 0, 0, 5) == 0
    np.testing.assert_array_equal(io, io2)


def test_stop_test_matches_oracle(cuda):
    M, _ = data.make_modulus(_spec(128, 128), 4)
    p = oracle.SwParams(8, 1e9, 0.9, 0.04, 0.2, 3.0, 0.01, 4)   # E < 1e9 after cycle 0
    ref = oracle.shrinkwrap(M, p)
    out, n, errs, _ = _run_gpu(M, p)
    assert ref.cycles_run == 1 and n == 1
    assert _rel(out, ref.out) < 1e-4


def test_reference_cuda_defaults(cuda):
    """All-zero parameters select cudaShrinkWrap's defaults (cu:193-200):
    20 cycles x 20 HIO iterations, autocorrelation cutoff 0.02."""
    M, _ = data.make_modulus(_spec(64, 64), 5)
    plan = imr.Plan(64, 64, imr.Params())
    assert plan.launches() == 1 + 20 * (2 + 2 * 20) + 2
    out = plan.execute_host(M)
    n, errs = plan.stats()
    assert 1 <= n <= 20 and np.all(np.isfinite(out))
    # same run with the defaults spelled out
    plan2 = imr.Plan(64, 64, imr.Params(20, 1e-5, 0.9, 0.02, 0.2, 3.0, 0.01, 20))
    np.testing.assert_array_equal(plan2.execute_host(M), out)


def test_unsupported_size_is_an_error(cuda):
    with pytest.raises(imr.ImrError) as e:
        imr.Plan(2500, 64)
    assert e.value.status == 2
    io = np.zeros(4097 * 2, np.float32)
    assert imr.cuda_shrink_wrap(io, 4097, 2) == 2


def test_full_config0_run(cuda):
    """The 256x256 blob workload, 64 cycles x 20 iterations: runs every
    cycle, reports finite errors of the same magnitude as the oracle's."""
    M, _ = data.make_modulus(data.cfg0_spec(), 0)
    p = oracle.SwParams(64, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 20)
    out, n, errs, mask = _run_gpu(M, p)
    assert n == 64
    assert np.all(np.isfinite(out)) and np.all(np.isfinite(errs))
    assert 0 < errs[-1] < 10

"""Pins the CPU oracle (oracle/) before anything is checked against it.

1. The project FFT against numpy's FP64 pocketfft (FFTW itself is not
   installed; no reference test pins FFT output).
2. The restated CPU path against the reference's own shrinkWrap compiled
   from its sources (oracle/_ref): bit-for-bit.
3. The known-answer tests of the reference's test suite for this path:
   tests/imresh/algorithms/testGaussian.cpp (Dirac deltas 217-337, single
   row/column 340-397, constant images 400-544, random-data properties
   134-148 and 547-677), tests/imresh/algorithms/testVectorReduce.cu
   (length-1 and planted +-7.37519 extrema 75-194, Pythagorean HIO error
   248-413).
"""
import numpy as np
import pytest

import oracle
from imresh_b200 import data

FLT_EPS = float(np.finfo(np.float32).eps)
FLT_MIN = float(np.finfo(np.float32).tiny)


def _ref_or_skip():
    L = oracle.ref_lib()
    if L is None:
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    return L


# ------------------------------------------------------------------ FFT
@pytest.mark.parametrize("shape", [(1, 1), (2, 3), (8, 8), (16, 12), (30, 45), (64, 64),
                                   (97, 101), (127, 128), (256, 256), (1, 257), (210, 385),
                                   (1031, 7), (192, 384)])
def test_fft_matches_numpy(shape):
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    for sign in (-1, 1):
        ref = np.fft.fft2(x) if sign < 0 else np.fft.ifft2(x) * x.size
        y64 = oracle.fft2(x.astype(np.complex128), sign)
        y32 = oracle.fft2(x.astype(np.complex64), sign)
        assert np.linalg.norm(y64 - ref) / np.linalg.norm(ref) < 1e-13
        assert np.linalg.norm(y32 - ref) / np.linalg.norm(ref) < 1e-6


def test_fft_rows_cols_compose():
    rng = np.random.default_rng(2)
    x = (rng.standard_normal((48, 80)) + 1j * rng.standard_normal((48, 80))).astype(np.complex64)
    a = oracle.fft_cols(oracle.fft_rows(x, -1), -1)
    np.testing.assert_array_equal(a, oracle.fft2(x, -1))


# ------------------------------------------------------------------ weights
@pytest.mark.parametrize("sigma", [0.1, 0.5, 1, 1.3, 1.5, 1.7, 2, 3, 4, 2.9403, 7.5])
def test_gaussian_weights_match_reference(sigma):
    L = _ref_or_skip()
    w = oracle.gaussian_weights(sigma)
    wr = np.zeros(64, np.float32)
    k = L.imro_ref_weights(sigma, wr.ctypes.data, 64)
    assert k == w.size
    np.testing.assert_array_equal(w, wr[:k])
    # sum to one, symmetric, peaked at the centre
    assert abs(float(w.astype(np.float64).sum()) - 1.0) < 1e-6
    np.testing.assert_array_equal(w, w[::-1])


# ------------------------------------------------------------------ blur KATs
SIGMAS = [0.1, 0.5, 1, 1.3, 1.7, 2, 3, 4]
SIZES = [1, 2, 3, 5, 10, 31, 37, 234, 512, 1021]


def _rel_err(a, b):
    m = max(np.abs(a).max(), np.abs(b).max())
    return np.abs(a - b).max() / (m if m else 1.0)


@pytest.mark.parametrize("sigma", SIGMAS)
def test_blur_dirac_deltas(sigma):
    """testGaussianDiracDeltas: deltas one kernel width apart blur into exact
    copies of the weights; tolerance maxAbsDiff/maxAbs <= 30*FLT_EPSILON."""
    w = oracle.gaussian_weights(sigma)
    K = w.size
    half = (K - 1) // 2
    for nx in SIZES:
        ny = 5
        if nx >= K:
            img = np.zeros((ny, nx), np.float32)
            img[:, half:nx - half:K] = 1
            sol = np.zeros_like(img)
            c = 0
            while c + K - 1 < nx:
                sol[:, c:c + K] = w
                c += K
            assert _rel_err(oracle.blur(img, sigma, "h"), sol) <= 30 * FLT_EPS
            assert _rel_err(oracle.blur(img.T.copy(), sigma, "v"), sol.T) <= 30 * FLT_EPS


@pytest.mark.parametrize("shape", [(1, 1), (1, 37), (37, 1), (5, 1021), (234, 10), (64, 64)])
def test_blur_constant_and_single_line(shape):
    """testGaussianConstantValues / testGaussianRandomSingleData: constant
    images are invariant; a single row blurred vertically (or a single column
    blurred horizontally) is unchanged up to rounding (clamp border), within
    the reference's 30*FLT_EPSILON relative tolerance."""
    rng = np.random.default_rng(350471643)
    const = np.full(shape, 0.73, np.float32)
    out = oracle.blur(const, 3.0, "hv")
    assert _rel_err(out, const) <= 30 * FLT_EPS
    r = (rng.random(shape) - 0.5).astype(np.float32)
    for sigma in SIGMAS:
        if shape[0] == 1:
            assert _rel_err(oracle.blur(r, sigma, "v"), r) <= 30 * FLT_EPS
        if shape[1] == 1:
            assert _rel_err(oracle.blur(r, sigma, "h"), r) <= 30 * FLT_EPS


def test_blur_random_properties():
    """checkGaussian: range does not widen and the max neighbour difference
    does not grow, per row (horizontal) and per column (vertical)."""
    rng = np.random.default_rng(350471643)
    img = (rng.random((97, 131)) - 0.5).astype(np.float32)
    h = oracle.blur(img, 3.0, "h")
    v = oracle.blur(img, 3.0, "v")
    for y in range(img.shape[0]):
        assert h[y].min() >= img[y].min() and h[y].max() <= img[y].max()
        assert np.abs(np.diff(h[y])).max() <= np.abs(np.diff(img[y])).max()
    for x in range(img.shape[1]):
        assert v[:, x].min() >= img[:, x].min() and v[:, x].max() <= img[:, x].max()
        assert np.abs(np.diff(v[:, x])).max() <= np.abs(np.diff(img[:, x])).max()


@pytest.mark.parametrize("shape", [(1, 1), (3, 5), (37, 234), (256, 256), (1021, 31)])
@pytest.mark.parametrize("sigma", [0.5, 1.5, 3.0, 4.0])
def test_blur_bitexact_vs_reference(shape, sigma):
    L = _ref_or_skip()
    rng = np.random.default_rng(7)
    img = rng.random(shape).astype(np.float32)
    for axis, fn in (("h", L.imro_ref_blur_h), ("v", L.imro_ref_blur_v), ("hv", L.imro_ref_blur)):
        ref = img.copy()
        fn(ref.reshape(-1), shape[1], shape[0], sigma)
        np.testing.assert_array_equal(oracle.blur(img, sigma, axis), ref)


# ------------------------------------------------------------------ reductions
def test_vector_max_kats():
    """testVectorReduce: length 1, and planted +-7.37519 in U(-0.5, 0.5) data."""
    rng = np.random.default_rng(350471643)
    d = (rng.random(1 << 20) - 0.5).astype(np.float32)
    assert oracle.vector_max(d[:1]) == d[0]
    for n in (2, 17, 1000, 65537, 1 << 20):
        k = int(rng.integers(0, n))
        x = d[:n].copy()
        x[k] = np.float32(7.37519)
        assert oracle.vector_max(x) == np.float32(7.37519)
    L = oracle.ref_lib()
    if L is not None:
        x = d.copy()
        x[12345] = np.float32(7.37519)
        assert L.imro_ref_vector_max(x, x.size) == np.float32(7.37519)


@pytest.mark.parametrize("n", [1, 2, 33, 1000, 65536, 1 << 20])
def test_hio_error_pythagorean(n):
    """testCalculateHioError: masked pixels hold (3, 4), so the total is
    exactly 5 * count; the CPU reference agrees within sqrt(n)*eps."""
    rng = np.random.default_rng(n)
    mask = (rng.random(n) < 0.3).astype(np.float32)
    g = rng.random((n, 2)).astype(np.float32)
    g[mask == 1] = (3.0, 4.0)
    gc = g.view(np.complex64).reshape(-1)
    e, tot, cnt = oracle.hio_error(gc, mask)
    assert cnt == mask.sum()
    assert tot == 5.0 * cnt
    if cnt:
        assert e == pytest.approx(np.sqrt(tot) / cnt, rel=1e-15)
    L = oracle.ref_lib()
    if L is not None and cnt:
        import ctypes as C
        t, c = C.c_float(), C.c_float()
        L.imro_ref_hio_error(g.reshape(-1), mask, n, C.byref(t), C.byref(c))
        assert c.value == cnt
        assert abs(t.value - tot) <= np.sqrt(n) * FLT_EPS * tot


# ------------------------------------------------------------------ full path
@pytest.mark.parametrize("shape,cycles,hio", [((48, 64), 4, 6), ((64, 64), 3, 10), ((45, 30), 2, 5)])
def test_restated_shrinkwrap_bitexact_vs_reference(shape, cycles, hio):
    _ref_or_skip()
    H, W = shape
    spec = data.BlobSpec(W, H, 10, min(W, H) / 5.0, (1.5, 2.5), (0.5, 1.0), None)
    M, _ = data.make_modulus(spec, 0)
    p = oracle.SwParams(cycles, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, hio)
    ours = oracle.shrinkwrap(M, p)
    ref = oracle.ref_shrinkwrap(M, p)
    np.testing.assert_array_equal(ours.out, ref)
    assert ours.cycles_run == cycles


def test_restated_shrinkwrap_stops_like_reference():
    _ref_or_skip()
    M, _ = data.make_modulus(data.BlobSpec(32, 32, 6, 6.0, (1.5, 1.5), (0.5, 1.0), None), 3)
    p = oracle.SwParams(6, 1e9, 0.9, 0.04, 0.2, 3.0, 0.01, 4)   # stops after cycle 0
    ours = oracle.shrinkwrap(M, p)
    assert ours.cycles_run == 1
    np.testing.assert_array_equal(ours.out, oracle.ref_shrinkwrap(M, p))


def test_fp64_oracle_is_close_at_short_horizon():
    M, _ = data.make_modulus(data.BlobSpec(64, 64, 10, 12.0, (2.0, 2.0), (0.5, 1.0), None), 0)
    p = oracle.SwParams(1, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 2)
    a = oracle.shrinkwrap(M, p).out
    b = oracle.shrinkwrap(M, p, fp64=True).out
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5


# ------------------------------------------------------------------ fixed-support HIO
def _hio_case(H, W, seed=3):
    spec = data.BlobSpec(W, H, 8, min(W, H) / 6.0, (1.5, 2.0), (0.5, 1.0), None)
    M, _ = data.make_modulus(spec, seed)
    return data.centrosymmetric(M), data.support_mask(spec)


def test_rand_field_is_the_c_library_stream():
    """The oracle's random field is srand(2623091912)/rand() itself, checked
    against glibc's published additive feedback generator restated here."""
    f = oracle.rand_field(400)
    r = [2623091912 - (1 << 32)]
    for i in range(1, 31):
        r.append((16807 * r[i - 1]) % 2147483647)
    r = [x & 0xFFFFFFFF for x in r]
    r += [r[i - 31] for i in range(31, 34)]
    for i in range(34, 344 + 400):
        r.append((r[i - 31] + r[i - 3]) & 0xFFFFFFFF)
    want = (np.array([x >> 1 for x in r[344:]], np.int64).astype(np.float32)
            / np.float32(2147483647.0))
    np.testing.assert_array_equal(f, want)


@pytest.mark.parametrize("shape,n,target", [((48, 64), 1, 0.0), ((48, 64), 5, 0.0),
                                            ((64, 64), 30, -1.0), ((30, 42), 12, 0.0),
                                            ((1, 8), 3, 0.0), ((48, 64), 3, 1e30),
                                            ((17, 24), 7, 0.0)])
def test_restated_hio_bitexact_vs_reference(shape, n, target):
    _ref_or_skip()
    M, mask = _hio_case(*shape)
    ours = oracle.hio(M, mask, n, target, 0.9)
    ref = oracle.ref_hio(M, mask, n, target, 0.9)
    np.testing.assert_array_equal(ours.out, ref)
    assert ours.iterations == (0 if target > 1 else n)


def test_restated_hio_stops_like_reference():
    _ref_or_skip()
    M, mask = _hio_case(64, 64, seed=5)
    errs = oracle.hio(M, mask, 60, 1e-30, 0.9).errors
    # first new minimum that beats every earlier error by a clear margin
    k = next(k for k in range(5, 60) if errs[k] < 0.98 * errs[:k].min())
    target = float(0.5 * (errs[k] + errs[:k].min()))
    ours = oracle.hio(M, mask, 60, target, 0.9)
    assert ours.iterations == k
    np.testing.assert_array_equal(ours.out, oracle.ref_hio(M, mask, 60, target, 0.9))


def test_hio_defaults_follow_reference():
    """beta <= 0 selects 0.9 (hybridInputOutput.cpp:209)."""
    M, mask = _hio_case(32, 32)
    a = oracle.hio(M, mask, 4, 0.0, 0.9).out
    np.testing.assert_array_equal(oracle.hio(M, mask, 4, 0.0, 0.0).out, a)
    np.testing.assert_array_equal(oracle.hio(M, mask, 4, 0.0, -1.0).out, a)

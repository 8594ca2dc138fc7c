"""Parity of whole reconstructions at the benchmark sizes and lengths: the
256x256 blob workload run in full (64 cycles x 20 HIO iterations) and the
2048x2048 Poisson workload for 4 cycles x 20 iterations, through the drop-in
call, against the reference's own CPU shrinkWrap (oracle/_ref, FP32) and the
FP64 restatement of it.

Why statistics and not images.  HIO amplifies rounding differences by about
2x per iteration on these inputs.  The reference's FP32 path and its FP64
restatement agree to 1e-6 after one cycle of five iterations, then part:
after 64 cycles (cfg 256^2) or 4 cycles (2048^2) their Re(g') are, after
twin/translation alignment, about as far apart (relative L2 1.1-1.4) as two
unrelated images of equal norm (sqrt(2)); so are reference runs whose inputs
differ by one float ulp in a few pixels.  No FP32 implementation, the
reference included, can reach 1e-3 on final images; what one can require is
that the GPU's run is statistically one more member of the ensemble the
reference's own runs form.  Short horizons, where images must agree, are
pinned in test_gpu_shrinkwrap.py (1 and 5 iterations within 1e-4, masks equal).

Tolerances (spread of the CPU ensemble measured with the reference's own
code in brackets):
* the restated oracle equals the reference's shrinkWrap bit for bit over the
  whole 64 x 20 run;
* per-cycle HIO error after cycle 0 (20 iterations) within 2 % of the
  reference's [0.7 %]; at 2048^2 the errors of cycles 0 and 1, before the
  runs separate, within 1 % [0.1 %], those of cycles 2 and 3 within 5 % of
  the reference's and of the FP64 run [12 reference runs on inputs moved by
  one ulp in 10 pixels: -3.4 % .. +0.3 % around the unperturbed run];
* 256^2: median error over the last 32 cycles, mean over the last 48 and the
  minimum over the run each within 10 % of the ensemble mean [4 %];
* aligned relative L2 of the GPU result to the FP64 run, and to the FP32
  reference run, at most 1.2 x the largest such distance of an FP32
  ensemble member [members: 1.11-1.42];
* aligned relative L2 to the ground-truth object at most 1.15 x the largest
  of the ensemble [1.03-1.10 at 256^2, 1.18-1.21 at 2048^2].
The numbers are printed (pytest -s) for the record.
"""
import numpy as np
import pytest

import imresh_b200 as imr
import oracle
from imresh_b200 import data
from imresh_b200.metrics import aligned_rel_l2

pytestmark = pytest.mark.gpu
FLT_MIN = imr.FLT_MIN


def _perturbed(M, seed, k=10):
    """M with k nonzero pixels moved up by one float ulp."""
    rng = np.random.default_rng(seed)
    Mp = M.copy()
    nz = np.flatnonzero(Mp)
    for i in rng.choice(nz, size=k, replace=False):
        Mp.flat[i] = np.nextafter(Mp.flat[i], np.float32(np.inf))
    return Mp


def _gpu(M, p: oracle.SwParams):
    H, W = M.shape
    io = M.reshape(-1).copy()
    rc = imr.cuda_shrink_wrap(io, W, H, 0, 0, 0, p.n_cycles, p.target_error, p.beta, p.cut_auto,
                              p.cut, p.sigma0, p.sigma_change, p.n_hio)
    assert rc == 0, imr.last_error()
    plan = imr.Plan(W, H, imr.Params(p.n_cycles, p.target_error, p.beta, p.cut_auto, p.cut,
                                     p.sigma0, p.sigma_change, p.n_hio))
    out = plan.execute_host(M)
    n, errs = plan.stats()
    plan.close()
    np.testing.assert_array_equal(out, io.reshape(H, W))   # drop-in == plan
    return out, errs


def _ref_or_restated(M, p):
    if oracle.ref_lib() is not None:
        return oracle.ref_shrinkwrap(M, p), "reference"
    return oracle.shrinkwrap(M, p).out, "restated"


def _report(name, rows):
    print(f"\n{name}")
    for k, v in rows.items():
        print(f"  {k:44s} {v}")


@pytest.fixture(scope="module")
def full_256(cuda):
    M, obj = data.make_modulus(data.cfg0_spec(), 0)
    p = oracle.SwParams(64, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 20)
    N = M.size
    gpu, gerr = _gpu(M, p)
    r32 = oracle.shrinkwrap(M, p)
    ref, kind = _ref_or_restated(M, p)
    r64 = oracle.shrinkwrap(M, p, fp64=True)
    pert = [oracle.shrinkwrap(_perturbed(M, s), p) for s in (1, 2)]
    return dict(M=M, obj=obj, N=N, gpu=gpu, gerr=gerr, r32=r32, ref=ref, kind=kind, r64=r64, pert=pert)


def test_full_256_restated_oracle_is_the_reference(full_256):
    if full_256["kind"] != "reference":
        pytest.skip("oracle/_ref not built")
    np.testing.assert_array_equal(full_256["r32"].out, full_256["ref"])


def test_full_256_error_curve_matches_the_ensemble(full_256):
    f = full_256
    g = f["gerr"]
    assert len(g) == 64
    members = [f["r32"].errors, f["r64"].errors] + [r.errors for r in f["pert"]]
    stats = lambda e: (float(np.median(e[32:])), float(np.mean(e[16:])), float(np.min(e)))
    ens = np.array([stats(e) for e in members])
    mean = ens.mean(axis=0)
    got = np.array(stats(g))
    _report("256x256, 64 x 20: HIO error statistics (median last 32, mean last 48, min)",
            {"gpu": np.round(got, 5), "ensemble mean": np.round(mean, 5),
             "ensemble members": np.round(ens, 5).tolist(),
             "cycle 0 error gpu / reference": (float(g[0]), float(f["r32"].errors[0]))})
    assert abs(g[0] - f["r32"].errors[0]) <= 0.02 * f["r32"].errors[0]
    assert np.all(np.abs(got - mean) <= 0.10 * mean), (got, mean)


def test_full_256_final_image_within_the_chaos_yardstick(full_256):
    f = full_256
    N = f["N"]
    gpu = f["gpu"] / N
    f64 = f["r64"].out / N
    ref = f["ref"] / N
    members = [f["r32"].out / N] + [r.out / N for r in f["pert"]]
    yard64 = max(aligned_rel_l2(m, f64) for m in members)
    yard32 = max(aligned_rel_l2(m, ref) for m in members[1:])
    d64 = aligned_rel_l2(gpu, f64)
    d32 = aligned_rel_l2(gpu, ref)
    objs = [aligned_rel_l2(m, f["obj"]) for m in members + [f64]]
    dobj = aligned_rel_l2(gpu, f["obj"])
    _report("256x256, 64 x 20: aligned relative L2",
            {"gpu vs fp64 / yardstick (fp32 members vs fp64)": (round(d64, 4), round(yard64, 4)),
             "gpu vs reference fp32 / yardstick": (round(d32, 4), round(yard32, 4)),
             "gpu vs object / ensemble max": (round(dobj, 4), round(max(objs), 4))})
    assert np.all(np.isfinite(gpu))
    assert d64 <= 1.2 * yard64
    assert d32 <= 1.2 * yard32
    assert dobj <= 1.15 * max(objs)


def test_2048_four_cycles_match_the_ensemble(cuda):
    """The restated FP32 oracle stands for the reference here: it equals the
    reference's shrinkWrap bit for bit (pinned above and in test_oracle.py)."""
    M, obj = data.make_modulus(data.cfg1_spec(), 1)
    p = oracle.SwParams(4, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 20)
    N = M.size
    gpu, gerr = _gpu(M, p)
    r32 = oracle.shrinkwrap(M, p)
    r64 = oracle.shrinkwrap(M, p, fp64=True)
    d64 = aligned_rel_l2(gpu / N, r64.out / N)
    yard = aligned_rel_l2(r32.out / N, r64.out / N)
    dobj = aligned_rel_l2(gpu / N, obj)
    objs = [aligned_rel_l2(r32.out / N, obj), aligned_rel_l2(r64.out / N, obj)]
    _report("2048x2048, 4 x 20",
            {"per-cycle error gpu": np.round(gerr, 5).tolist(),
             "per-cycle error fp32 / fp64": (np.round(r32.errors, 5).tolist(), np.round(r64.errors, 5).tolist()),
             "aligned gpu vs fp64 / fp32 vs fp64": (round(d64, 4), round(yard, 4)),
             "aligned gpu vs object / cpu max": (round(dobj, 4), round(max(objs), 4))})
    assert len(gerr) == 4
    np.testing.assert_allclose(gerr[:2], r32.errors[:2], rtol=0.01)
    np.testing.assert_allclose(gerr[2:], r32.errors[2:], rtol=0.05)
    np.testing.assert_allclose(gerr[2:], r64.errors[2:], rtol=0.05)
    assert d64 <= 1.2 * max(yard, 1.0)
    assert dobj <= 1.15 * max(objs)

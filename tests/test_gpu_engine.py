"""The batched / served engine through the C ABI: every reconstruction in a
mixed batch (uneven sizes, different cycle and HIO counts, admitted under a
memory budget) is bit-identical to the same reconstruction run alone; the
reference-API C++ program (cudaShrinkWrap + task queue) runs; the forward
model matches numpy."""
import subprocess

import numpy as np
import pytest

import imresh_b200 as imr
from imresh_b200 import data

pytestmark = pytest.mark.gpu
FLT_MIN = imr.FLT_MIN

MIX = [  # (W, H, cycles, hio)
    (128, 128, 3, 5), (192, 256, 2, 4), (256, 192, 4, 3), (384, 128, 2, 5), (512, 512, 3, 2),
    (96, 64, 3, 4), (256, 256, 1, 6), (128, 384, 2, 5), (160, 120, 2, 3), (64, 64, 5, 2),
    (100, 97, 2, 4), (131, 77, 2, 3), (97, 100, 3, 2),   # Bluestein widths / heights
]


def _inputs():
    out = []
    for i, (W, H, c, h) in enumerate(MIX):
        M, _ = data.make_modulus(data.BlobSpec(W, H, 10, 0.15 * min(W, H), (1.0, 3.0), (0.3, 1.0), 1e8),
                                 7, i)
        out.append((M, imr.Params(c, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, h)))
    return out


def _alone(M, p):
    H, W = M.shape
    plan = imr.Plan(W, H, p)
    out = plan.execute_host(M)
    n, errs = plan.stats()
    plan.close()
    return out, n


def test_mixed_batch_equals_alone(cuda):
    inputs = _inputs()
    eng = imr.Engine()
    for i, (M, p) in enumerate(inputs):
        eng.submit(M, p, tag=i)
    eng.run()
    res = {r["tag"]: r for r in eng.poll()}
    assert sorted(res) == list(range(len(inputs)))
    for i, (M, p) in enumerate(inputs):
        r = res[i]
        assert r["status"] == 0
        alone, n = _alone(M, p)
        assert r["cycles_done"] == n == p.n_cycles
        np.testing.assert_array_equal(r["out"], alone)
    info = eng.info()
    assert info["active"] == 0 and info["pending"] == 0
    eng.close()


def test_half_tile_column_pass(cuda):
    """A plan whose column tiles fill at most half of the resident CTAs runs each
    tile as two half tiles (two threads per 16-value column sequence, one parity
    each); the engine runs the same jobs as whole tiles.  Both give the same bits,
    also where a half tile lies partly or wholly past the image's width (260 x 256
    and 200 x 512: the last tile's second half is outside the image)."""
    shapes = [(256, 256), (512, 512), (260, 256), (200, 512), (128, 128), (512, 256)]
    inputs = []
    for i, (W, H) in enumerate(shapes):
        M, _ = data.make_modulus(data.BlobSpec(W, H, 12, 0.15 * min(W, H), (1.0, 3.0), (0.3, 1.0), 1e8), 9, i)
        inputs.append((M, imr.Params(3, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 4)))
    eng = imr.Engine()
    for i, (M, p) in enumerate(inputs):
        eng.submit(M, p, tag=i)
    eng.run()
    res = {r["tag"]: r for r in eng.poll()}
    eng.close()
    for i, (M, p) in enumerate(inputs):
        alone, n = _alone(M, p)
        assert res[i]["status"] == 0 and n == p.n_cycles
        np.testing.assert_array_equal(res[i]["out"], alone, err_msg=str(shapes[i]))


def test_submit_intensity_equals_modulus(cuda):
    """A request submitted as a measured intensity I gives the bits of the same
    request submitted as the modulus sqrtf(I) (the engine takes the square root
    at admission), alone and beside modulus requests."""
    inputs = _inputs()[:6]
    eng = imr.Engine()
    for i, (M, p) in enumerate(inputs):
        eng.submit(M, p, tag=i)
        I = (M.astype(np.float64) ** 2).astype(np.float32)
        eng.submit(I, p, tag=100 + i, intensity=True)
    eng.run()
    res = {r["tag"]: r for r in eng.poll()}
    eng.close()
    for i, (M, p) in enumerate(inputs):
        I = (M.astype(np.float64) ** 2).astype(np.float32)
        want = np.sqrt(I)   # float32, correctly rounded
        alone, _ = _alone(want, p)
        assert res[100 + i]["status"] == 0
        np.testing.assert_array_equal(res[100 + i]["out"], alone)
        if np.array_equal(want, M):
            np.testing.assert_array_equal(res[100 + i]["out"], res[i]["out"])


def test_several_cycles_per_step(cuda):
    """Four cycles per step graph: the same bits as one request alone, about a
    quarter of the steps, and no step queued after the last request's final
    cycle (the engine waits for that step's state instead)."""
    inputs = _inputs()
    eng = imr.Engine()
    eng.set_cycles_per_step(4)
    for i, (M, p) in enumerate(inputs):
        eng.submit(M, p, tag=i)
    eng.run()
    res = {r["tag"]: r for r in eng.poll()}
    info = eng.info()
    eng.close()
    assert info["cycles_per_step"] == 4
    longest = max(p.n_cycles for _, p in inputs) + 1
    assert info["steps"] <= (longest + 3) // 4 + 1, info
    assert sorted(res) == list(range(len(inputs)))
    for i, (M, p) in enumerate(inputs):
        alone, n = _alone(M, p)
        assert res[i]["status"] == 0 and res[i]["cycles_done"] == n == p.n_cycles
        np.testing.assert_array_equal(res[i]["out"], alone)


def test_admission_under_memory_budget(cuda):
    inputs = [(data.make_modulus(data.BlobSpec(256, 256, 10, 38.0, (1.5, 2.5), (0.5, 1.0), None), 9, i)[0],
               imr.Params(2, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 3)) for i in range(6)]
    per_job = 33 * 256 * 256
    eng = imr.Engine(device_bytes=int(2.5 * per_job))
    for i, (M, p) in enumerate(inputs):
        eng.submit(M, p, tag=i)
    steps = 0
    while True:
        info = eng.info()
        if info["pending"] == 0 and info["active"] == 0:
            break
        assert info["resident"] <= 2
        eng.step()
        steps += 1
    res = {r["tag"]: r for r in eng.poll()}
    assert len(res) == 6 and steps >= 9
    assert eng.info()["device_bytes_peak"] <= int(2.5 * per_job)
    for i, (M, p) in enumerate(inputs):
        np.testing.assert_array_equal(res[i]["out"], _alone(M, p)[0])
    eng.close()


def test_late_arrivals_join_running_batch(cuda):
    """Requests submitted while others are mid-run are admitted at the next
    step and still produce their stand-alone result."""
    inputs = _inputs()[:6]
    eng = imr.Engine()
    for i, (M, p) in enumerate(inputs[:3]):
        eng.submit(M, p, tag=i)
    eng.step()
    eng.step()
    for i, (M, p) in enumerate(inputs[3:], start=3):
        eng.submit(M, p, tag=i)
    eng.run()
    res = {r["tag"]: r for r in eng.poll()}
    for i, (M, p) in enumerate(inputs):
        np.testing.assert_array_equal(res[i]["out"], _alone(M, p)[0])
    eng.close()


def test_diffraction_intensity_matches_numpy(cuda):
    rng = np.random.default_rng(3)
    obj = rng.random((192, 256)).astype(np.float32)
    got = imr.diffraction_intensity(obj)
    ref = np.abs(np.fft.fft2(obj.astype(np.float64)))
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5


def test_reference_api_cpp_program_runs(cuda, tmp_path):
    from tests.cpp_build import build_drop_in
    exe = build_drop_in(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout


def test_suspend_resume_is_bit_identical(cuda):
    """A reconstruction saved between steps, removed, and resumed in another
    engine finishes exactly as it would have uninterrupted; the engine it left
    finishes its other work unchanged."""
    p = imr.Params(6, imr.FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 5)
    Ma, _ = data.make_modulus(data.BlobSpec(256, 192, 20, 30.0, (1.5, 2.5), (0.5, 1.0), 1e8), 7, 0)
    Mb, _ = data.make_modulus(data.BlobSpec(128, 128, 12, 20.0, (1.5, 2.5), (0.5, 1.0), None), 7, 1)
    ref = imr.Engine()
    ra, rb = ref.submit(Ma, p, tag=1), ref.submit(Mb, p, tag=2)
    ref.run()
    cyc = {r["tag"]: r["cycles_done"] for r in ref.poll()}
    ref.close()

    E = imr.Engine()
    E.submit(Ma, p, tag=1)
    ob = E.submit(Mb, p, tag=2)
    E.step()
    E.step()
    snap = E.suspend(1)
    assert E.info()["active"] == 1
    E.step()
    E2 = imr.Engine()
    oa = E2.resume(snap)
    E2.run()
    E.run()
    res2 = E2.poll()
    assert [r["tag"] for r in res2] == [1] and res2[0]["cycles_done"] == cyc[1]
    np.testing.assert_array_equal(oa, ra)
    np.testing.assert_array_equal(ob, rb)
    assert [r["tag"] for r in E.poll()] == [2]
    E.close()
    E2.close()


def test_checkpoint_keeps_running_and_restarts_identically(cuda):
    p = imr.Params(5, imr.FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 4)
    M, _ = data.make_modulus(data.BlobSpec(192, 256, 16, 30.0, (1.5, 2.5), (0.5, 1.0), 1e8), 9, 0)
    ref = imr.Engine()
    r = ref.submit(M, p, tag=5)
    ref.run()
    ref.close()
    E = imr.Engine()
    o = E.submit(M, p, tag=5)
    E.step()
    cp = E.checkpoint(5)
    E.run()
    np.testing.assert_array_equal(o, r)
    E2 = imr.Engine()
    o2 = E2.resume(cp)
    E2.run()
    np.testing.assert_array_equal(o2, r)
    E.close()
    E2.close()


def test_snapshot_rejects_unknown_tags_and_bad_buffers(cuda):
    E = imr.Engine()
    with pytest.raises(imr.ImrError):
        E.checkpoint(99)
    with pytest.raises(imr.ImrError):
        E.resume(b"IMRSNAP1" + bytes(200))
    E.close()


def test_chained_schedule_equals_grouped(cuda):
    """The chained step graph (one branch per kernel class) gives the same
    bits as the grouped one and as each reconstruction alone."""
    inputs = _inputs()
    outs = {}
    for sched in (imr.SCHEDULE_GROUPED, imr.SCHEDULE_CHAINED):
        eng = imr.Engine()
        eng.set_schedule(sched)
        for i, (M, p) in enumerate(inputs):
            eng.submit(M, p, tag=i)
        eng.step()
        eng.run()
        outs[sched] = {r["tag"]: r["out"] for r in eng.poll()}
        eng.close()
    for i, (M, p) in enumerate(inputs):
        np.testing.assert_array_equal(outs[imr.SCHEDULE_CHAINED][i], outs[imr.SCHEDULE_GROUPED][i])
        np.testing.assert_array_equal(outs[imr.SCHEDULE_CHAINED][i], _alone(M, p)[0])


@pytest.mark.parametrize("name", ["miniExample", "threadedExample"])
def test_reference_examples_run_unchanged(cuda, tmp_path, name):
    """The reference's own callers, examples/miniExample.cpp (cudaShrinkWrap on
    a 600x300 atom cluster, 64 cycles) and examples/threadedExample.cpp (task
    queue init / diffractionIntensity / deinit), compiled unmodified from the
    reference's tree against include/imresh and linked with libimresh_b200.so
    (oracle/Makefile, target examples), run to completion."""
    import oracle
    exe = oracle.example(name)
    if exe is None:
        pytest.skip("reference examples not built (oracle/Makefile examples)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr


def test_autotuner_explores_once_then_uses_its_cache(cuda, tmp_path):
    """The engine's tuner runs each candidate step configuration (two
    schedules x two persistent-grid sizes) for two steps of a new admitted
    set, times the second, keeps the fastest, and writes it to its cache file; a second engine
    with the same cache and the same set starts with that configuration and
    explores nothing.  Every configuration gives the same bits."""
    p = imr.Params(14, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 4)
    shapes = [(128, 128), (256, 192), (192, 256), (256, 256), (128, 384), (384, 128)]
    inputs = [data.make_modulus(data.BlobSpec(W, H, 10, 0.15 * min(W, H), (1.0, 3.0), (0.3, 1.0), 1e8), 13, i)[0]
              for i, (W, H) in enumerate(shapes)]
    cache = str(tmp_path / "tune.txt")
    runs = []
    for attempt in range(2):
        eng = imr.Engine()
        eng.set_autotune(True, cache)
        for i, M in enumerate(inputs):
            eng.submit(M, p, tag=i)
        eng.run()
        res = {r["tag"]: r["out"] for r in eng.poll()}
        runs.append((res, eng.info()))
        eng.close()
    (res0, info0), (res1, info1) = runs
    assert info0["tune_explored"] == 8 and info0["tune_cache_hits"] == 0, info0   # 4 candidates x 2 steps
    assert info1["tune_explored"] == 0 and info1["tune_cache_hits"] == 1, info1
    assert (info1["schedule"], info1["grid_pct"]) == (info0["schedule"], info0["grid_pct"])
    lines = open(cache).read().strip().splitlines()
    assert len(lines) == 1 and "\t" in lines[0]
    for i, M in enumerate(inputs):
        alone = _alone(M, p)[0]
        np.testing.assert_array_equal(res0[i], alone)
        np.testing.assert_array_equal(res1[i], alone)


def test_admission_bounds_keep_results_and_the_bound(cuda):
    """A pixel bound admits requests only while the resident pixels stay
    within it (or one request when nothing runs); a step-time target admits
    by the measured cost per pixel.  Neither changes any result."""
    inputs = _inputs()[:8]
    bound = 256 * 256 + 192 * 256
    eng = imr.Engine()
    eng.set_admission(bound)
    for i, (M, p) in enumerate(inputs):
        eng.submit(M, p, tag=i)
    peak = 0
    while True:
        info = eng.info()
        if info["pending"] == 0 and info["active"] == 0:
            break
        assert info["resident_px"] <= bound or info["resident"] == 1, info
        peak = max(peak, info["resident_px"])
        eng.step()
    res = {r["tag"]: r for r in eng.poll()}
    eng.close()
    assert len(res) == len(inputs) and peak > 0
    eng = imr.Engine()
    eng.set_schedule(imr.SCHEDULE_CHAINED)
    eng.set_step_target(2.0)
    for i, (M, p) in enumerate(inputs):
        eng.submit(M, p, tag=i)
    eng.run()
    res2 = {r["tag"]: r for r in eng.poll()}
    assert eng.info()["ms_per_mpx"] > 0
    eng.close()
    for i, (M, p) in enumerate(inputs):
        alone = _alone(M, p)[0]
        np.testing.assert_array_equal(res[i]["out"], alone)
        np.testing.assert_array_equal(res2[i]["out"], alone)


def test_chained_schedule_with_more_classes_than_branch_streams(cuda):
    """More (row kernel, column kernel) classes than the graph's 16 branch
    streams: chains share streams in turn and every result still equals the
    reconstruction alone."""
    # widths and heights of distinct kernel classes: powers of two and 3*2^k,
    # a runtime-radix length (100) and Bluestein lengths of three work sizes
    shapes = [(W, H) for W in (64, 128, 192, 97, 131) for H in (64, 256, 100, 263)]
    p = imr.Params(2, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 3)
    inputs = [data.make_modulus(data.BlobSpec(W, H, 6, 0.15 * min(W, H), (1.0, 2.0), (0.3, 1.0), 1e8), 17, i)[0]
              for i, (W, H) in enumerate(shapes)]
    eng = imr.Engine()
    eng.set_schedule(imr.SCHEDULE_CHAINED)
    for i, M in enumerate(inputs):
        eng.submit(M, p, tag=i)
    eng.step()
    assert eng.info()["kernels_per_step"] >= 17 * (2 + 2 * 3)
    eng.run()
    res = {r["tag"]: r["out"] for r in eng.poll()}
    eng.close()
    for i, M in enumerate(inputs):
        np.testing.assert_array_equal(res[i], _alone(M, p)[0])

"""Failure handling through the C ABI, in the forms that fault, trap or hang
no GPU.  The reference prints and exits the process on any CUDA error
(src/imresh/libs/cudacommon.cu:39-56) and on an oversized kernel
(src/imresh/algorithms/cuda/cudaGaussian.cu:288-293); here every failure is a
status code and the context stays usable:

* device side: every copy wait of the pipelined passes is bounded; a wait
  on a barrier that nothing completes gives up after its limit and reports
  IMR_ERR_DEVICE_TIMEOUT (no trap, no fault); a plan's per-launch limit is
  plumbed to its passes, and a pass that gave up still lets its copies in
  flight land before it returns;
* host side: the engine's device allocations are made to fail on purpose
  (a fake of the failing call), and requests are cancelled between steps.
"""
import ctypes as C

import numpy as np
import pytest

import imresh_b200 as imr
from imresh_b200 import data

pytestmark = pytest.mark.gpu
FLT_MIN = imr.FLT_MIN


def _sigs():
    L = imr.lib()
    L.imr_bounded_wait_check.argtypes = [C.c_ulonglong, C.POINTER(C.c_ulonglong), C.c_void_p]
    L.imr_plan_set_wait_limit.argtypes = [C.c_void_p, C.c_ulonglong]
    return L


def _modulus(W, H, k=0, photons=None):
    return data.make_modulus(data.BlobSpec(W, H, 12, 0.15 * min(W, H), (1.5, 2.5), (0.5, 1.0), photons), 21, k)[0]


def _alone(M, p):
    H, W = M.shape
    plan = imr.Plan(W, H, p)
    out = plan.execute_host(M)
    plan.close()
    return out


def test_bounded_wait_gives_up_and_the_context_survives(cuda):
    L = _sigs()
    for limit in (1_000_000, 20_000_000):   # 1 ms, 20 ms
        t = C.c_ulonglong()
        rc = L.imr_bounded_wait_check(limit, C.byref(t), None)
        assert rc == 7, rc   # IMR_ERR_DEVICE_TIMEOUT
        assert limit <= t.value < limit + 200_000_000, t.value
        assert "gave up" in imr.last_error()
    # the context is still usable: a reconstruction runs and is deterministic
    M = _modulus(128, 96)
    p = imr.Params(2, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 3)
    np.testing.assert_array_equal(_alone(M, p), _alone(M, p))


def test_plan_wait_limit_reaches_the_passes(cuda):
    """A generous per-launch limit changes nothing; a limit far below a copy's
    latency (1 ns) may make waits give up -- then the plan reports
    IMR_ERR_DEVICE_TIMEOUT instead of a result -- and never faults; the
    default limit afterwards restores the exact result."""
    L = _sigs()
    M = _modulus(1024, 1024, photons=1e9)
    p = imr.Params(2, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 4)
    plan = imr.Plan(1024, 1024, p)
    want = plan.execute_host(M)
    assert L.imr_plan_set_wait_limit(plan._h, 50_000_000) == 0
    np.testing.assert_array_equal(plan.execute_host(M), want)
    assert plan.stats()[0] == 2
    assert L.imr_plan_set_wait_limit(plan._h, 1) == 0
    plan.execute_host(M)
    n = C.c_int()
    rc = imr.lib().imr_plan_stats(plan._h, None, C.byref(n), None)
    assert rc in (0, 7), rc
    if rc == 7:
        assert "timed out" in imr.last_error()
    assert L.imr_plan_set_wait_limit(plan._h, 0) == 0
    np.testing.assert_array_equal(plan.execute_host(M), want)
    assert plan.stats()[0] == 2
    plan.close()


def test_failed_allocation_is_retried_while_others_run(cuda):
    p = imr.Params(3, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 3)
    Ms = [_modulus(128, 128, k) for k in range(3)]
    E = imr.Engine()
    E.submit(Ms[0], p, tag=0)
    E.step()                        # request 0 admitted and running
    E.inject_alloc_failures(2)
    E.submit(Ms[1], p, tag=1)
    E.submit(Ms[2], p, tag=2)
    E.run()
    res = {r["tag"]: r for r in E.poll()}
    assert sorted(res) == [0, 1, 2]
    assert E.info()["alloc_failures"] == 2
    for k in range(3):
        assert res[k]["status"] == 0
        np.testing.assert_array_equal(res[k]["out"], _alone(Ms[k], p))
    E.close()


def test_failed_allocation_with_nothing_running_is_reported(cuda):
    p = imr.Params(2, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 2)
    E = imr.Engine()
    E.inject_alloc_failures(1)
    E.submit(_modulus(64, 64), p, tag=7)
    E.run()                         # returns: the request cannot be served
    (r,) = E.poll()
    assert r["tag"] == 7 and r["status"] == 3   # IMR_ERR_OUT_OF_MEMORY
    # the engine keeps serving
    M = _modulus(64, 64, 1)
    E.submit(M, p, tag=8)
    E.run()
    (r,) = E.poll()
    assert r["status"] == 0
    np.testing.assert_array_equal(r["out"], _alone(M, p))
    E.close()


def test_cancel_pending_and_running_requests(cuda):
    p = imr.Params(6, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 3)
    Ms = [_modulus(192, 128, k) for k in range(3)]
    E = imr.Engine(device_bytes=1)   # one request resident at a time
    outs = [E.submit(M, p, tag=k) for k, M in enumerate(Ms)]
    for o in outs:
        o.fill(-7.0)
    E.step()
    E.step()
    E.cancel(0)                     # running
    E.cancel(2)                     # pending
    with pytest.raises(imr.ImrError):
        E.cancel(99)
    E.run()
    res = {r["tag"]: r for r in E.poll()}
    assert res[0]["status"] == 8 and res[2]["status"] == 8
    assert np.all(outs[0] == -7.0) and np.all(outs[2] == -7.0)
    assert res[1]["status"] == 0
    np.testing.assert_array_equal(res[1]["out"], _alone(Ms[1], p))
    assert E.info()["resident"] == 0
    E.close()


def test_engine_step_is_one_graph_launch(cuda):
    """Once the active set is fixed, a step is one host launch of the
    captured step graph (plus the column init of newly admitted requests);
    the graph is captured once for the set, not per step."""
    p = imr.Params(6, FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 5)
    shapes = [(128, 128), (192, 256), (256, 192), (384, 128), (512, 512), (128, 384)]
    Ms = [_modulus(W, H, k) for k, (W, H) in enumerate(shapes)]
    E = imr.Engine()
    for k, M in enumerate(Ms):
        E.submit(M, p, tag=k)
    E.run()
    info = E.info()
    res = {r["tag"]: r for r in E.poll()}
    assert len(res) == len(Ms)
    builds = info["graph_builds"] + info["graph_updates"]
    assert builds <= 3, info                      # the set, then its retirement
    direct = info["host_launches"] - info["steps"]
    assert direct <= 2 * len(Ms), info            # column init and modulus tiles only
    assert info["kernels_per_step"] >= 10 * info["host_launches"] / info["steps"], info
    for k, M in enumerate(Ms):
        np.testing.assert_array_equal(res[k]["out"], _alone(M, p))
    E.close()

"""imr_shrink_wrap_noalloc: the reconstruction entry point that allocates no
device memory, for callers that cannot call cudaMalloc -- code whose device
memory belongs to a fixed arena or a framework's allocator, loops that must
not take the driver's allocation locks, processes that reserve all device
memory up front.  Its working memory is a static array inside the library
(at most 512*512 pixels), so the caller only passes the modulus and the
output buffer.

Checked through the C ABI against the existing entry point (the plan API,
same kernels), on two calls in a row that reuse the shared array: the second
call must not see the first one's state.  Runs alone in a fresh process and
after the rest of the suite (this file is collected last).
"""
import ctypes as C

import numpy as np
import pytest

import imresh_b200 as imr
from imresh_b200 import data

pytestmark = pytest.mark.gpu


def _noalloc():
    L = imr.lib()
    f = L.imr_shrink_wrap_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint, C.c_uint, C.POINTER(imr.CParams), C.c_void_p]
    f.restype = C.c_int
    return f


def _existing(M, p):
    H, W = M.shape
    plan = imr.Plan(W, H, p)
    out = plan.execute_host(M)
    plan.close()
    return out


CASES = [  # (W, H, params): a square pipelined size, then a rectangular one
    (256, 256, imr.Params(3, imr.FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 5)),
    (384, 128, imr.Params(2, imr.FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 4)),
]


def test_noalloc_matches_existing_entry_point_twice_in_a_row(cuda):
    import torch
    f = _noalloc()
    stream = torch.cuda.current_stream().cuda_stream
    for k, (W, H, p) in enumerate(CASES):
        M, _ = data.make_modulus(data.BlobSpec(W, H, 12, 0.15 * min(W, H), (1.5, 2.5), (0.5, 1.0), None), 11, k)
        d_m = torch.from_numpy(M).cuda()
        d_o = torch.full_like(d_m, float("nan"))
        cp = p.c()
        rc = f(d_m.data_ptr(), d_o.data_ptr(), W, H, C.byref(cp), stream)
        assert rc == 0, imr.last_error()
        torch.cuda.synchronize()
        got = d_o.cpu().numpy()
        ref = _existing(M, p)
        # same kernels as the plan path: identical up to the tests' 1e-5 tolerance
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-5 * float(np.abs(ref).max()))


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    f = _noalloc()
    d = torch.zeros(1024 * 1024, device="cuda")
    cp = imr.Params().c()
    rc = f(d.data_ptr(), d.data_ptr(), 1024, 1024, C.byref(cp), torch.cuda.current_stream().cuda_stream)
    assert rc == 2
    assert "exceeds the static scratch" in imr.last_error()

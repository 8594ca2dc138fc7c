"""imr_shrink_wrap_noalloc: the reconstruction entry point that allocates no
device memory, for callers that cannot call cudaMalloc -- code whose device
memory belongs to a fixed arena or a framework's allocator, loops that must
not take the driver's allocation locks, processes that reserve all device
memory up front.  Its working memory is a static array inside the library
(at most 512*512 pixels), so the caller only passes the modulus and the
output buffer.

Checked through the C ABI against the existing entry point (the plan API),
on two calls in a row that reuse the shared array: the second call must not
see the first one's state.  Both entry points do the same arithmetic in the
same order over the same data (the modulus copied, its column tiles built;
a plan may run a column tile as two half tiles, which compute the same
operations), so the results must be bit-identical: a tolerance would hide an
ordering difference.  Runs alone in a fresh process and after
the rest of the suite (this file is collected last).
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


def _noalloc_stats(stream):
    L = imr.lib()
    f = L.imr_shrink_wrap_noalloc_stats
    f.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_void_p, C.c_int]
    f.restype = C.c_int
    n = C.c_int(-1)
    errs = np.zeros(64, np.float32)
    rc = f(stream, C.byref(n), errs.ctypes.data, errs.size)
    return rc, n.value, errs


def _existing(M, p):
    H, W = M.shape
    plan = imr.Plan(W, H, p)
    out = plan.execute_host(M)
    n, errs = plan.stats()
    plan.close()
    return out, n, errs


CASES = [  # (W, H, params, in place)
    # a square size on the pipelined column pass with the column-tiled modulus
    (256, 256, imr.Params(3, imr.FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 5), False),
    # rectangular, modulus and output in one buffer (the reference works in place)
    (384, 128, imr.Params(2, imr.FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 4), True),
    # a width that is not a multiple of 4: the per-tile column pass, runtime-length rows
    (90, 60, imr.Params(2, imr.FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 3), False),
]


@pytest.mark.parametrize("repeat", [0, 1])
def test_noalloc_matches_existing_entry_point_twice_in_a_row(cuda, repeat):
    import torch
    f = _noalloc()
    stream = torch.cuda.current_stream().cuda_stream
    for k, (W, H, p, in_place) in enumerate(CASES):
        M, _ = data.make_modulus(data.BlobSpec(W, H, 12, 0.15 * min(W, H), (1.5, 2.5), (0.5, 1.0), None), 11, k)
        d_m = torch.from_numpy(M).cuda()
        d_o = d_m if in_place else torch.full_like(d_m, float("nan"))
        cp = p.c()
        rc = f(d_m.data_ptr(), d_o.data_ptr(), W, H, C.byref(cp), stream)
        assert rc == 0, imr.last_error()
        rc, n, errs = _noalloc_stats(stream)
        assert rc == 0, imr.last_error()
        got = d_o.cpu().numpy()
        ref, n_ref, errs_ref = _existing(M, p)
        np.testing.assert_array_equal(got, ref)
        assert n == n_ref == p.n_cycles
        np.testing.assert_array_equal(errs[:n], errs_ref[:n])


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    f = _noalloc()
    stream = torch.cuda.current_stream().cuda_stream
    d = torch.zeros(1024 * 1024, device="cuda")
    cp = imr.Params().c()
    rc = f(d.data_ptr(), d.data_ptr(), 1024, 1024, C.byref(cp), stream)
    assert rc == 2
    assert "exceeds the static scratch" in imr.last_error()
    # a side with a prime factor above 7 (Bluestein's transform needs allocated tables)
    rc = f(d.data_ptr(), d.data_ptr(), 257, 64, C.byref(cp), stream)
    assert rc == 2
    assert "2^a 3^b 5^c 7^d" in imr.last_error()
    cp = imr.Params(2000).c()
    rc = f(d.data_ptr(), d.data_ptr(), 64, 64, C.byref(cp), stream)
    assert rc == 1
    assert "at most 1024 cycles" in imr.last_error()

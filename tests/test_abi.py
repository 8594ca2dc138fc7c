"""CPU-only checks of the drop-in boundary: the C-ABI library loads without a
GPU, exports every function include/imresh_b200.h declares, and its host-side
logic (status strings, supported lengths, Gaussian weights, parameter
validation that needs no device) behaves as documented."""
import ctypes as C
import os

import numpy as np
import pytest

import imresh_b200 as imr
import oracle


def test_library_exports_every_declared_symbol():
    L = imr.lib()
    names = imr.header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings():
    assert imr.status_string(0) == "success"
    assert imr.status_string(2) == "unsupported image size"
    assert imr.status_string(999) == "unknown status"


@pytest.mark.parametrize("n,ok", [(1, True), (2, True), (64, True), (192, True), (210, True),
                                  (343, True), (4096, True), (3072, True), (2187, False), (2400, False),
                                  (2048, True), (4097, False), (11, True), (1031, True), (2039, True),
                                  (0, False), (8192, False), (2049, False)])
def test_side_supported(n, ok):
    assert imr.side_supported(n) == ok
    assert imr.lib().imr_max_side() == 4096


@pytest.mark.parametrize("sigma", [0.1, 0.5, 1.0, 1.5, 2.2, 3.0, 4.0, 7.5])
def test_gaussian_weights_match_oracle(sigma):
    np.testing.assert_array_equal(imr.gaussian_weights(sigma), oracle.gaussian_weights(sigma))


def test_invalid_arguments_rejected_without_device():
    L = imr.lib()
    buf = np.zeros(16, np.float32)
    assert L.imr_cuda_shrink_wrap(None, 4, 4, None, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0) == 1
    assert L.imr_cuda_shrink_wrap(buf.ctypes.data, 0, 4, None, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0) == 1
    assert L.imr_fft2d(None, 4, 4, -1, None) == 1
    assert L.imr_fft2d(buf.ctypes.data, 4, 4, 0, None) == 1
    assert L.imr_gaussian_blur(None, None, 4, 4, 1.0, 3, None) == 1
    h = C.c_void_p()
    assert L.imr_plan_create(C.byref(h), 0, 4, None) == 1
    assert L.imr_plan_destroy(None) == 0
    assert L.imr_engine_resume(None, buf.ctypes.data, 64, buf.ctypes.data) == 1
    assert L.imr_engine_checkpoint(None, 0, buf.ctypes.data, 64) == 1


def test_cpp_drop_in_compiles_and_links(tmp_path):
    """A caller written against the reference's C++ API (header paths,
    namespaces, default arguments) builds and links against the library."""
    from tests.cpp_build import build_drop_in
    exe = build_drop_in(str(tmp_path))
    assert os.path.exists(exe)


def test_reference_symbols_exported():
    import subprocess
    out = subprocess.run(["nm", "-DC", imr.LIB_PATH], capture_output=True, text=True).stdout
    for sym in ("imresh::algorithms::cuda::cudaShrinkWrap(", "imresh::io::taskQueueInit()",
                "imresh::io::taskQueueDeinit()", "imresh::io::addTask(",
                "imresh::io::writeOutFuncs::justFree(", "imresh::libs::diffractionIntensity(",
                "imresh::libs::hybridInputOutput(", "imresh::io::readInFuncs::readTxt(",
                "imresh::io::readInFuncs::readNpy(", "imresh::io::writeOutFuncs::writeOutNpy(",
                "imresh::io::writeOutFuncs::writeOutAndFreeNpy(", "imresh::io::writeOutFuncs::writeOutTxt(",
                "imresh::io::writeOutFuncs::writeOutRaw("):
        assert sym in out, sym

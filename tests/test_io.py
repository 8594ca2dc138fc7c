"""Image files behind the task queue's read-in / write-out callbacks
(readInFuncs / writeOutFuncs, src/imresh/io/readInFuncs/readInFuncs.hpp:57-84,
src/imresh/io/writeOutFuncs/writeOutFuncs.hpp:52-106), through the C ABI,
checked against numpy's own readers and writers.  Host code only."""
import ctypes as C
import os

import numpy as np
import pytest

import imresh_b200 as imr


def _lib():
    L = imr.lib()
    cp, fp, u = C.c_char_p, C.c_void_p, C.c_uint
    for fn in ("imr_write_npy", "imr_write_txt", "imr_write_raw"):
        getattr(L, fn).argtypes = [cp, fp, u, u]
    for fn in ("imr_read_npy", "imr_read_txt"):
        getattr(L, fn).argtypes = [cp, C.POINTER(C.POINTER(C.c_float)), C.POINTER(u), C.POINTER(u)]
    L.imr_free_image.argtypes = [C.POINTER(C.c_float)]
    return L


def _read(fn, path):
    L = _lib()
    d, w, h = C.POINTER(C.c_float)(), C.c_uint(), C.c_uint()
    rc = getattr(L, fn)(str(path).encode(), C.byref(d), C.byref(w), C.byref(h))
    if rc != 0:
        return rc, None
    a = np.ctypeslib.as_array(d, shape=(h.value, w.value)).copy()
    L.imr_free_image(d)
    return rc, a


def _img(h, w, seed=0):
    return (np.random.default_rng(seed).standard_normal((h, w)) * 1e3).astype(np.float32)


@pytest.mark.parametrize("shape", [(1, 1), (3, 5), (96, 256), (257, 31)])
def test_npy_write_is_read_by_numpy(tmp_path, shape):
    a = _img(*shape)
    p = tmp_path / "a.npy"
    assert _lib().imr_write_npy(str(p).encode(), a.ctypes.data, shape[1], shape[0]) == 0
    b = np.load(p)
    assert b.dtype == np.float32 and b.shape == shape
    np.testing.assert_array_equal(a, b)
    assert (10 + int.from_bytes(open(p, "rb").read()[8:10], "little")) % 64 == 0   # aligned header


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape", [(7,), (4, 9), (128, 64)])
def test_npy_from_numpy_is_read(tmp_path, dtype, shape):
    a = np.random.default_rng(1).standard_normal(shape).astype(dtype)
    p = tmp_path / "b.npy"
    np.save(p, a)
    rc, b = _read("imr_read_npy", p)
    assert rc == 0
    np.testing.assert_array_equal(b, a.astype(np.float32).reshape(b.shape))
    assert b.shape == (shape if len(shape) == 2 else (1, shape[0]))


def test_npy_rejects_what_it_cannot_read(tmp_path):
    p = tmp_path / "f.npy"
    np.save(p, np.asfortranarray(np.ones((3, 4), np.float32)))
    assert _read("imr_read_npy", p)[0] == 1
    np.save(p, np.ones((2, 3, 4), np.float32))
    assert _read("imr_read_npy", p)[0] == 1
    np.save(p, np.ones((3, 4), np.int32))
    assert _read("imr_read_npy", p)[0] == 1
    p.write_bytes(b"not an array")
    assert _read("imr_read_npy", p)[0] == 1
    assert _read("imr_read_npy", tmp_path / "missing.npy")[0] == 1


@pytest.mark.parametrize("shape", [(1, 1), (2, 3), (40, 17)])
def test_txt_round_trip_is_exact(tmp_path, shape):
    a = _img(*shape, seed=2)
    p = tmp_path / "a.txt"
    assert _lib().imr_write_txt(str(p).encode(), a.ctypes.data, shape[1], shape[0]) == 0
    np.testing.assert_array_equal(np.loadtxt(p, dtype=np.float32, ndmin=2), a)
    rc, b = _read("imr_read_txt", p)
    assert rc == 0
    np.testing.assert_array_equal(b, a)


def test_txt_reads_rows_per_line(tmp_path):
    """The reference's readTxt counts a row's values from its first line
    (readInFuncs.cpp:55-70); here every line is one image row."""
    p = tmp_path / "r.txt"
    p.write_text("1 2 3\n\n4\t5   6\n7 8 9.5e1\n")
    rc, b = _read("imr_read_txt", p)
    assert rc == 0
    np.testing.assert_array_equal(b, np.array([[1, 2, 3], [4, 5, 6], [7, 8, 95]], np.float32))
    p.write_text("1 2 3\n4 5\n")
    assert _read("imr_read_txt", p)[0] == 1
    p.write_text("1 x 3\n")
    assert _read("imr_read_txt", p)[0] == 1
    p.write_text("")
    assert _read("imr_read_txt", p)[0] == 1


def test_raw_is_float32_width_contiguous(tmp_path):
    a = _img(12, 20, seed=3)
    p = tmp_path / "a.f32"
    assert _lib().imr_write_raw(str(p).encode(), a.ctypes.data, 20, 12) == 0
    np.testing.assert_array_equal(np.fromfile(p, np.float32).reshape(12, 20), a)
    assert os.path.getsize(p) == a.nbytes


def test_writers_reject_bad_arguments(tmp_path):
    L = _lib()
    a = np.zeros(4, np.float32)
    assert L.imr_write_npy(None, a.ctypes.data, 2, 2) == 1
    assert L.imr_write_txt(str(tmp_path / "x").encode(), None, 2, 2) == 1
    assert L.imr_write_raw(str(tmp_path / "x").encode(), a.ctypes.data, 0, 2) == 1
    assert L.imr_write_npy(str(tmp_path / "no" / "dir.npy").encode(), a.ctypes.data, 2, 2) == 1

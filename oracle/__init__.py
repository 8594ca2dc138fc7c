"""ORACLE / TEST INFRASTRUCTURE -- not part of the product.

ctypes front end to two CPU libraries:

* ``liboracle.so`` -- this project's C restatement of the reference's CPU
  shrink-wrap path and of its fixed-support random-phase HIO (float and FP64)
  over the project-written FFT (``shrinkwrap_oracle.c``, ``hio_oracle.c``,
  ``imro_fft.c``);
* ``_ref/libimresh_ref.so`` -- the reference's own CPU ``shrinkWrap`` and the
  functions it calls, compiled unmodified from its sources over the FFTW shim
  (``Makefile`` target ``ref``; present only where it was built).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker or as the timed
CPU baseline.  The product (``imresh_b200``) never calls into it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def reference_tree() -> str:
    """The reference project's source tree: $IMRESH_REF, else the directory
    ``reference`` beside this repository."""
    return os.environ.get("IMRESH_REF") or os.path.normpath(os.path.join(_HERE, "..", "..", "reference"))


def build(ref: bool = True) -> None:
    """Compile liboracle.so and, where the reference tree exists, _ref/."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    if ref and os.path.isdir(reference_tree()):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", "REF=" + reference_tree()], check=True)
        subprocess.run(["make", "-s", "-C", _HERE, "examples", "REF=" + reference_tree()], check=True)


def example(name: str):
    """Path of the reference's example program `name` built by `make examples`
    (oracle/_ref/examples), or None."""
    path = os.path.join(_HERE, "_ref", "examples", name)
    return path if os.path.exists(path) else None


class _HioTrace(C.Structure):
    _fields_ = [("iterations", C.c_int), ("last_error", C.c_float), ("errors", C.c_void_p),
                ("errors_cap", C.c_int)]


class _Trace(C.Structure):
    _fields_ = [("cycles_run", C.c_int), ("errors", C.c_void_p),
                ("mask", C.c_void_p), ("gprime", C.c_void_p)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        for s in ("f32", "f64"):
            p = _f32p if s == "f32" else _f64p
            for fn in ("imro_c2c_2d_", "imro_c2c_cols_"):
                getattr(L, fn + s).argtypes = [p, C.c_int, C.c_int, C.c_int]
            getattr(L, "imro_c2c_rows_" + s).argtypes = [p, C.c_int, C.c_int, C.c_int]
        L.imro_gaussian_weights_f32.argtypes = [C.c_double, C.c_void_p, C.c_int]
        L.imro_gaussian_weights_f32.restype = C.c_int
        L.imro_gaussian_weights_f64.argtypes = [C.c_double, C.c_void_p, C.c_int]
        L.imro_gaussian_weights_f64.restype = C.c_int
        for fn in ("imro_blur_h_f32", "imro_blur_v_f32", "imro_blur_f32"):
            getattr(L, fn).argtypes = [_f32p, C.c_int, C.c_int, C.c_double]
        L.imro_blur_f64.argtypes = [_f64p, C.c_int, C.c_int, C.c_double]
        L.imro_vector_max_f32.argtypes = [_f32p, C.c_long]
        L.imro_vector_max_f32.restype = C.c_float
        L.imro_hio_error_f64sum.argtypes = [_f32p, _f32p, C.c_long,
                                            C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.imro_hio_error_f64sum.restype = C.c_double
        L.imro_apply_modulus_f32.argtypes = [_f32p, _f32p, C.c_long]
        sw_args = [C.c_uint, C.c_uint, C.c_uint, C.c_float, C.c_float, C.c_float,
                   C.c_float, C.c_float, C.c_float, C.c_uint, C.POINTER(_Trace)]
        L.imro_shrinkwrap_f32.argtypes = [_f32p] + sw_args
        L.imro_shrinkwrap_f64.argtypes = [_f64p] + sw_args
        u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
        hio_args = [u8p, C.c_uint, C.c_uint, C.c_uint, C.c_float, C.c_float, C.c_uint,
                    C.POINTER(_HioTrace)]
        L.imro_hio_f32.argtypes = [_f32p] + hio_args
        L.imro_hio_f64.argtypes = [_f64p] + hio_args
        L.imro_random_phase_f32.argtypes = [_f32p, _f32p, C.c_uint, C.c_uint, C.c_uint]
        _LIB = L
    return _LIB


def ref_lib():
    """The reference's own CPU path (oracle/_ref), or None when not built."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libimresh_ref.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.imro_ref_shrinkwrap.argtypes = [_f32p, C.c_uint, C.c_uint, C.c_uint, C.c_float,
                                          C.c_float, C.c_float, C.c_float, C.c_float,
                                          C.c_float, C.c_uint]
        L.imro_ref_shrinkwrap.restype = C.c_int
        for fn in ("imro_ref_blur", "imro_ref_blur_h", "imro_ref_blur_v"):
            getattr(L, fn).argtypes = [_f32p, C.c_uint, C.c_uint, C.c_double]
        L.imro_ref_weights.argtypes = [C.c_double, C.c_void_p, C.c_uint]
        L.imro_ref_weights.restype = C.c_int
        L.imro_ref_vector_max.argtypes = [_f32p, C.c_uint]
        L.imro_ref_vector_max.restype = C.c_float
        L.imro_ref_hio_error.argtypes = [_f32p, _f32p, C.c_uint,
                                         C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.imro_ref_hio_error.restype = C.c_float
        L.imro_ref_hio.argtypes = [_f32p, np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS"),
                                   C.c_uint, C.c_uint, C.c_uint, C.c_float, C.c_float]
        L.imro_ref_hio.restype = C.c_int
        _REF = L
    return _REF


# ---------------------------------------------------------------- FFT
def fft2(x: np.ndarray, sign: int) -> np.ndarray:
    """Unnormalised 2D C2C transform of a complex64/complex128 [H, W] array."""
    if x.dtype == np.complex64:
        a = np.ascontiguousarray(x).view(np.float32).copy()
        lib().imro_c2c_2d_f32(a, x.shape[0], x.shape[1], sign)
        return a.view(np.complex64).reshape(x.shape)
    a = np.ascontiguousarray(x, dtype=np.complex128).view(np.float64).copy()
    lib().imro_c2c_2d_f64(a, x.shape[0], x.shape[1], sign)
    return a.view(np.complex128).reshape(x.shape)


def fft_rows(x: np.ndarray, sign: int) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.complex64).view(np.float32).copy()
    lib().imro_c2c_rows_f32(a, x.shape[-1], int(np.prod(x.shape[:-1])), sign)
    return a.view(np.complex64).reshape(x.shape)


def fft_cols(x: np.ndarray, sign: int) -> np.ndarray:
    a = np.ascontiguousarray(x, dtype=np.complex64).view(np.float32).copy()
    lib().imro_c2c_cols_f32(a, x.shape[0], x.shape[1], sign)
    return a.view(np.complex64).reshape(x.shape)


# ---------------------------------------------------------------- kernels
def gaussian_weights(sigma: float, dtype=np.float32) -> np.ndarray:
    L = lib()
    if dtype == np.float32:
        k = L.imro_gaussian_weights_f32(sigma, None, 0)
        w = np.zeros(k, np.float32)
        L.imro_gaussian_weights_f32(sigma, w.ctypes.data, k)
    else:
        k = L.imro_gaussian_weights_f64(sigma, None, 0)
        w = np.zeros(k, np.float64)
        L.imro_gaussian_weights_f64(sigma, w.ctypes.data, k)
    return w


def blur(img: np.ndarray, sigma: float, axis: str = "hv") -> np.ndarray:
    """Clamp-border Gaussian blur of a float32 [H, W] image ("h", "v", "hv")."""
    a = np.ascontiguousarray(img, dtype=np.float32).copy()
    H, W = a.shape
    fn = {"h": lib().imro_blur_h_f32, "v": lib().imro_blur_v_f32, "hv": lib().imro_blur_f32}[axis]
    fn(a.reshape(-1), W, H, float(sigma))
    return a


def vector_max(x: np.ndarray) -> float:
    a = np.ascontiguousarray(x, dtype=np.float32).reshape(-1)
    return float(lib().imro_vector_max_f32(a, a.size))


def hio_error(gprime: np.ndarray, mask: np.ndarray):
    """(error, total, count) with double sums; gprime complex64, mask float32."""
    g = np.ascontiguousarray(gprime, dtype=np.complex64).reshape(-1).view(np.float32)
    m = np.ascontiguousarray(mask, dtype=np.float32).reshape(-1)
    t, c = C.c_double(), C.c_double()
    e = lib().imro_hio_error_f64sum(g, m, m.size, C.byref(t), C.byref(c))
    return e, t.value, c.value


def apply_modulus(G: np.ndarray, modulus: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(G, dtype=np.complex64).copy()
    m = np.ascontiguousarray(modulus, dtype=np.float32).reshape(-1)
    lib().imro_apply_modulus_f32(a.reshape(-1).view(np.float32), m, m.size)
    return a


# ---------------------------------------------------------------- full path
@dataclass
class SwParams:
    n_cycles: int = 20
    target_error: float = 1e-5
    beta: float = 0.9
    cut_auto: float = 0.04
    cut: float = 0.2
    sigma0: float = 3.0
    sigma_change: float = 0.01
    n_hio: int = 20

    def args(self):
        return (self.n_cycles, self.target_error, self.beta, self.cut_auto, self.cut,
                self.sigma0, self.sigma_change, self.n_hio)


@dataclass
class SwResult:
    out: np.ndarray
    cycles_run: int
    errors: np.ndarray
    mask: np.ndarray
    gprime: np.ndarray


def shrinkwrap(modulus: np.ndarray, p: SwParams, fp64: bool = False) -> SwResult:
    """The restated CPU shrinkWrap; modulus is [H, W]."""
    H, W = modulus.shape
    n = H * W
    errs = np.zeros(max(p.n_cycles, 1), np.float32)
    mask = np.zeros(n, np.uint8)
    gp = np.zeros(2 * n, np.float32)
    tr = _Trace(0, errs.ctypes.data, mask.ctypes.data, gp.ctypes.data)
    if fp64:
        io = np.ascontiguousarray(modulus, dtype=np.float64).reshape(-1).copy()
        lib().imro_shrinkwrap_f64(io, W, H, *p.args(), C.byref(tr))
    else:
        io = np.ascontiguousarray(modulus, dtype=np.float32).reshape(-1).copy()
        lib().imro_shrinkwrap_f32(io, W, H, *p.args(), C.byref(tr))
    return SwResult(io.reshape(H, W), tr.cycles_run, errs[:tr.cycles_run],
                    mask.reshape(H, W), gp.view(np.complex64).reshape(H, W))


def ref_shrinkwrap(modulus: np.ndarray, p: SwParams) -> np.ndarray:
    """The reference's own CPU shrinkWrap (oracle/_ref); raises if not built."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/libimresh_ref.so is not built")
    H, W = modulus.shape
    io = np.ascontiguousarray(modulus, dtype=np.float32).reshape(-1).copy()
    rc = L.imro_ref_shrinkwrap(io, W, H, *p.args())
    if rc != 0:
        raise RuntimeError(f"reference shrinkWrap returned {rc}")
    return io.reshape(H, W)


# ---------------------------------------------------------------- fixed-support HIO
HIO_SEED = 2623091912   # srand() seed of addRandomPhase (hybridInputOutput.cpp:160)


@dataclass
class HioResult:
    out: np.ndarray
    iterations: int
    last_error: float
    errors: np.ndarray


def hio(modulus: np.ndarray, mask: np.ndarray, n_cycles: int = 0, target_error: float = 1e-6,
        beta: float = 0.9, seed: int = HIO_SEED, fp64: bool = False, errors_cap: int = 4096) -> HioResult:
    """The restated hybridInputOutput; modulus float [H, W], mask uint8 [H, W]."""
    H, W = modulus.shape
    m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    errs = np.zeros(errors_cap, np.float32)
    tr = _HioTrace(0, 0.0, errs.ctypes.data, errors_cap)
    if fp64:
        io = np.ascontiguousarray(modulus, dtype=np.float64).reshape(-1).copy()
        lib().imro_hio_f64(io, m, W, H, n_cycles, target_error, beta, seed, C.byref(tr))
    else:
        io = np.ascontiguousarray(modulus, dtype=np.float32).reshape(-1).copy()
        lib().imro_hio_f32(io, m, W, H, n_cycles, target_error, beta, seed, C.byref(tr))
    return HioResult(io.reshape(H, W), tr.iterations, tr.last_error,
                     errs[:min(tr.iterations + 1, errors_cap)])


def random_phase(modulus: np.ndarray, seed: int = HIO_SEED) -> np.ndarray:
    """addRandomPhase: complex64 [H, W] = M e^{i phase}."""
    H, W = modulus.shape
    m = np.ascontiguousarray(modulus, dtype=np.float32).reshape(-1)
    out = np.zeros(2 * m.size, np.float32)
    lib().imro_random_phase_f32(m, out, W, H, seed)
    return out.view(np.complex64).reshape(H, W)


def rand_field(n: int, seed: int = HIO_SEED) -> np.ndarray:
    """The C library's (float)rand()/RAND_MAX sequence after srand(seed)."""
    libc = C.CDLL(None)
    libc.srand(C.c_uint(seed))
    r = np.fromiter((libc.rand() for _ in range(n)), dtype=np.int64, count=n)
    return (r.astype(np.float32) / np.float32(2147483647.0)).astype(np.float32)


def ref_hio(modulus: np.ndarray, mask: np.ndarray, n_cycles: int = 0, target_error: float = 1e-6,
            beta: float = 0.9) -> np.ndarray:
    """The reference's own hybridInputOutput (oracle/_ref); raises if not built."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/libimresh_ref.so is not built")
    H, W = modulus.shape
    io = np.ascontiguousarray(modulus, dtype=np.float32).reshape(-1).copy()
    m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    rc = L.imro_ref_hio(io, m, W, H, n_cycles, target_error, beta)
    if rc != 0:
        raise RuntimeError(f"reference hybridInputOutput returned {rc}")
    return io.reshape(H, W)

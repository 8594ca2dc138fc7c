"""imresh_b200 -- B200 shrink-wrap / HIO phase retrieval.

Python front end over the C ABI of ``lib/libimresh_b200.so``
(declared in ``include/imresh_b200.h``).  Every compute call goes through
that library; there is no CPU fallback: if the library is missing the calls
raise.  Device buffers may be given as torch CUDA tensors or raw pointers.

Entry points mirror the reference's API for this path:

* :func:`cuda_shrink_wrap` -- ``imresh::algorithms::cuda::cudaShrinkWrap``
  (src/imresh/algorithms/cuda/cudaShrinkWrap.hpp:114-130): host buffer,
  modulus in, object out, synchronous, returns 0 on success.
* :class:`Plan` -- reusable device-resident reconstruction of one size.
* :func:`fft2d`, :func:`gaussian_blur`, :func:`vector_max`,
  :func:`gaussian_weights` -- the kernel-level operations of the path.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libimresh_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "imresh_b200.h")
FLT_MIN = float(np.finfo(np.float32).tiny)
_LIB = None


class ImrError(RuntimeError):
    def __init__(self, status: int, where: str = ""):
        self.status = status
        msg = f"{where}: {status_string(status)} ({status})"
        detail = last_error()
        if detail:
            msg += f" [{detail}]"
        super().__init__(msg)


class CParams(C.Structure):
    _fields_ = [("nCycles", C.c_uint), ("targetError", C.c_float), ("hioBeta", C.c_float),
                ("intensityCutOffAutoCorel", C.c_float), ("intensityCutOff", C.c_float),
                ("sigma0", C.c_float), ("sigmaChange", C.c_float), ("nHioCycles", C.c_uint)]


@dataclass
class Params:
    """cudaShrinkWrap's parameters; 0 selects the reference's CUDA default."""
    n_cycles: int = 0
    target_error: float = 0.0
    hio_beta: float = 0.0
    cut_off_auto_corel: float = 0.0
    cut_off: float = 0.0
    sigma0: float = 0.0
    sigma_change: float = 0.0
    n_hio_cycles: int = 0

    def c(self) -> CParams:
        return CParams(self.n_cycles, self.target_error, self.hio_beta, self.cut_off_auto_corel,
                       self.cut_off, self.sigma0, self.sigma_change, self.n_hio_cycles)


def lib() -> C.CDLL:
    """Load the native library (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python __graft_entry__.py` "
                           "(or `make -C imresh_b200/csrc`)")
    L = C.CDLL(LIB_PATH)
    vp, u, f, i = C.c_void_p, C.c_uint, C.c_float, C.c_int
    L.imr_status_string.restype = C.c_char_p
    L.imr_status_string.argtypes = [i]
    L.imr_last_error.restype = C.c_char_p
    L.imr_max_side.restype = u
    L.imr_side_supported.argtypes = [u]
    L.imr_cuda_shrink_wrap.argtypes = [vp, u, u, vp, u, u, u, f, f, f, f, f, f, u]
    L.imr_plan_create.argtypes = [C.POINTER(vp), u, u, C.POINTER(CParams)]
    L.imr_plan_execute.argtypes = [vp, vp, vp, vp]
    L.imr_plan_execute_host.argtypes = [vp, vp, vp, vp]
    L.imr_plan_stats.argtypes = [vp, vp, C.POINTER(i), vp]
    L.imr_plan_launches.argtypes = [vp, C.POINTER(C.c_long)]
    L.imr_plan_copy_state.argtypes = [vp, i, vp, vp]
    L.imr_plan_destroy.argtypes = [vp]
    L.imr_plan_profile.argtypes = [vp, i, vp, C.POINTER(f), C.POINTER(f)]
    L.imr_plan_pass_bytes.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.imr_fft2d.argtypes = [vp, u, u, i, vp]
    L.imr_fft2d_split.argtypes = [vp, u, u, i, i, vp]
    L.imr_plan_set_precision.argtypes = [vp, i]
    L.imr_plan_set_wait_limit.argtypes = [vp, C.c_ulonglong]
    L.imr_gaussian_blur.argtypes = [vp, vp, u, u, C.c_double, i, vp]
    L.imr_gaussian_weights.argtypes = [C.c_double, vp, i]
    L.imr_vector_max.argtypes = [vp, C.c_size_t, C.POINTER(f), vp]
    _LIB = L
    return L


def header_functions() -> list:
    """Names of the functions include/imresh_b200.h declares."""
    text = open(HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(imr_[a-z0-9_]+)\s*\(", text)))


def status_string(rc: int) -> str:
    return lib().imr_status_string(rc).decode()


def last_error() -> str:
    try:
        return lib().imr_last_error().decode()
    except Exception:   # library not loadable
        return ""


def _check(rc: int, where: str):
    if rc != 0:
        raise ImrError(rc, where)


def _ptr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_contiguous():
            raise ValueError("device tensor must be contiguous")
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        if not x.flags.c_contiguous:
            raise ValueError("host array must be C-contiguous")
        return x.ctypes.data
    raise TypeError(f"cannot take a pointer of {type(x)}")


def _stream(s) -> int:
    if s is None:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.cuda.current_stream().cuda_stream
        except Exception:
            pass
        return 0
    if isinstance(s, int):
        return s
    return s.cuda_stream


def side_supported(n: int) -> bool:
    return bool(lib().imr_side_supported(n))


# ------------------------------------------------------------------ drop-in
def cuda_shrink_wrap(io: np.ndarray, width: int, height: int, stream=0, n_blocks: int = 256,
                     n_threads: int = 256, n_cycles: int = 0, target_error: float = 0.0,
                     hio_beta: float = 0.0, cut_off_auto_corel: float = 0.0, cut_off: float = 0.0,
                     sigma0: float = 0.0, sigma_change: float = 0.0, n_hio_cycles: int = 0) -> int:
    """cudaShrinkWrap: ``io`` (float32, width*height, host) holds the Fourier
    modulus on entry and Re(g') on return.  Returns 0 on success, else an
    imr_status code (the reference returns 0 and exits the process on error)."""
    if io.dtype != np.float32 or not io.flags.c_contiguous or io.size != width * height:
        raise ValueError("io must be a C-contiguous float32 array of width*height values")
    return lib().imr_cuda_shrink_wrap(io.ctypes.data, width, height, _stream(stream) if stream else 0,
                                      n_blocks, n_threads, n_cycles, target_error, hio_beta,
                                      cut_off_auto_corel, cut_off, sigma0, sigma_change,
                                      n_hio_cycles)


class Plan:
    """Device-resident reconstruction plan for one (width, height, params)."""

    def __init__(self, width: int, height: int, params: Params | None = None):
        self.width, self.height = width, height
        self.params = params or Params()
        h = C.c_void_p()
        cp = self.params.c()
        _check(lib().imr_plan_create(C.byref(h), width, height, C.byref(cp)), "imr_plan_create")
        self._h = h

    def execute(self, d_modulus, d_out, stream=None):
        _check(lib().imr_plan_execute(self._h, _ptr(d_modulus), _ptr(d_out), _stream(stream)),
               "imr_plan_execute")

    def execute_host(self, modulus: np.ndarray, out: np.ndarray | None = None, stream=None):
        m = np.ascontiguousarray(modulus, dtype=np.float32)
        if out is None:
            out = np.empty_like(m)
        _check(lib().imr_plan_execute_host(self._h, _ptr(m), _ptr(out), _stream(stream)),
               "imr_plan_execute_host")
        return out

    def stats(self, stream=None):
        """(cycles_done, per-cycle errors)."""
        n = C.c_int()
        cyc = max(self.params.n_cycles or 20, 1)
        errs = np.zeros(cyc, np.float32)
        _check(lib().imr_plan_stats(self._h, _stream(stream), C.byref(n), errs.ctypes.data),
               "imr_plan_stats")
        return n.value, errs[:n.value]

    def set_precision(self, precision: int):
        """Column-pass arithmetic: PREC_FP32 (default), PREC_BF16X3 or PREC_FP16X3."""
        _check(lib().imr_plan_set_precision(self._h, precision), "imr_plan_set_precision")

    def launches(self) -> int:
        n = C.c_long()
        _check(lib().imr_plan_launches(self._h, C.byref(n)), "imr_plan_launches")
        return n.value

    def profile(self, iters: int = 20, stream=None):
        """Mean (row pass ms, column pass ms) over `iters` HIO iterations."""
        a, b = C.c_float(), C.c_float()
        _check(lib().imr_plan_profile(self._h, iters, _stream(stream), C.byref(a), C.byref(b)),
               "imr_plan_profile")
        return a.value, b.value

    def pass_bytes(self):
        a, b = C.c_double(), C.c_double()
        _check(lib().imr_plan_pass_bytes(self._h, C.byref(a), C.byref(b)), "imr_plan_pass_bytes")
        return a.value, b.value

    def state(self, what: str, stream=None) -> np.ndarray:
        W, H = self.width, self.height
        code, arr = {"mask": (0, np.zeros((H, W), np.uint8)),
                     "x": (1, np.zeros((H, W), np.complex64)),
                     "gprev": (2, np.zeros((H, W), np.complex64)),
                     "blurred": (3, np.zeros((H, W), np.float32))}[what]
        _check(lib().imr_plan_copy_state(self._h, code, arr.ctypes.data, _stream(stream)),
               "imr_plan_copy_state")
        return arr

    def close(self):
        if getattr(self, "_h", None):
            lib().imr_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ kernels
def fft2d(d_data, width: int, height: int, sign: int, stream=None):
    """In-place unnormalised 2D C2C transform of a device complex64 buffer."""
    _check(lib().imr_fft2d(_ptr(d_data), width, height, sign, _stream(stream)), "imr_fft2d")


PREC_FP32, PREC_BF16X3, PREC_FP16X3 = 0, 1, 2
SCHEDULE_GROUPED, SCHEDULE_CHAINED = 0, 1


def fft2d_split(d_data, width: int, height: int, sign: int, precision: int = PREC_BF16X3, stream=None):
    """fft2d with the column transform on the split-precision tensor-core passes."""
    _check(lib().imr_fft2d_split(_ptr(d_data), width, height, sign, precision, _stream(stream)),
           "imr_fft2d_split")


def gaussian_blur(d_data, d_tmp, width: int, height: int, sigma: float, axes: int = 3, stream=None):
    _check(lib().imr_gaussian_blur(_ptr(d_data), _ptr(d_tmp), width, height, float(sigma), axes,
                                   _stream(stream)), "imr_gaussian_blur")


def gaussian_weights(sigma: float) -> np.ndarray:
    k = lib().imr_gaussian_weights(float(sigma), None, 0)
    w = np.zeros(k, np.float32)
    lib().imr_gaussian_weights(float(sigma), w.ctypes.data, k)
    return w


def vector_max(d_data, n: int, stream=None) -> float:
    r = C.c_float()
    _check(lib().imr_vector_max(_ptr(d_data), n, C.byref(r), _stream(stream)), "imr_vector_max")
    return r.value


# ------------------------------------------------------------------ engine
class CResult(C.Structure):
    _fields_ = [("tag", C.c_longlong), ("width", C.c_uint), ("height", C.c_uint),
                ("cycles_done", C.c_int), ("last_error", C.c_float), ("latency_ms", C.c_double),
                ("status", C.c_int)]


class CEngineInfo(C.Structure):
    _fields_ = [("pending", C.c_int), ("active", C.c_int), ("done", C.c_int),
                ("device_bytes_used", C.c_size_t), ("device_bytes_peak", C.c_size_t),
                ("device_bytes_budget", C.c_size_t), ("launches", C.c_long), ("steps", C.c_long),
                ("host_launches", C.c_long), ("kernels_per_step", C.c_long), ("graph_builds", C.c_long),
                ("graph_updates", C.c_long), ("alloc_failures", C.c_long), ("resident", C.c_int),
                ("resident_px", C.c_size_t), ("last_step_ms", C.c_double), ("ms_per_mpx", C.c_double),
                ("device_ms", C.c_double), ("schedule", C.c_int), ("grid_pct", C.c_int),
                ("tune_explored", C.c_long), ("tune_cache_hits", C.c_long), ("cycles_per_step", C.c_int)]


def _engine_sigs(L):
    vp = C.c_void_p
    L.imr_engine_create.argtypes = [C.POINTER(vp), C.c_size_t, C.c_int, vp]
    L.imr_engine_submit.argtypes = [vp, vp, vp, C.c_uint, C.c_uint, C.POINTER(CParams), C.c_longlong]
    L.imr_engine_submit_intensity.argtypes = [vp, vp, vp, C.c_uint, C.c_uint, C.POINTER(CParams), C.c_longlong]
    L.imr_engine_step.argtypes = [vp]
    L.imr_engine_run.argtypes = [vp]
    L.imr_engine_poll.argtypes = [vp, C.POINTER(CResult), C.c_int, C.POINTER(C.c_int)]
    L.imr_engine_stats.argtypes = [vp, C.POINTER(CEngineInfo)]
    L.imr_engine_destroy.argtypes = [vp]
    L.imr_diffraction_intensity.argtypes = [vp, C.c_uint, C.c_uint, vp]
    L.imr_engine_snapshot_size.argtypes = [vp, C.c_longlong, C.POINTER(C.c_size_t)]
    L.imr_engine_checkpoint.argtypes = [vp, C.c_longlong, vp, C.c_size_t]
    L.imr_engine_suspend.argtypes = [vp, C.c_longlong, vp, C.c_size_t]
    L.imr_engine_resume.argtypes = [vp, vp, C.c_size_t, vp]
    L.imr_engine_cancel.argtypes = [vp, C.c_longlong]
    L.imr_engine_inject_alloc_failures.argtypes = [vp, C.c_int]
    L.imr_engine_set_admission.argtypes = [vp, C.c_size_t]
    L.imr_engine_set_step_target.argtypes = [vp, C.c_double]
    L.imr_engine_set_schedule.argtypes = [vp, C.c_int]
    L.imr_engine_set_autotune.argtypes = [vp, C.c_int, C.c_char_p]
    L.imr_engine_set_cycles_per_step.argtypes = [vp, C.c_int]


class Engine:
    """Batched, continuously-admitting engine (imr_engine_*).

    submit() queues a host modulus and a host output buffer (both kept alive
    here until the result is polled); step() runs one shrink-wrap cycle of
    every active reconstruction; poll() returns finished results."""

    def __init__(self, device_bytes: int = 0, max_jobs: int = 4096, stream=None):
        L = lib()
        _engine_sigs(L)
        h = C.c_void_p()
        _check(L.imr_engine_create(C.byref(h), device_bytes, max_jobs, _stream(stream)),
               "imr_engine_create")
        self._h = h
        self._keep = {}

    def submit(self, modulus: np.ndarray, params: Params | None = None, tag: int = 0,
               out: np.ndarray | None = None, intensity: bool = False) -> np.ndarray:
        """Queue one reconstruction of `modulus` ([H, W]); with intensity=True the
        array is a measured intensity and the engine takes its square root."""
        m = np.ascontiguousarray(modulus, dtype=np.float32)
        H, W = m.shape
        if out is None:
            out = np.empty_like(m)
        cp = (params or Params()).c()
        name = "imr_engine_submit_intensity" if intensity else "imr_engine_submit"
        _check(getattr(lib(), name)(self._h, m.ctypes.data, out.ctypes.data, W, H, C.byref(cp), tag), name)
        self._keep[tag] = (m, out)
        return out

    def step(self):
        _check(lib().imr_engine_step(self._h), "imr_engine_step")

    def run(self):
        _check(lib().imr_engine_run(self._h), "imr_engine_run")

    def poll(self, max_results: int = 4096):
        res = (CResult * max_results)()
        n = C.c_int()
        _check(lib().imr_engine_poll(self._h, res, max_results, C.byref(n)), "imr_engine_poll")
        out = []
        for r in res[:n.value]:
            m, o = self._keep.pop(r.tag, (None, None))
            out.append(dict(tag=r.tag, width=r.width, height=r.height, cycles_done=r.cycles_done,
                            last_error=r.last_error, latency_ms=r.latency_ms, status=r.status,
                            out=o))
        return out

    def _snapshot(self, fn, tag: int) -> bytes:
        n = C.c_size_t()
        _check(lib().imr_engine_snapshot_size(self._h, tag, C.byref(n)), "imr_engine_snapshot_size")
        buf = np.empty(n.value, np.uint8)
        _check(getattr(lib(), fn)(self._h, tag, buf.ctypes.data, n.value), fn)
        return buf.tobytes()

    def checkpoint(self, tag: int) -> bytes:
        """Saved state of the running reconstruction `tag` (it keeps running)."""
        return self._snapshot("imr_engine_checkpoint", tag)

    def suspend(self, tag: int) -> bytes:
        """Saved state of the running reconstruction `tag`, which leaves the engine."""
        snap = self._snapshot("imr_engine_suspend", tag)
        self._keep.pop(tag, None)
        return snap

    def resume(self, snapshot: bytes, out: np.ndarray | None = None) -> np.ndarray:
        """Queue a saved reconstruction; it continues where it was saved."""
        buf = np.frombuffer(snapshot, np.uint8)
        W, H = np.frombuffer(snapshot[8:16], np.uint32)
        tag = int(np.frombuffer(snapshot[48:56], np.int64)[0])
        if out is None:
            out = np.empty((int(H), int(W)), np.float32)
        _check(lib().imr_engine_resume(self._h, buf.ctypes.data, buf.size, out.ctypes.data),
               "imr_engine_resume")
        self._keep[tag] = (buf, out)
        return out

    def cancel(self, tag: int):
        """Cancel a pending or running request (reported with IMR_ERR_CANCELLED)."""
        _check(lib().imr_engine_cancel(self._h, tag), "imr_engine_cancel")

    def set_admission(self, max_active_pixels: int):
        """Admit requests only while the resident pixels stay within the bound (0: none)."""
        _check(lib().imr_engine_set_admission(self._h, max_active_pixels), "imr_engine_set_admission")

    def set_schedule(self, schedule: int):
        """SCHEDULE_GROUPED (default) or SCHEDULE_CHAINED step graphs."""
        _check(lib().imr_engine_set_schedule(self._h, schedule), "imr_engine_set_schedule")

    def set_autotune(self, enable: bool = True, cache_path: str | None = None):
        """Pick the step configuration per admitted set by timing real steps; cache in a file."""
        _check(lib().imr_engine_set_autotune(self._h, 1 if enable else 0,
                                             cache_path.encode() if cache_path else None),
               "imr_engine_set_autotune")

    def set_step_target(self, ms: float):
        """Admit requests only while the predicted step time stays within `ms` (0: off)."""
        _check(lib().imr_engine_set_step_target(self._h, float(ms)), "imr_engine_set_step_target")

    def set_cycles_per_step(self, cycles: int):
        """Shrink-wrap cycles captured into one step's graph (1..256; default 1)."""
        _check(lib().imr_engine_set_cycles_per_step(self._h, int(cycles)), "imr_engine_set_cycles_per_step")

    def inject_alloc_failures(self, count: int):
        """Make the device allocations of the next `count` admissions fail (tests)."""
        _check(lib().imr_engine_inject_alloc_failures(self._h, count), "imr_engine_inject_alloc_failures")

    def info(self) -> dict:
        i = CEngineInfo()
        _check(lib().imr_engine_stats(self._h, C.byref(i)), "imr_engine_stats")
        return {k: getattr(i, k) for k, _ in CEngineInfo._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().imr_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def diffraction_intensity(obj: np.ndarray) -> np.ndarray:
    """|FFT2(obj)| of a real float32 image on the engine's FFT (host in/out)."""
    L = lib()
    _engine_sigs(L)
    a = np.ascontiguousarray(obj, dtype=np.float32).copy()
    H, W = a.shape
    _check(L.imr_diffraction_intensity(a.ctypes.data, W, H, _stream(None)), "imr_diffraction_intensity")
    return a


# ------------------------------------------------------------------ fixed-support HIO
HIO_SEED = 2623091912   # srand() seed of libs::addRandomPhase (hybridInputOutput.cpp:160)
MASK_F32, MASK_U8 = 0, 1


def _hio_sigs(L):
    vp, u, f, i = C.c_void_p, C.c_uint, C.c_float, C.c_int
    L.imr_hybrid_input_output.argtypes = [vp, vp, u, u, u, f, f, vp]
    L.imr_hio_plan_create.argtypes = [C.POINTER(vp), u, u, u, f, f]
    L.imr_hio_plan_execute.argtypes = [vp, vp, vp, vp, u, vp]
    L.imr_hio_plan_execute_host.argtypes = [vp, vp, vp, vp, u, vp]
    L.imr_hio_plan_stats.argtypes = [vp, vp, C.POINTER(i), C.POINTER(f), vp, i]
    L.imr_hio_plan_destroy.argtypes = [vp]
    L.imr_calculate_hio_error.argtypes = [vp, vp, i, C.c_size_t, i, C.POINTER(f), C.POINTER(f),
                                          C.POINTER(f), vp]
    L.imr_rand_field.argtypes = [vp, C.c_size_t, u, vp]


def rand_field(d_out, n: int, seed: int = HIO_SEED, stream=None):
    """Device complex64 ((float)rand()/RAND_MAX, 0) after srand(seed)."""
    L = lib()
    _hio_sigs(L)
    _check(L.imr_rand_field(_ptr(d_out), n, seed, _stream(stream)), "imr_rand_field")


def hybrid_input_output(io: np.ndarray, mask: np.ndarray, n_cycles: int = 0,
                        target_error: float = 1e-6, beta: float = 0.9, stream=0) -> int:
    """libs::hybridInputOutput: ``io`` (float32 [H][W], host) holds the Fourier
    modulus on entry and Re(g') on return; ``mask`` (uint8 [H][W]) is 1 outside
    the support.  Defaults as the reference's (hybridInputOutput.hpp:81-90).
    Returns 0 on success, else an imr_status code."""
    if io.dtype != np.float32 or not io.flags.c_contiguous or io.ndim != 2:
        raise ValueError("io must be a C-contiguous float32 [H][W] array")
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    if m.shape != io.shape:
        raise ValueError("mask must have the shape of io")
    L = lib()
    _hio_sigs(L)
    H, W = io.shape
    return L.imr_hybrid_input_output(io.ctypes.data, m.ctypes.data, W, H, n_cycles, target_error,
                                     beta, _stream(stream) if stream else 0)


class HioPlan:
    """Reusable fixed-support HIO plan (random initial phase) for one size."""

    def __init__(self, width: int, height: int, n_cycles: int = 0, target_error: float = 1e-6,
                 beta: float = 0.9):
        L = lib()
        _hio_sigs(L)
        self.width, self.height = width, height
        h = C.c_void_p()
        _check(L.imr_hio_plan_create(C.byref(h), width, height, n_cycles, target_error, beta),
               "imr_hio_plan_create")
        self._h = h

    def execute(self, d_modulus, d_mask, d_out, seed: int = HIO_SEED, stream=None):
        _check(lib().imr_hio_plan_execute(self._h, _ptr(d_modulus), _ptr(d_mask), _ptr(d_out), seed,
                                          _stream(stream)), "imr_hio_plan_execute")

    def execute_host(self, modulus: np.ndarray, mask: np.ndarray, out: np.ndarray | None = None,
                     seed: int = HIO_SEED, stream=None):
        m = np.ascontiguousarray(modulus, dtype=np.float32)
        k = np.ascontiguousarray(mask, dtype=np.uint8)
        if out is None:
            out = np.empty_like(m)
        _check(lib().imr_hio_plan_execute_host(self._h, _ptr(m), _ptr(k), _ptr(out), seed,
                                               _stream(stream)), "imr_hio_plan_execute_host")
        return out

    def stats(self, cap: int = 4096, stream=None):
        """(iterations, last tested error, per-iteration errors)."""
        n, e = C.c_int(), C.c_float()
        errs = np.zeros(cap, np.float32)
        _check(lib().imr_hio_plan_stats(self._h, _stream(stream), C.byref(n), C.byref(e),
                                        errs.ctypes.data, cap), "imr_hio_plan_stats")
        return n.value, e.value, errs[:min(n.value + 1, cap)]

    def close(self):
        if getattr(self, "_h", None):
            lib().imr_hio_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def calculate_hio_error(d_data, d_mask, n: int, invert_mask: bool = False, stream=None):
    """cudaCalculateHioError over device buffers: (total, count, error).  The
    mask is float32 or uint8 (a torch tensor's dtype decides)."""
    L = lib()
    _hio_sigs(L)
    kind = MASK_U8 if str(getattr(d_mask, "dtype", "")).endswith("uint8") else MASK_F32
    t, c, e = C.c_float(), C.c_float(), C.c_float()
    _check(L.imr_calculate_hio_error(_ptr(d_data), _ptr(d_mask), kind, n, int(invert_mask),
                                     C.byref(t), C.byref(c), C.byref(e), _stream(stream)),
           "imr_calculate_hio_error")
    return t.value, c.value, e.value

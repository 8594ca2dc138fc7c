"""Seeded synthetic diffraction inputs (Gaussian-blob objects).

The reference ships no dataset for this path; its own test inputs are
procedurally generated atom clusters (examples/createTestData/createAtomCluster.cpp:45-145)
pushed through ``diffractionIntensity`` (src/imresh/libs/diffractionIntensity.cpp:49-80),
which returns |FFT2(object)| -- the Fourier *modulus* that ``shrinkWrap`` and
``cudaShrinkWrap`` take as input (they scale G' to that value,
src/imresh/algorithms/vectorElementwise.cpp:77-79).

This module builds the blob recipe used by the benchmark workloads:
object = sum of isotropic Gaussian blobs a*exp(-r^2/(2 s^2)) with centres
uniform in a centred disk, zero beyond 5 s of every centre; intensity
I = |FFT2(object)|^2 (unnormalised, DC at [0, 0]), optionally with Poisson
photon noise at a given total count; the engine is fed M = sqrt(I).

Every request draws from its own numpy ``Generator`` seeded with
``[seed, index]``, so a request's input is the same whether it is generated
alone or inside a batch.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class BlobSpec:
    width: int
    height: int
    n_blobs: int
    radius: float                     # disk radius for the centres, px
    sigma: tuple = (2.0, 2.0)         # blob sigma ~ U(lo, hi)
    amp: tuple = (0.5, 1.0)           # amplitude ~ U(lo, hi)
    photons: float | None = None      # total counts for Poisson noise, None = exact


def render_object(spec: BlobSpec, rng: np.random.Generator) -> np.ndarray:
    """float64 [H, W] object."""
    W, H = spec.width, spec.height
    n = spec.n_blobs
    r = spec.radius * np.sqrt(rng.random(n))
    th = 2.0 * np.pi * rng.random(n)
    cx = W / 2.0 + r * np.cos(th)
    cy = H / 2.0 + r * np.sin(th)
    sig = rng.uniform(spec.sigma[0], spec.sigma[1], n) if spec.sigma[1] > spec.sigma[0] \
        else np.full(n, float(spec.sigma[0]))
    amp = rng.uniform(spec.amp[0], spec.amp[1], n)
    obj = np.zeros((H, W), np.float64)
    for i in range(n):
        h = int(np.ceil(5.0 * sig[i]))
        x0, x1 = max(0, int(np.floor(cx[i])) - h), min(W, int(np.floor(cx[i])) + h + 2)
        y0, y1 = max(0, int(np.floor(cy[i])) - h), min(H, int(np.floor(cy[i])) + h + 2)
        if x0 >= x1 or y0 >= y1:
            continue
        xs = np.arange(x0, x1) - cx[i]
        ys = np.arange(y0, y1) - cy[i]
        d2 = ys[:, None] ** 2 + xs[None, :] ** 2
        blob = amp[i] * np.exp(-d2 / (2.0 * sig[i] ** 2))
        blob[d2 > (5.0 * sig[i]) ** 2] = 0.0
        obj[y0:y1, x0:x1] += blob
    return obj


def intensity(obj: np.ndarray, photons: float | None, rng: np.random.Generator) -> np.ndarray:
    """|FFT2(obj)|^2 in float64, with optional Poisson noise at `photons` counts."""
    I = np.abs(np.fft.fft2(obj)) ** 2
    if photons:
        s = photons / I.sum()
        I = rng.poisson(I * s).astype(np.float64) / s
    return I


def make_modulus(spec: BlobSpec, seed: int, index: int = 0):
    """(modulus float32 [H, W], object float64 [H, W]) for one request."""
    rng = np.random.default_rng([seed, index])
    obj = render_object(spec, rng)
    I = intensity(obj, spec.photons, rng)
    return np.sqrt(I).astype(np.float32), obj


# ---- the benchmark workloads (sizes and recipes of the five named configs)
def cfg0_spec() -> BlobSpec:
    """256x256, 60 blobs sigma 2, amplitudes U(0.5, 1), disk r = 40, no noise."""
    return BlobSpec(256, 256, 60, 40.0, (2.0, 2.0), (0.5, 1.0), None)


def cfg1_spec() -> BlobSpec:
    """2048x2048, 400 blobs sigma U(1.5, 3), amplitudes U(0.3, 1), r = 300, 1e9 photons."""
    return BlobSpec(2048, 2048, 400, 300.0, (1.5, 3.0), (0.3, 1.0), 1e9)


def cfg3_spec() -> BlobSpec:
    """4096x4096, 1500 blobs, r = 600 (blob sigma/amplitude as the 2048 recipe)."""
    return BlobSpec(4096, 4096, 1500, 600.0, (1.5, 3.0), (0.3, 1.0), None)


CFG2_SIDES = (128, 192, 256, 384, 512)


def cfg2_specs(n: int = 512, seed: int = 2):
    """Uneven batch: W, H each from {128,192,256,384,512}; 20-200 blobs with
    sigma U(1, 3) in a disk of radius 0.15*min(W, H); Poisson at log-uniform
    1e7..1e9 counts."""
    rng = np.random.default_rng([seed, 1 << 30])
    specs = []
    for _ in range(n):
        W = int(rng.choice(CFG2_SIDES))
        H = int(rng.choice(CFG2_SIDES))
        nb = int(rng.integers(20, 201))
        ph = float(10 ** rng.uniform(7, 9))
        specs.append(BlobSpec(W, H, nb, 0.15 * min(W, H), (1.0, 3.0), (0.3, 1.0), ph))
    return specs


def cfg4_specs(n: int = 20000, seed: int = 4):
    """Serving stream: W, H log-uniform integers in [64, 2048]; 0.5-3 blobs per
    1000 px^2; Poisson at log-uniform 1e6..1e9 counts."""
    rng = np.random.default_rng([seed, 1 << 30])
    specs = []
    for _ in range(n):
        W = int(round(np.exp(rng.uniform(np.log(64), np.log(2048)))))
        H = int(round(np.exp(rng.uniform(np.log(64), np.log(2048)))))
        dens = rng.uniform(0.5, 3.0)
        nb = max(1, int(dens * W * H / 1000.0))
        ph = float(10 ** rng.uniform(6, 9))
        specs.append(BlobSpec(W, H, nb, 0.15 * min(W, H), (1.0, 3.0), (0.3, 1.0), ph))
    return specs


# ---- inputs of the fixed-support HIO (libs::hybridInputOutput)
def centrosymmetric(M: np.ndarray) -> np.ndarray:
    """max(M[k], M[-k]) per frequency: exactly centrosymmetric, as the
    modulus of a real object is (the reference's debug build asserts it,
    src/imresh/libs/hybridInputOutput.cpp:140-158)."""
    return np.maximum(M, np.roll(np.flip(M), 1, axis=(0, 1)))


def support_mask(spec: BlobSpec, margin: float = 1.5) -> np.ndarray:
    """uint8 [H, W]: 1 outside a centred disk that holds every blob centre's
    disk plus `margin` blob widths (the fixed support of the HIO)."""
    W, H = spec.width, spec.height
    r = spec.radius + margin * 5.0 * spec.sigma[1]
    yy, xx = np.mgrid[:H, :W]
    return (((xx - W / 2.0) ** 2 + (yy - H / 2.0) ** 2) > r * r).astype(np.uint8)

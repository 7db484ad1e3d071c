"""Seeded synthetic acquisitions in the shapes of the frame-aligner workloads.

There is no public dataset for this path: acquisitions are generated. A reference is a background
plus a sum of Gaussian blobs scaled to a target mean photon count; each frame is the continuous
reference sampled along a known scan-time displacement (a clipped random walk over the nD control
points) with Poisson noise. Randomness comes from ``numpy.random.Generator(PCG64(seed))``; the
deterministic blob sums are evaluated by ``csrc/fa_synth.c`` (``libfa_synth.so``).

Scan timing for every workload: line duration 1, interline 1.01, interframe = frame duration
(n_y * 1.01), unidirectional -- values that satisfy the warper's last-interval check
(FrameAligner/FrameWarper.cpp:280-281) for all sizes used here.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def _synth():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "libfa_synth.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run __graft_entry__.build() or make -C frame-aligner_b200")
        L = C.CDLL(path)
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        L.fa_synth_render.argtypes = [C.c_int, C.c_int, C.c_int, f64p, C.c_int, C.c_double, C.c_double, C.c_void_p,
                                      C.c_int, C.c_void_p, C.c_int, C.c_int, f32p]
        _lib = L
    return _lib


def scan_durations(nz, ny, nx, nD, line=1.0, interline=1.01, interframe=None):
    """ImageScanParameters (FrameAligner/ImageScanParameters.h:7-20) then processScanParameters
    (FrameAligner/FrameWarper.cpp:223-236). Returns (line, interline, interframe, t_pixel,
    t_frame, t_stack) after processing."""
    if interline < line:
        interline = 1.01 * line
    t_frame = ny * interline
    if interframe is None:
        interframe = t_frame
    t_pixel = line / nx
    stack = (nz - 1) * interframe + t_frame
    cap = nz * t_frame / (nD - nz) if nD != nz else float("inf")
    if interframe - t_frame > cap:
        interframe = t_frame + cap
        stack = (nz - 1) * interframe + t_frame
    return line, interline, interframe, t_pixel, t_frame, stack


@dataclass
class BlobSpec:
    n_blobs: int
    sigma_xy: tuple
    sigma_z: tuple
    amplitude: tuple = (5.0, 50.0)
    background: float = 2.0
    mean: float = 20.0


@dataclass
class WalkSpec:
    step_xy: float
    bound_xy: float
    step_z: float = 0.0
    bound_z: float = 0.0


@dataclass
class Acquisition:
    reference: np.ndarray          # (nz, ny, nx) float32, noise-free photon rate
    frames: np.ndarray             # (n_frames, nz, ny, nx) float32 photon counts
    D_true: np.ndarray             # (n_frames, nD, 3) float64
    nD: int
    scan: tuple                    # (line, interline, interframe) as passed to the warper
    blobs: np.ndarray = field(repr=False, default=None)
    scale: float = 1.0


def _render(shape, blobs, background, scale, D=None, nD=0, scan=None, n_threads=None):
    nz, ny, nx = shape
    out = np.empty(nz * ny * nx, np.float32)
    if n_threads is None:
        n_threads = min(32, os.cpu_count() or 1)
    b = np.ascontiguousarray(blobs, np.float64)
    if D is not None:
        Dc = np.ascontiguousarray(D, np.float64)
        sc = np.ascontiguousarray(scan, np.float64)
        _synth().fa_synth_render(nz, ny, nx, b, b.shape[0], background, scale, Dc.ctypes.data, nD, sc.ctypes.data,
                                 0, n_threads, out)
    else:
        _synth().fa_synth_render(nz, ny, nx, b, b.shape[0], background, scale, None, 0, None, 0, n_threads, out)
    return out.reshape(shape)


def random_walk(rng, nD, walk: WalkSpec, start=None):
    D = np.zeros((nD, 3), np.float64)
    cur = np.zeros(3) if start is None else np.array(start, np.float64)
    for i in range(nD):
        step = np.array([rng.normal(0, walk.step_xy), rng.normal(0, walk.step_xy),
                         rng.normal(0, walk.step_z) if walk.step_z > 0 else 0.0])
        cur = cur + step
        cur[:2] = np.clip(cur[:2], -walk.bound_xy, walk.bound_xy)
        cur[2] = np.clip(cur[2], -walk.bound_z, walk.bound_z) if walk.bound_z > 0 else 0.0
        D[i] = cur
    return D


def make_acquisition(shape, nD, n_frames, blobs: BlobSpec, walk: WalkSpec, seed: int, poisson=True,
                     continue_walk=False) -> Acquisition:
    """One reference and n_frames displaced, noisy frames (seeded)."""
    nz, ny, nx = shape
    rng = np.random.Generator(np.random.PCG64(seed))
    n = blobs.n_blobs
    P = np.empty((n, 7), np.float64)
    P[:, 0] = rng.uniform(0, nx, n)
    P[:, 1] = rng.uniform(0, ny, n)
    P[:, 2] = rng.uniform(0, nz, n) if nz > 1 else 0.0
    P[:, 3] = rng.uniform(*blobs.sigma_xy, n)
    P[:, 4] = P[:, 3]
    P[:, 5] = rng.uniform(*blobs.sigma_z, n) if nz > 1 else 1.0
    P[:, 6] = rng.uniform(*blobs.amplitude, n)
    raw = _render(shape, P, blobs.background, 1.0)
    scale = blobs.mean / float(raw.mean(dtype=np.float64))
    reference = _render(shape, P, blobs.background, scale)
    line, interline, interframe, t_pixel, _, stack = scan_durations(nz, ny, nx, nD)
    scan_vec = (t_pixel, interline, interframe, stack)
    frames = np.empty((n_frames,) + tuple(shape), np.float32)
    D_true = np.empty((n_frames, nD, 3), np.float64)
    start = None
    for k in range(n_frames):
        frng = np.random.Generator(np.random.PCG64(seed * 1000 + k + 1))
        D = random_walk(frng, nD, walk, start=start)
        if nz == 1:
            D[:, 2] = 0.0
        D_true[k] = D
        if continue_walk:
            start = D[-1]
        lam = _render(shape, P, blobs.background, scale, D=D, nD=nD, scan=scan_vec)
        frames[k] = frng.poisson(np.maximum(lam, 0)).astype(np.float32) if poisson else lam
    return Acquisition(reference, frames, D_true, nD, (line, interline, interframe), P, scale)


# Workload shapes. Blob specs follow the workload descriptions; seeds are fixed per workload.
CONFIG0 = dict(shape=(1, 256, 256), nD=10, n_frames=20,
               blobs=BlobSpec(200, (2.0, 8.0), (1.0, 1.0), mean=20.0), walk=WalkSpec(1.5, 6.0), seed=0)
CONFIG1 = dict(shape=(16, 512, 512), nD=32, n_frames=50,
               blobs=BlobSpec(1000, (2.0, 6.0), (1.0, 2.0), mean=30.0), walk=WalkSpec(1.0, 8.0, 0.3, 2.0), seed=1000)
CONFIG4 = dict(shape=(64, 1024, 1024), nD=64, n_frames=200,
               blobs=BlobSpec(5000, (2.0, 6.0), (1.0, 2.0), mean=15.0), walk=WalkSpec(1.0, 12.0, 0.3, 3.0), seed=4000)


def config2_acquisitions(n_per_size=64, seed=2000):
    """Batched uneven sizes: single-plane 128^2 / 256^2 / 512^2 / 1024^2 with nD 8/16/32/64."""
    out = []
    for j, (n, nD) in enumerate([(128, 8), (256, 16), (512, 32), (1024, 64)]):
        nblobs = int(200 * (n / 256) ** 2)
        out.append(make_acquisition((1, n, n), nD, n_per_size, BlobSpec(nblobs, (2.0, 8.0), (1.0, 1.0), mean=20.0),
                                    WalkSpec(1.5, 6.0), seed=seed + j))
    return out


# Served stream: eight concurrent acquisitions of different sizes.
CONFIG3_SHAPES = [(1, 256, 256), (1, 512, 512), (8, 512, 512), (16, 512, 512), (1, 1024, 1024), (32, 256, 256),
                  (32, 512, 512), (4, 1024, 1024)]


def config3_nD(shape):
    """Control points scale with the lines of a plane (16 per 256 lines), at least 2 per plane of a
    stack (so that processScanParameters keeps the inter-plane gap), at most 64."""
    nz, ny, _ = shape
    return int(min(64, max(16 * ny // 256, 2 * nz if nz > 1 else 0)))


def config3_acquisitions(n_frames=8, seed=3000, shapes=None):
    """The served-stream acquisitions: each its own blob reference; the displacement walk continues
    across consecutive frames (the case a warm start from the previous solution serves)."""
    out = []
    for j, shape in enumerate(shapes or CONFIG3_SHAPES):
        nz, ny, nx = shape
        nblobs = int(200 * ny * nx / 65536 * (1 if nz == 1 else max(1, nz // 4)))
        out.append(make_acquisition(shape, config3_nD(shape), n_frames,
                                    BlobSpec(nblobs, (2.0, 6.0), (1.0, 2.0) if nz > 1 else (1.0, 1.0), mean=20.0),
                                    WalkSpec(1.0, 8.0, 0.3 if nz > 1 else 0.0, 2.0 if nz > 1 else 0.0),
                                    seed=seed + j, continue_walk=True))
    return out


def make_config(cfg: dict, n_frames=None, shape=None, **kw) -> Acquisition:
    c = dict(cfg)
    if n_frames is not None:
        c["n_frames"] = n_frames
    if shape is not None:
        c["shape"] = shape
    c.update(kw)
    return make_acquisition(c["shape"], c["nD"], c["n_frames"], c["blobs"], c["walk"], c["seed"])

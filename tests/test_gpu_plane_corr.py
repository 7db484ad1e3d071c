"""GPU: the phase correlator's fused kx-plane passes (csrc/fa_plane_corr.cu) against a CPU DFT and
against the cuFFT path, through the C ABI test hook fa_test_correlation_surface.

The CPU statement is VolumePhaseCorrelator.cpp:57-103 in numpy FP64: square-root Hann window in x
and y, 3-D DFT, times the conjugate of the reference's DFT, divided by its modulus + DBL_MIN,
unnormalised inverse DFT. Tolerance: |surface - cpu| <= 1e-9 * max|cpu| per voxel (FP64 DFTs of
different factorisations), and the first maximum equal to the CPU surface's.
"""
import numpy as np
import pytest

import fa_b200 as fa

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    ok, msg = fa.gpu_support()
    assert ok, msg
    return fa.Context()


def _hann(n):
    if n == 1:
        return np.ones(1)
    return np.sqrt(0.5 * (1 - np.cos(2 * np.pi / (n - 1) * np.arange(n))))


def cpu_surface(reference, volume):
    nz, ny, nx = reference.shape
    w = _hann(ny)[None, :, None] * _hann(nx)[None, None, :]
    a = np.fft.fftn(volume.astype(np.float64) * w)
    b = np.fft.fftn(reference.astype(np.float64) * w)
    c = a * np.conj(b)
    c = c / (np.abs(c) + np.finfo(np.float64).tiny)
    return np.fft.ifftn(c).real * c.size


def _pair(shape, shift, seed):
    rng = np.random.default_rng(seed)
    ref = (rng.random(shape) * 1000).astype(np.float32)
    vol = np.roll(ref, shift, axis=(0, 1, 2)) + (rng.random(shape) * 50).astype(np.float32)
    return ref, vol.astype(np.float32)


PLANE_SHAPES = [(1, 8, 16), (2, 16, 16), (1, 64, 64), (4, 64, 128), (8, 32, 64), (16, 8, 32), (1, 256, 256),
                (2, 16, 512), (16, 64, 64), (1, 8, 4096), (16, 512, 512),
                # planes of 8192 points, one per pair of CTAs (a 2-CTA cluster)
                (16, 512, 64), (8, 1024, 32), (4, 2048, 16),
                # split (z, y) pass: y-line, z-column and inverse y-line kernels
                (32, 16, 16), (64, 32, 32), (16, 1024, 32), (8, 2048, 16), (64, 128, 128), (128, 16, 64)]


@pytest.mark.parametrize("shape", PLANE_SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_plane_surface_matches_cpu_dft(ctx, shape):
    nz, ny, nx = shape
    ref, vol = _pair(shape, (1 % nz, -3 % ny, 5 % nx), seed=nz * 131 + ny * 7 + nx)
    c = fa.Correlator(ctx, ref)
    want = cpu_surface(ref, vol)
    got = c.surface(vol, planes=True)
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 1e-9 * scale
    assert int(np.argmax(got)) == int(np.argmax(want))
    via_cufft = c.surface(vol, planes=False)
    assert np.abs(via_cufft - want).max() <= 1e-9 * scale
    # the integer shift the correlator reports comes from the same first maximum
    idx = np.unravel_index(int(np.argmax(want)), shape)
    expect = [idx[2] - nx if idx[2] > nx // 2 else idx[2], idx[1] - ny if idx[1] > ny // 2 else idx[1],
              idx[0] - nz if idx[0] > nz // 2 else idx[0]]
    assert np.array_equal(c.compute_shift(vol), np.array(expect, np.float64))
    c.close()


@pytest.mark.parametrize("shape", [(3, 20, 30), (32, 8, 16), (1, 4, 64), (1, 64, 12)], ids=lambda s: "x".join(map(str, s)))
def test_outside_plane_dims_uses_cufft(ctx, shape):
    ref, vol = _pair(shape, (0, 2, -1), seed=5)
    c = fa.Correlator(ctx, ref)
    with pytest.raises(fa.FaError):
        c.surface(vol, planes=True)
    want = cpu_surface(ref, vol)
    got = c.surface(vol, planes=False)
    assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max()
    c.close()


def test_host_and_device_shifts_agree(ctx):
    """Host and device entry points find the CPU surface's first maximum."""
    shape = (16, 128, 256)
    rng = np.random.default_rng(3)
    ref = (rng.random(shape) * 3000).astype(np.float32)
    c = fa.Correlator(ctx, ref)
    import torch

    frames = []
    for k in range(12):
        sh = (int(rng.integers(-3, 4)), int(rng.integers(-20, 21)), int(rng.integers(-40, 41)))
        frames.append(np.roll(ref, sh, axis=(0, 1, 2)) + (rng.random(shape) * 100).astype(np.float32))
    single = [c.compute_shift(f) for f in frames]
    dev = [torch.from_numpy(f).cuda() for f in frames]
    torch.cuda.synchronize()
    on_device = [c.compute_shift_device(t.data_ptr()) for t in dev]
    assert np.array_equal(np.array(single), np.array(on_device))
    for f, s in zip(frames, single):
        want = cpu_surface(ref, f)
        idx = np.unravel_index(int(np.argmax(want)), shape)
        expect = [v - n if v > n // 2 else v for v, n in zip((idx[2], idx[1], idx[0]), (shape[2], shape[1], shape[0]))]
        assert np.array_equal(s, np.array(expect, np.float64))
    c.close()

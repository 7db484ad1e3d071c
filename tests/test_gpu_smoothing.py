"""Gaussian pre-smoothing (smoothStack, FrameWarpAligner.cpp:46-64) on the device.

The oracle states OpenCV's documented GaussianBlur for float images (OpenCV itself is not part of
this build, so parity with it is unpinned); the device blur must equal that statement bit for bit,
which the Sobel gradient of the aligner's smoothed reference shows (Sobel is bit-exact). Aligned
displacements: RMS <= 0.01 px against the CPU solve of the same smoothed frames; correlations of
the smoothed frames: |a - b| <= 1e-9.
"""
import numpy as np
import pytest

import fa_b200 as fa
import fa_synth as S
import oracle_py as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    ok, msg = fa.gpu_support()
    assert ok, msg
    return fa.Context()


def _rms(a, b, n_dim):
    d = (np.asarray(a) - np.asarray(b))[..., :n_dim]
    return float(np.sqrt((d ** 2).sum(-1).mean()))


CASES = [((1, 96, 128), 8, 1.5, np.uint16), ((4, 40, 64), 9, 0.8, np.float32), ((3, 33, 21), 7, 2.5, np.uint16)]


@pytest.mark.parametrize("shape,nD,sigma,dtype", CASES)
def test_smoothed_reference_bitwise(ctx, shape, nD, sigma, dtype):
    acq = S.make_acquisition(shape, nD, 1, S.BlobSpec(40, (2.0, 5.0), (1.0, 2.0), mean=20.0), S.WalkSpec(1.0, 3.0),
                             seed=31)
    nz, ny, nx = shape
    line, il, ifr = acq.scan
    ref = acq.reference.astype(dtype) if dtype == np.float32 else np.round(acq.reference).astype(np.uint16)
    al = fa.Aligner(ctx, nD=nD, precision=fa.PREC_F32, smoothing=sigma)
    al.set_reference(ref, fa.scan_params(line, il, ifr, nx, ny, nz))
    g = al.reference_gradient()
    al.close()
    sm = O.smooth_stack(ref.astype(np.float32), sigma) + np.float32(1.0)
    gx, gy, gz = O.sobel3d(sm)
    assert np.array_equal(g[0], gx) and np.array_equal(g[1], gy) and np.array_equal(g[2], gz)


@pytest.mark.parametrize("precision", [fa.PREC_F32, fa.PREC_MIXED])
def test_smoothed_alignment_against_oracle(ctx, precision):
    sigma = 1.2
    acq = S.make_acquisition((1, 128, 128), 8, 3, S.BlobSpec(60, (2.0, 6.0), (1.0, 1.0), mean=20.0),
                             S.WalkSpec(1.0, 3.0), seed=33)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    raw = np.ascontiguousarray(acq.frames.astype(np.uint16))
    al = fa.Aligner(ctx, nD=acq.nD, precision=precision, smoothing=sigma)
    al.set_reference(acq.reference, fa.scan_params(line, il, ifr, nx, ny, nz))
    D, _ = al.add_frames([raw[k] for k in range(3)])
    res = al.results([raw[k] for k in range(3)], D)
    al.close()
    sref = O.smooth_stack(acq.reference.astype(np.float32), sigma) + np.float32(1.0)
    ow = O.OracleWarper(sref, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
    for k in range(3):
        frame = raw[k].astype(np.float32)
        sm = O.smooth_stack(frame, sigma) + np.float32(1.0)
        shift = O.phase_shift(acq.reference, frame)  # the rigid start uses the raw data
        D_cpu, _ = ow.align_frame(sm, shift, 100)
        assert _rms(D[k], D_cpu, 2) <= 0.01, (k, _rms(D[k], D_cpu, 2))
        _, cov = ow.warp_image(frame, D[k])
        m = (cov > 0).astype(np.uint8)
        unal = O.correlation(sm.ravel(), sref.ravel(), m.ravel())
        assert abs(res[k]["unaligned_correlation"] - unal) <= 1e-9


def test_smoothed_server_equals_aligner(ctx):
    sigma = 1.2
    acq = S.make_acquisition((2, 64, 96), 5, 4, S.BlobSpec(40, (2.0, 5.0), (1.0, 2.0), mean=20.0),
                             S.WalkSpec(1.0, 3.0, 0.2, 1.0), seed=35)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    scan = fa.scan_params(line, il, ifr, nx, ny, nz)
    raw = np.ascontiguousarray(acq.frames.astype(np.uint16))
    al = fa.Aligner(ctx, nD=acq.nD, precision=fa.PREC_MIXED, smoothing=sigma)
    al.set_reference(acq.reference, scan)
    D, _ = al.add_frames([raw[k] for k in range(4)])
    al.close()
    srv = fa.Server(ctx, warm_start=False)
    aid = srv.add_acquisition(acq.reference, scan, frame_dtype=np.uint16, nD=acq.nD, smoothing=sigma)
    got = [srv.wait(srv.submit(aid, raw[k]), 120.0)[0] for k in range(4)]
    srv.close()
    assert np.max(np.abs(np.array(got) - D)) <= 1e-9

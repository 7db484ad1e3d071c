"""The aligner's batched solve as it runs on the device: rigid starts taken from the device
phase-correlation peaks (unravelled, wrapped and scaled by the binning without a host read), the
solve repeated by a while-conditional graph node until no frame is active or the iteration limit is
reached, and several solve groups queued at once.

Tolerances: D within 0.01 px RMS of the CPU solve of the same frames from the same integer
phase-correlation peak and with the same iteration limit (FrameWarpAligner.cpp:140-219, the
trust region's max_iter); the iteration count of every frame at most the limit. Host and
device-resident inputs of the same frames give identical D (the same kernels on the same values).
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


def _scan(acq):
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    return fa.scan_params(line, il, ifr, nx, ny, nz)


@pytest.mark.parametrize("max_iterations", [1, 2, 100])
def test_iteration_limit(ctx, max_iterations):
    """A small limit ends the device-side loop with the trust region's own max_iter rule: every frame
    stops at the limit or earlier, with the CPU solve's D under the same limit."""
    import torch

    n = 4
    acq = S.make_acquisition((4, 96, 128), 13, n, S.BlobSpec(60, (2.0, 6.0), (1.0, 2.0), mean=25.0),
                             S.WalkSpec(1.0, 4.0, 0.3, 0.8), seed=55)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    al = fa.Aligner(ctx, nD=acq.nD, precision=fa.PREC_F32, max_iterations=max_iterations)
    al.set_reference(acq.reference, _scan(acq))
    raw = np.ascontiguousarray(acq.frames.astype(np.uint16))
    D, st = al.add_frames([raw[k] for k in range(n)])
    dev = torch.from_numpy(raw.view(np.int16)).to("cuda:0")
    torch.cuda.synchronize()
    D_dev, st_dev = al.add_frames_device([dev[k].data_ptr() for k in range(n)], fa.U16, n)
    assert np.array_equal(D, D_dev)
    ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
    for k in range(n):
        assert 1 <= st[k]["iterations"] <= max_iterations, (k, st[k])
        assert st[k]["iterations"] == st_dev[k]["iterations"]
        shift = O.phase_shift(acq.reference, acq.frames[k])
        D_cpu, _ = ow.align_frame(acq.frames[k] + 1, shift, max_iterations)
        r = _rms(D[k], D_cpu, 3)
        assert r <= 0.01, (k, max_iterations, r)
    if max_iterations == 1:
        assert any(s["status"] == 1 for s in st)  # at least one frame was stopped by the limit
    corr_ms, total_ms = al.last_phase_ms()
    assert 0.0 < corr_ms <= total_ms
    al.close()


def test_two_solve_groups_queued_at_once(ctx):
    """20 frames are solved in two groups (the first overlapping the second's uploads and
    correlation, both queued before the host waits): D against the CPU solve of every frame, and
    identical for the same frames given from host and from device memory."""
    import torch

    n = 20
    acq = S.make_acquisition((1, 96, 128), 8, n, S.BlobSpec(50, (2.0, 6.0), (1.0, 1.0), mean=25.0),
                             S.WalkSpec(1.0, 4.0), seed=56)
    al = fa.Aligner(ctx, nD=acq.nD, precision=fa.PREC_MIXED)
    al.set_reference(acq.reference, _scan(acq))
    raw = np.ascontiguousarray(acq.frames.astype(np.uint16))
    D, st = al.add_frames([raw[k] for k in range(n)])
    dev = torch.from_numpy(raw.view(np.int16)).to("cuda:0")
    torch.cuda.synchronize()
    D_dev, _ = al.add_frames_device([dev[k].data_ptr() for k in range(n)], fa.U16, n)
    assert np.array_equal(D, D_dev)
    shifts = np.array([O.phase_shift(acq.reference, acq.frames[k]) for k in range(n)])
    if O.ref_available():
        line, il, ifr = acq.scan
        D_cpu = O.RefPool(acq.reference + 1, acq.nD, line, il, ifr, 8).align(acq.frames + 1, shifts, 100)[0]
    else:
        nz, ny, nx = acq.reference.shape
        line, il, ifr = acq.scan
        ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
        D_cpu = ow.align_frames_mt(acq.frames + 1, shifts, 8, 100)[0]
    for k in range(n):
        r = _rms(D[k], D_cpu[k], 2)
        assert r <= 0.01, (k, r)
        assert st[k]["iterations"] >= 1
    al.close()


@pytest.mark.parametrize("factor", [2, 3])
def test_device_peak_start_wraps_and_scales(ctx, factor):
    """Rigid starts from device peaks: frames shifted by known whole-pixel amounts in both directions
    (negative shifts wrap to the upper half of the correlation surface) with binning; the recovered
    D against the CPU solve from the CPU phase correlation of the downsampled volumes, x and y
    scaled by the factor (FrameWarpAligner.cpp:186-188)."""
    nz, ny, nx = 1, 120, 144
    acq = S.make_acquisition((nz, ny, nx), 8, 1, S.BlobSpec(70, (2.0, 6.0), (1.0, 1.0), mean=25.0),
                             S.WalkSpec(0.3, 1.0), seed=57)
    frames = []
    for dy, dx in [(-7, 5), (6, -9), (0, 0)]:
        frames.append(np.roll(acq.frames[0], (dy, dx), axis=(1, 2)))
    frames = np.stack(frames)
    al = fa.Aligner(ctx, spatial_binning=factor, nD=acq.nD, precision=fa.PREC_F32)
    al.set_reference(acq.reference, _scan(acq))
    D, _ = al.add_frames([np.ascontiguousarray(f.astype(np.uint16)) for f in frames])
    ds_ref = O.downsample(acq.reference, factor)
    shifts = np.array([O.phase_shift(ds_ref, O.downsample(f, factor)) for f in frames])
    shifts[:, :2] *= factor
    line, il, ifr = acq.scan
    ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
    for k in range(len(frames)):
        D_cpu, _ = ow.align_frame(frames[k] + 1, shifts[k], 100)
        r = _rms(D[k], D_cpu, 2)
        assert r <= 0.01, (k, shifts[k], r)
    al.close()


@pytest.mark.parametrize("precision", [fa.PREC_MIXED, fa.PREC_F32], ids=["mixed", "f32"])
def test_slots_written_by_the_correlator(ctx, precision):
    """Without smoothing or binning the phase correlator's first pass writes each frame + 1 into its
    slot as it reads the frame: raw uint16 counts (saturated) from uint16 frames and FP16 values from
    FP32 frames in mixed precision, FP32 values in FP32 precision. The same counts given as uint16 and
    as FP32 frames fill slots with the same values (counts below 2048 are exact in FP16), so D is
    identical; host and device inputs give identical D; and D is within 0.01 px of the CPU solve
    (the reference's 256 x 256 single-plane case, nD = 10)."""
    import torch

    n = 3
    acq = S.make_config(S.CONFIG0, n_frames=n)
    assert acq.frames.max() + 1 < 2048
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    al = fa.Aligner(ctx, nD=acq.nD, precision=precision)
    al.set_reference(acq.reference, _scan(acq))
    Ds = []
    for dtype, view, kind in ((np.uint16, np.int16, fa.U16), (np.float32, np.float32, fa.F32)):
        host = np.ascontiguousarray(acq.frames.astype(dtype))
        D, _ = al.add_frames([host[k] for k in range(n)])
        dev = torch.from_numpy(host.view(view)).to("cuda:0")
        torch.cuda.synchronize()
        D_dev, _ = al.add_frames_device([dev[k].data_ptr() for k in range(n)], kind, n)
        assert np.array_equal(D, D_dev)
        Ds.append(D)
    assert np.array_equal(Ds[0], Ds[1])
    ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
    for k in range(n):
        shift = O.phase_shift(acq.reference, acq.frames[k])
        D_cpu, _ = ow.align_frame(acq.frames[k] + 1, shift, 100)
        r = _rms(Ds[0][k], D_cpu, 2)
        assert r <= 0.01, (k, r)
    al.close()

"""GPU parity of the mixed-precision path the headline figures time, and of the aligner options the
other parity tests leave out.

Tolerances (stated per quantity):
  * recovered displacements: RMS over control points <= 0.01 px against the CPU solve of the same
    frames (the reference's own CpuFrameWarper compiled from its sources when present, otherwise the
    restated oracle), starting from the same integer phase-correlation peak;
  * reduction error of one evaluation, against an FP64 statement of the same evaluation
    (oracle_py.fp64_error_jacobian):
      - summation only (the FP64 statement fed the very values the device stores: BF16 reference and
        gradient, FP16 frame): f relative 5e-6, J^T e 5e-5 of max|J^T e|. The device sums the terms
        of one lane of one tile in FP32 (fused multiply-add; tile voxels / 32 terms, 128 for the
        default 4096-voxel tiles), then pairwise across the 32 lanes of a warp (shuffle tree), then
        in FP64 across tiles: blocked pairwise summation, whose error grows with the block length,
        not with the voxel count;
      - storage included (the FP64 statement on the FP32 reference, gradient and frame): f relative
        1e-3, J^T e 2e-3 of max|J^T e| (BF16 keeps 8 significant bits of each reference and gradient
        value);
      - the FP32 path (FP32 storage) against the same FP64 statement: f 2e-6, J^T e 2e-5;
  * downsample (spatial_binning > 1): bit-exact against the reference's loop order.
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


def _cpu_solve(acq, frames_plus1, shifts, n_threads=None):
    """CPU solves of the +1 frames from the given rigid shifts: the reference build (RefPool) when it
    is present, else the restated oracle; one frame per thread."""
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    n = frames_plus1.shape[0]
    t = n_threads or n
    if O.ref_available():
        return O.RefPool(acq.reference + 1, acq.nD, line, il, ifr, t).align(frames_plus1, shifts, 100)[0]
    ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
    return ow.align_frames_mt(frames_plus1, shifts, t, 100)[0]


def test_headline_aligner_mixed_u16_512x512x16(ctx):
    """The path the headline `value` times: fa_aligner_add_frames_device, mixed precision (BF16
    reference and gradient, raw uint16 frames decoded in the fused pass), 512x512x16, nD = 32, three
    displacement components, four frames in one batched solve; the device phase-correlation start
    and trust region against the CPU solve of the same frames (FrameWarper.cpp:4-69,147-167;
    FrameWarpAligner.cpp:140-219)."""
    import torch

    n = 4
    acq = S.make_config(S.CONFIG1, n_frames=n)
    al = fa.Aligner(ctx, nD=acq.nD, precision=fa.PREC_MIXED)
    al.set_reference(acq.reference, _scan(acq))
    raw = np.ascontiguousarray(acq.frames.astype(np.uint16))
    dev = torch.from_numpy(raw.view(np.int16)).to("cuda:0")
    torch.cuda.synchronize()
    D, st = al.add_frames_device([dev[k].data_ptr() for k in range(n)], fa.U16, n)
    shifts = np.array([O.phase_shift(acq.reference, acq.frames[k]) for k in range(n)])
    D_cpu = _cpu_solve(acq, acq.frames[:n] + 1, shifts)
    for k in range(n):
        r = _rms(D[k], D_cpu[k], 3)
        assert r <= 0.01, (k, r)
        assert st[k]["iterations"] >= 1
    al.close()


@pytest.mark.parametrize("shape,nD", [((1, 256, 256), 10), ((4, 96, 128), 13), ((16, 128, 128), 32)])
def test_mixed_reduction_error_bounds(ctx, shape, nD):
    acq = S.make_acquisition(shape, nD, 1, S.BlobSpec(int(200 * shape[1] * shape[2] / 65536) + 20, (2.0, 6.0),
                                                      (1.0, 2.0), mean=30.0),
                             S.WalkSpec(1.0, 4.0, 0.3 if shape[0] > 1 else 0.0, 1.0 if shape[0] > 1 else 0.0),
                             seed=77)
    nz, ny, nx = shape
    line, il, ifr = acq.scan
    ref_p1 = acq.reference + 1
    ow = O.OracleWarper(ref_p1, nD, O.scan_init(line, il, ifr, nx, ny, nz))
    grad = ow.gradient()
    frame = (acq.frames[0] + 1).astype(np.float32)
    rounded = [O.round_bf16(ref_p1), [O.round_bf16(g) for g in grad], frame.astype(np.float16).astype(np.float32)]
    mixed = fa.Reference(ctx, ref_p1, nD, _scan(acq), fa.PREC_MIXED)
    plain = fa.Reference(ctx, ref_p1, nD, _scan(acq), fa.PREC_F32)
    fm = fa.Frame(mixed, frame.astype(np.float16))
    fp = fa.Frame(plain, frame)
    rng = np.random.Generator(np.random.PCG64(8))
    for D in (np.zeros((nD, 3)), acq.D_true[0] + rng.normal(0, 0.3, (nD, 3))):
        if nz == 1:
            D[:, 2] = 0.0
        f_st, g_st = O.fp64_error_jacobian(ow, rounded[0], rounded[1], rounded[2], D)
        f_64, g_64 = O.fp64_error_jacobian(ow, ref_p1, grad, frame, D)
        f_m, g_m = fm.get_error(D), fm.get_jacobian(D)
        f_p, g_p = fp.get_error(D), fp.get_jacobian(D)
        # summation error of the mixed pass (same stored values)
        assert abs(f_m - f_st) <= 5e-6 * f_st, (f_m, f_st)
        assert np.max(np.abs(g_m - g_st)) <= 5e-5 * np.max(np.abs(g_st))
        # total error of the mixed pass (storage rounding included)
        assert abs(f_m - f_64) <= 1e-3 * f_64, (f_m, f_64)
        assert np.max(np.abs(g_m - g_64)) <= 2e-3 * np.max(np.abs(g_64))
        # the FP32 pass against the same FP64 statement
        assert abs(f_p - f_64) <= 2e-6 * f_64, (f_p, f_64)
        assert np.max(np.abs(g_p - g_64)) <= 2e-5 * np.max(np.abs(g_64))
    for h in (fm, fp, mixed, plain):
        h.close()


def test_uneven_sizes_one_frame_each(ctx):
    """The batched uneven workload's four single-plane sizes (128^2 ... 1024^2, nD 8 / 16 / 32 / 64),
    mixed precision with raw uint16 frames through the aligner: one frame per size against the CPU
    solve of the same frame."""
    for acq in S.config2_acquisitions(n_per_size=1):
        al = fa.Aligner(ctx, nD=acq.nD, precision=fa.PREC_MIXED)
        al.set_reference(acq.reference, _scan(acq))
        D, _ = al.add_frames([np.ascontiguousarray(acq.frames[0].astype(np.uint16))])
        shift = O.phase_shift(acq.reference, acq.frames[0])
        D_cpu = _cpu_solve(acq, acq.frames[:1] + 1, shift[None])
        r = _rms(D[0], D_cpu[0], 2)
        assert r <= 0.01, (acq.reference.shape, r)
        al.close()


@pytest.mark.parametrize("shape", [(1, 97, 130), (3, 50, 63), (2, 64, 64)])
@pytest.mark.parametrize("factor", [2, 3])
def test_downsample_matches_reference_loop(ctx, shape, factor):
    """downsample (AbstractFrameAligner.cpp:37-56): float sums of factor x factor blocks in the
    reference's loop order, ceil-sized, ragged last blocks; float32 and uint16 inputs."""
    rng = np.random.Generator(np.random.PCG64(sum(shape) * factor))
    vol = rng.gamma(2.0, 12.0, shape).astype(np.float32)
    assert np.array_equal(fa.test_downsample(ctx, vol, factor), O.downsample(vol, factor))
    counts = rng.poisson(40.0, shape).astype(np.uint16)
    assert np.array_equal(fa.test_downsample(ctx, counts, factor), O.downsample(counts.astype(np.float32), factor))


@pytest.mark.parametrize("shape,nD", [((1, 97, 130), 10), ((4, 66, 90), 13)])
@pytest.mark.parametrize("factor", [2, 3])
def test_aligner_spatial_binning(ctx, shape, nD, factor):
    """RealignmentParameters::spatial_binning > 1: the phase correlation runs on the downsampled raw
    reference and frame, and the rigid start's x and y are multiplied by the factor
    (FrameWarpAligner.cpp:92-98,160,186-188); the solve then runs at full resolution. D within
    0.01 px of the CPU solve from the same scaled shift."""
    nz, ny, nx = shape
    acq = S.make_acquisition(shape, nD, 2, S.BlobSpec(60, (2.0, 6.0), (1.0, 2.0), mean=25.0),
                             S.WalkSpec(1.0, 4.0, 0.2 if nz > 1 else 0.0, 0.8 if nz > 1 else 0.0), seed=41 + factor)
    for precision in (fa.PREC_F32, fa.PREC_MIXED):
        al = fa.Aligner(ctx, spatial_binning=factor, nD=nD, precision=precision)
        al.set_reference(acq.reference, _scan(acq))
        D, _ = al.add_frames([np.ascontiguousarray(acq.frames[k].astype(np.uint16)) for k in range(2)])
        ds_ref = O.downsample(acq.reference, factor)
        shifts = np.array([O.phase_shift(ds_ref, O.downsample(acq.frames[k], factor)) for k in range(2)])
        shifts[:, :2] *= factor
        D_cpu = _cpu_solve(acq, acq.frames[:2] + 1, shifts)
        for k in range(2):
            r = _rms(D[k], D_cpu[k], 3 if nz > 1 else 2)
            assert r <= 0.01, (precision, k, r)
        al.close()

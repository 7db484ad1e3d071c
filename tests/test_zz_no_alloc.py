"""fa_get_error_jacobian_static: the fused error + J^T e evaluation for callers that cannot
allocate device memory when they evaluate a frame (a host application that has reserved the device
memory pool for its own allocator, or a real-time acquisition loop that must not allocate between
frames). The frame lives in the caller's own device memory (allocated here through torch, as such a
caller's framework would), and all scratch lives in the library's fixed static device array.

The results must match the registered-frame path (fa_get_error / fa_get_jacobian) within the
tolerances of the parity tests -- f: 2e-6 relative, J^T e: 2e-5 of max|J^T e| -- on two calls in a
row, which also checks that the second call does not see stale contents of the shared array. The
cases cover rows that are a multiple of 4 voxels (the four-voxels-per-lane kernel), rows that are not
and a frame pointer that is not 16-byte aligned (both take the one-voxel-per-thread kernel), and more
than 64 control points (the host stages the control-point parameters in chunks of 64). Invalid
calls -- a D with a non-finite entry, a volume whose scratch exceeds the array -- are rejected with
FA_ERR_BAD_ARG before any device work.
This file is collected last so that a run stopping at the first failure has run every other test."""
import numpy as np
import pytest

import fa_b200 as fa
import fa_synth as S

pytestmark = pytest.mark.gpu


def _ctx():
    ok, msg = fa.gpu_support()
    assert ok, msg
    return fa.Context()


@pytest.mark.parametrize("shape,nD,offset", [((4, 96, 128), 13, 0), ((1, 160, 192), 9, 0), ((1, 40, 30), 6, 0),
                                             ((2, 48, 64), 7, 1), ((1, 256, 128), 70, 0)])
@pytest.mark.parametrize("precision", [fa.PREC_F32, fa.PREC_MIXED])
def test_static_scratch_matches_registered_frame(shape, nD, offset, precision):
    import torch

    ctx = _ctx()
    acq = S.make_acquisition(shape, nD, 2, S.BlobSpec(60, (2.0, 6.0), (1.0, 2.0)), S.WalkSpec(1.0, 3.0, 0.2, 0.8),
                             seed=31)
    nz, ny, nx = shape
    line, il, ifr = acq.scan
    ref = fa.Reference(ctx, acq.reference + 1, nD, fa.scan_params(line, il, ifr, nx, ny, nz), precision)
    np_dtype, dtype = (np.float32, fa.F32) if precision == fa.PREC_F32 else (np.float16, fa.F16)
    view = np.int32 if np_dtype == np.float32 else np.int16
    rng = np.random.Generator(np.random.PCG64(4))
    for k in range(2):  # two calls in a row, different frames and displacements
        host = np.ascontiguousarray((acq.frames[k] + 1).astype(np_dtype))
        frame = fa.Frame(ref, host)
        # the caller's buffer, optionally starting `offset` elements into a torch allocation
        buf = torch.zeros(host.size + offset, dtype=torch.int32 if view == np.int32 else torch.int16,
                          device="cuda:0")
        buf[offset:] = torch.from_numpy(host.view(view).ravel()).to("cuda:0")
        torch.cuda.synchronize()
        ptr = buf.data_ptr() + offset * host.itemsize
        assert (ptr % 16 != 0) == (offset != 0)
        D = acq.D_true[k] + rng.normal(0, 0.4, acq.D_true[k].shape)
        if nz == 1:
            D[:, 2] = 0.0
        f_ref = frame.get_error(D)
        j_ref = frame.get_jacobian(D)
        f_s, j_s = fa.get_error_jacobian_static(ref, ptr, dtype, D)
        assert abs(f_s - f_ref) <= 2e-6 * abs(f_ref), (k, f_s, f_ref)
        assert np.max(np.abs(j_s - j_ref)) <= 2e-5 * np.max(np.abs(j_ref)), k
        frame.close()
    assert torch.cuda.current_device() == 0
    ref.close()


def test_static_scratch_rejects_bad_calls():
    import torch

    ctx = _ctx()
    acq = S.make_acquisition((1, 64, 64), 6, 1, S.BlobSpec(30, (2.0, 6.0), (1.0, 1.0)), S.WalkSpec(1.0, 3.0), seed=32)
    line, il, ifr = acq.scan
    ref = fa.Reference(ctx, acq.reference + 1, 6, fa.scan_params(line, il, ifr, 64, 64, 1))
    dev = torch.from_numpy((acq.frames[0] + 1).astype(np.float32)).to("cuda:0")
    D = np.zeros((6, 3))
    D[2, 1] = np.nan
    with pytest.raises(fa.FaError) as e:
        fa.get_error_jacobian_static(ref, dev.data_ptr(), fa.F32, D)
    assert e.value.status == 1 and "non-finite" in str(e.value)
    with pytest.raises(fa.FaError) as e:  # an FP32 reference takes FP32 frames
        fa.get_error_jacobian_static(ref, dev.data_ptr(), fa.F16, np.zeros((6, 3)))
    assert e.value.status == 1
    ref.close()
    # 24000 one-row tiles of 32 voxels: 24000 x 96 bytes of partial sums exceed the 2 MiB array
    ny, nx = 24000, 32
    big = np.full((1, ny, nx), 5.0, np.float32) + np.arange(nx, dtype=np.float32)[None, None, :] * 0.1
    line, il, ifr = S.scan_durations(1, ny, nx, 10)[:3]
    ref = fa.Reference(ctx, big, 10, fa.scan_params(line, il, ifr, nx, ny, 1))
    ref.retune(nx, 2)
    frame = torch.from_numpy(big).to("cuda:0")
    with pytest.raises(fa.FaError) as e:
        fa.get_error_jacobian_static(ref, frame.data_ptr(), fa.F32, np.zeros((10, 3)))
    assert e.value.status == 1 and "static scratch" in str(e.value)
    ref.close()

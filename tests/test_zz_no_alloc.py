"""fa_get_error_jacobian_static: the fused error + J^T e evaluation for callers that cannot
allocate device memory when they evaluate a frame (a host application that has reserved the device
memory pool for its own allocator, or a real-time acquisition loop that must not allocate between
frames). The frame lives in the caller's own device memory (allocated here through torch, as such a
caller's framework would), and all scratch lives in the library's fixed static device array.

The results must match the registered-frame path (fa_get_error / fa_get_jacobian) within the
tolerances of the parity tests -- f: 2e-6 relative, J^T e: 2e-5 of max|J^T e| -- on two calls in a
row, which also checks that the second call does not see stale contents of the shared array.
This file is collected last so that a run stopping at the first failure has run every other test."""
import numpy as np
import pytest

import fa_b200 as fa
import fa_synth as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,nD", [((4, 96, 128), 13), ((1, 160, 192), 9)])
@pytest.mark.parametrize("precision", [fa.PREC_F32, fa.PREC_MIXED])
def test_static_scratch_matches_registered_frame(shape, nD, precision):
    import torch

    ok, msg = fa.gpu_support()
    assert ok, msg
    ctx = fa.Context()
    acq = S.make_acquisition(shape, nD, 2, S.BlobSpec(60, (2.0, 6.0), (1.0, 2.0)), S.WalkSpec(1.0, 3.0, 0.2, 0.8),
                             seed=31)
    nz, ny, nx = shape
    line, il, ifr = acq.scan
    ref = fa.Reference(ctx, acq.reference + 1, nD, fa.scan_params(line, il, ifr, nx, ny, nz), precision)
    np_dtype, dtype = (np.float32, fa.F32) if precision == fa.PREC_F32 else (np.float16, fa.F16)
    rng = np.random.Generator(np.random.PCG64(4))
    for k in range(2):  # two calls in a row, different frames and displacements
        host = np.ascontiguousarray((acq.frames[k] + 1).astype(np_dtype))
        frame = fa.Frame(ref, host)
        dev = torch.from_numpy(host.view(np.int32 if np_dtype == np.float32 else np.int16)).to("cuda:0")
        torch.cuda.synchronize()
        D = acq.D_true[k] + rng.normal(0, 0.4, acq.D_true[k].shape)
        if nz == 1:
            D[:, 2] = 0.0
        f_ref = frame.get_error(D)
        j_ref = frame.get_jacobian(D)
        f_s, j_s = fa.get_error_jacobian_static(ref, dev.data_ptr(), dtype, D)
        assert abs(f_s - f_ref) <= 2e-6 * abs(f_ref), (k, f_s, f_ref)
        assert np.max(np.abs(j_s - j_ref)) <= 2e-5 * np.max(np.abs(j_ref)), k
        frame.close()

"""The large-volume workload on the GPU: 1024x1024x64 reference (5000 blobs, mean 15 photons),
nD = 64, three displacement components (random walk bounded at 12 px in x/y and 3 planes in z),
raw uint16 frames through the full aligner pipeline -- 3-D FP64 phase correlation of the whole
volume, then the batched mixed-precision solve -- against the CPU solve of the same frames from the
same integer peak (VolumePhaseCorrelator.cpp:57-139; FrameWarper.cpp:4-69,147-167;
FrameWarpAligner.cpp:140-219). Tolerance: displacement RMS over control points <= 0.01 px."""
import numpy as np
import pytest

import fa_b200 as fa
import fa_synth as S
import oracle_py as O

pytestmark = pytest.mark.gpu


def test_large_volume_two_frames_against_cpu():
    import torch

    ok, msg = fa.gpu_support()
    assert ok, msg
    ctx = fa.Context()
    n = 2
    acq = S.make_config(S.CONFIG4, n_frames=n)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    al = fa.Aligner(ctx, nD=acq.nD, precision=fa.PREC_MIXED)
    al.set_reference(acq.reference, fa.scan_params(line, il, ifr, nx, ny, nz))
    raw = np.ascontiguousarray(acq.frames.astype(np.uint16))
    dev = torch.from_numpy(raw.view(np.int16)).to("cuda:0")
    torch.cuda.synchronize()
    D, st = al.add_frames_device([dev[k].data_ptr() for k in range(n)], fa.U16, n)
    al.close()
    del dev
    torch.cuda.empty_cache()
    shifts = np.array([O.phase_shift(acq.reference, acq.frames[k]) for k in range(n)])
    if O.ref_available():
        D_cpu, _ = O.RefPool(acq.reference + 1, acq.nD, line, il, ifr, n).align(acq.frames + 1, shifts, 100)
    else:
        ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
        D_cpu, _ = ow.align_frames_mt(acq.frames + 1, shifts, n, 100)
    for k in range(n):
        rms = float(np.sqrt(((D[k] - D_cpu[k]) ** 2).sum(-1).mean()))
        assert rms <= 0.01, (k, rms)
        assert st[k]["iterations"] >= 1

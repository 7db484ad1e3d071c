"""Generates tests/golden/*.npz from the reference's own warper sources.

Run in a container that has the reference tree: ``make -C oracle`` builds oracle/_ref/libfa_ref.so
from FrameAligner/FrameWarper.cpp, Sobel3d.cpp, VolumePhaseCorrelator.cpp and OptimisationModel.cpp
(compiled unchanged against the stand-ins in oracle/ref_shim/), then::

    python tests/golden/make_golden.py

Each fixture holds seeded inputs and the reference's outputs for them: the precomputed interval
tables (Di, Df, D_range), the Sobel gradients, the Gauss-Newton Hessian, the error sum and J^T e
at two displacement sets, the interpolated and intensity-preserving warps, warpPoint samples, the
phase-correlation integer shift, and the full per-frame solve driven by the oracle's trust region.
The tests compare the oracle (fa_oracle.c) and the CUDA library against these files, so neither
needs the reference tree at run time.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "frame-aligner_b200"))

import fa_synth as S  # noqa: E402
import oracle_py as O  # noqa: E402

CASES = {
    # name: (shape, nD, blobs, walk, seed, bidirectional)
    "plane_48x40_nD6": ((1, 40, 48), 6, S.BlobSpec(14, (2.0, 5.0), (1.0, 1.0)), S.WalkSpec(1.0, 3.0), 11, False),
    "plane_64x64_nD10": ((1, 64, 64), 10, S.BlobSpec(25, (2.0, 6.0), (1.0, 1.0)), S.WalkSpec(1.5, 4.0), 12, False),
    "stack_32x24x4_nD9": ((4, 24, 32), 9, S.BlobSpec(12, (2.0, 5.0), (1.0, 2.0)), S.WalkSpec(1.0, 3.0, 0.3, 1.0),
                          13, False),
    "stack_33x21x3_nD7_odd": ((3, 21, 33), 7, S.BlobSpec(10, (2.0, 4.0), (1.0, 2.0)),
                              S.WalkSpec(0.8, 2.5, 0.2, 0.8), 14, False),
    "plane_40x30_nD5_bidir": ((1, 30, 40), 5, S.BlobSpec(10, (2.0, 4.0), (1.0, 1.0)), S.WalkSpec(1.0, 3.0), 15, True),
    "stack_16x16x2_nD4": ((2, 16, 16), 4, S.BlobSpec(6, (1.5, 3.0), (1.0, 1.5)), S.WalkSpec(0.7, 2.0, 0.2, 0.5),
                          16, False),
}


def make_case(name, shape, nD, blobs, walk, seed, bidir):
    nz, ny, nx = shape
    acq = S.make_acquisition(shape, nD, 2, blobs, walk, seed)
    line, interline, interframe = acq.scan
    ref = (acq.reference + 1).astype(np.float32)
    frame = (acq.frames[0] + 1).astype(np.float32)
    rw = O.RefWarper(ref, nD, line, interline, interframe, bidirectional=bidir)
    rw.set_frame(frame)
    out = dict(reference=ref, frame=frame, raw_reference=acq.reference.astype(np.float32),
               raw_frame=acq.frames[0].astype(np.float32), D_true=acq.D_true[0], nD=np.int32(nD),
               scan=np.array([line, interline, interframe], np.float64), bidirectional=np.int32(bidir))
    Di, Df, ranges = rw.precomp()
    out.update(Di=Di, Df=Df, ranges=ranges)
    gx, gy, gz = O.ref_sobel3d(ref)
    out.update(gx=gx, gy=gy, gz=gz)
    out["H"] = rw.hessian()
    rng = np.random.Generator(np.random.PCG64(seed + 500))
    D_a = acq.D_true[0].copy()
    D_b = acq.D_true[0] + rng.normal(0, 0.7, size=acq.D_true[0].shape)
    if nz == 1:
        D_b[:, 2] = 0.0
    for tag, D in (("a", D_a), ("b", D_b)):
        out[f"D_{tag}"] = D
        out[f"f_{tag}"] = np.float64(rw.get_error(D))
        out[f"jac_{tag}"] = rw.get_jacobian(D)
        out[f"warp0_{tag}"] = rw.warp_interpolated(D, 0)
        out[f"warpm1_{tag}"] = rw.warp_interpolated(D, -1)
        w, c = rw.warp_image(D)
        out[f"splat_{tag}"] = w
        out[f"coverage_{tag}"] = c
    pts = [(0, 0, 0), (nx - 1, ny - 1, nz - 1), (nx // 2, ny // 3, nz // 2), (3, 1, 0)]
    out["warp_point_xyz"] = np.array(pts, np.int32)
    out["warp_point"] = np.array([rw.warp_point(D_b, *p) for p in pts])
    shift = O.ref_phase_shift(acq.reference, acq.frames[0])
    out["phase_shift"] = shift
    D_solve, iters = rw.align_frame(frame, shift, max_iter=100)
    out["D_solve"] = D_solve
    out["solve_iterations"] = np.int32(iters)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return out


def make_phase_cases():
    """Known circular shifts of a blob volume, including the +-n/2 wrap boundary."""
    out = {}
    rng = np.random.Generator(np.random.PCG64(77))
    for shape in [(1, 32, 32), (4, 16, 24), (1, 20, 17)]:
        nz, ny, nx = shape
        acq = S.make_acquisition(shape, 2 * nz + 1, 1, S.BlobSpec(8, (1.5, 3.0), (1.0, 1.5)), S.WalkSpec(0.0, 0.0),
                                 seed=int(rng.integers(1 << 30)), poisson=False)
        ref = acq.reference
        for sx, sy, sz in [(3, -2, 0), (nx // 2, ny // 2, nz // 2), (-(nx // 2) + 1, 1, -(nz // 2)), (0, 0, 0)]:
            vol = np.roll(ref, shift=(sz, sy, sx), axis=(0, 1, 2)).astype(np.float32)
            key = f"{nz}x{ny}x{nx}_{sx}_{sy}_{sz}"
            out[f"ref_{key}"] = ref.astype(np.float32)
            out[f"vol_{key}"] = vol
            out[f"shift_{key}"] = O.ref_phase_shift(ref, vol)
    np.savez_compressed(os.path.join(HERE, "phase_shifts.npz"), **out)


if __name__ == "__main__":
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libfa_ref.so missing: run make -C oracle in a container with the reference")
    for name, args in CASES.items():
        make_case(name, *args)
        print("wrote", name)
    make_phase_cases()
    print("wrote phase_shifts")

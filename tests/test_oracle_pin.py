"""Pins the CPU oracle (oracle/fa_oracle.c) to the reference.

Against the committed golden fixtures (outputs of the reference's own FrameWarper.cpp, Sobel3d.cpp,
VolumePhaseCorrelator.cpp and OptimisationModel.cpp, see tests/golden/make_golden.py) every
quantity must be bit-identical. When oracle/_ref/libfa_ref.so is present the same comparison also
runs live on further seeded cases.
"""
import numpy as np
import pytest

import fa_synth as S
import oracle_py as O
from conftest import load_golden


def _warper(g):
    ref = g["reference"]
    nz, ny, nx = ref.shape
    line, interline, interframe = g["scan"]
    sc = O.scan_init(line, interline, interframe, nx, ny, nz, bool(g["bidirectional"]))
    return O.OracleWarper(ref, int(g["nD"]), sc)


def test_precompute_tables(golden):
    name, g = golden
    Di, Df, ranges = _warper(g).precomp()
    assert np.array_equal(Di, g["Di"])
    assert np.array_equal(Df, g["Df"])
    # The last D_range entry is never set by the reference (value-initialised to {0, 0}).
    assert np.array_equal(ranges, g["ranges"])


def test_sobel_gradient(golden):
    _, g = golden
    gx, gy, gz = O.sobel3d(g["reference"])
    assert np.array_equal(gx, g["gx"]) and np.array_equal(gy, g["gy"]) and np.array_equal(gz, g["gz"])
    wx, wy, wz = _warper(g).gradient()
    assert np.array_equal(wx, g["gx"]) and np.array_equal(wy, g["gy"])


def test_hessian(golden):
    _, g = golden
    H = _warper(g).hessian()
    assert np.array_equal(H, g["H"])
    assert np.array_equal(H, H.T)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_error_jacobian_and_warps(golden, tag):
    _, g = golden
    w = _warper(g)
    D = g[f"D_{tag}"]
    f, err = w.get_error(g["frame"], D, want_image=True)
    assert f == g[f"f_{tag}"]
    assert np.array_equal(w.get_jacobian_from_error(err), g[f"jac_{tag}"])
    assert np.array_equal(w.warp_interpolated(g["frame"], D, 0), g[f"warp0_{tag}"])
    assert np.array_equal(w.warp_interpolated(g["frame"], D, -1), g[f"warpm1_{tag}"])
    wimg, cov = w.warp_image(g["frame"], D)
    assert np.array_equal(wimg, g[f"splat_{tag}"]) and np.array_equal(cov, g[f"coverage_{tag}"])


def test_warp_point(golden):
    _, g = golden
    w = _warper(g)
    for p, want in zip(g["warp_point_xyz"], g["warp_point"]):
        assert np.array_equal(w.warp_point(g["D_b"], *[int(v) for v in p]), want)


def test_phase_shift(golden):
    _, g = golden
    assert np.array_equal(O.phase_shift(g["raw_reference"], g["raw_frame"]), g["phase_shift"])


def test_phase_shift_known_cases():
    d = load_golden("phase_shifts")
    keys = [k[len("shift_"):] for k in d if k.startswith("shift_")]
    assert len(keys) >= 12
    for k in keys:
        assert np.array_equal(O.phase_shift(d[f"ref_{k}"], d[f"vol_{k}"]), d[f"shift_{k}"]), k


def test_full_solve(golden):
    _, g = golden
    D, st = _warper(g).align_frame(g["frame"], g["phase_shift"], max_iter=100)
    assert np.array_equal(D, g["D_solve"])
    assert st.iterations == int(g["solve_iterations"])


def test_scan_init_matches_reference_constructor():
    s = O.scan_init(100.0, 50.0, 102.0, 0, 7, 3)  # interline < line -> 1.01 * line; n_x clamped to 1
    assert s.interline_duration == 1.01 * 100.0
    assert s.n_x == 1 and s.pixel_duration == 100.0
    assert s.frame_duration == 7 * 101.0
    assert s.stack_duration == 2 * 102.0 + 7 * 101.0


def test_last_interval_check_throws():
    # More control intervals than the scan can reach: the last voxel falls short of interval nD-2
    # and the reference throws "Something went wrong" (FrameWarper.cpp:280-281).
    ref = np.ones((3, 8, 8), np.float32)
    sc = O.scan_init(1.0, 1.01, 8 * 1.01, 8, 8, 3)
    with pytest.raises(RuntimeError, match="Something went wrong"):
        O.OracleWarper(ref, 500, sc)


@pytest.mark.skipif(not O.ref_available(), reason="reference build not present")
@pytest.mark.parametrize("seed", [101, 202, 303])
def test_live_against_reference_build(seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    nz = int(rng.integers(1, 4))
    ny, nx = int(rng.integers(10, 40)), int(rng.integers(10, 40))
    nD = int(rng.integers(2, 5)) * nz + 1
    acq = S.make_acquisition((nz, ny, nx), nD, 1, S.BlobSpec(8, (1.5, 4.0), (1.0, 2.0)),
                             S.WalkSpec(0.8, 2.0, 0.2, 0.6), seed=seed)
    line, il, ifr = acq.scan
    ref, fr = acq.reference + 1, acq.frames[0] + 1
    ow = O.OracleWarper(ref, nD, O.scan_init(line, il, ifr, nx, ny, nz))
    rw = O.RefWarper(ref, nD, line, il, ifr)
    rw.set_frame(fr)
    D = acq.D_true[0] + rng.normal(0, 0.5, acq.D_true[0].shape) * (np.array([1, 1, 1 if nz > 1 else 0]))
    assert ow.get_error(fr, D) == rw.get_error(D)
    assert np.array_equal(ow.get_jacobian(fr, D), rw.get_jacobian(D))
    assert np.array_equal(ow.hessian(), rw.hessian())
    assert np.array_equal(ow.warp_interpolated(fr, D, 0), rw.warp_interpolated(D, 0))


def test_warm_start_candidate():
    """The serving loop's fourth starting point: a candidate worse than {0, 0, rigid} is not taken
    (the solve is then bit-identical to the cold one); the frame's own solution as the candidate is
    taken and the solve stays there (within the 1e-8 stop rule's reach)."""
    import fa_synth as S

    acq = S.make_acquisition((1, 96, 96), 8, 1, S.BlobSpec(40, (2.0, 6.0), (1.0, 1.0), mean=20.0),
                             S.WalkSpec(1.0, 3.0), seed=5)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
    frame = acq.frames[0] + 1
    shift = O.phase_shift(acq.reference, acq.frames[0])
    cold, st_cold = ow.align_frame(frame, shift, 100)
    far, _ = ow.align_frame(frame, shift, 100, warm=cold + 40.0)
    assert np.array_equal(far, cold)
    again, st_again = ow.align_frame(frame, shift, 100, warm=cold)
    assert np.sqrt(((again - cold)[:, :2] ** 2).sum(-1).mean()) <= 1e-3
    assert st_again.iterations <= st_cold.iterations


def test_smoothing_statement():
    """smoothStack's kernel size rule cvRound(8 s + 1) | 1, symmetric weights summing to 1, and a
    constant plane staying constant (to float rounding)."""
    for sigma, n in [(0.5, 5), (1.0, 9), (1.5, 13), (2.6, 23), (3.0, 25)]:
        k = O.gaussian_kernel(sigma)
        assert len(k) == n and np.array_equal(k, k[::-1]) and abs(float(k.sum()) - 1) < 1e-6
    c = np.full((2, 17, 23), 7.0, np.float32)
    assert np.allclose(O.smooth_stack(c, 1.7), 7.0, rtol=1e-6, atol=0)


@pytest.mark.parametrize("shape,nD", [((1, 64, 80), 8), ((4, 48, 64), 9)])
def test_fp64_statement_matches_oracle(shape, nD):
    """The FP64 statement of one evaluation (oracle_py.fp64_error_jacobian, the yardstick of the
    mixed-precision reduction-error tests) agrees with the restated warper's float evaluation
    (pinned bit for bit to the reference above) to float rounding: f 1e-6 relative, J^T e 1e-5 of
    max|J^T e|."""
    acq = S.make_acquisition(shape, nD, 1, S.BlobSpec(40, (2.0, 6.0), (1.0, 2.0)), S.WalkSpec(1.0, 3.0, 0.2, 0.8),
                             seed=5)
    nz, ny, nx = shape
    line, il, ifr = acq.scan
    ow = O.OracleWarper(acq.reference + 1, nD, O.scan_init(line, il, ifr, nx, ny, nz))
    fr = (acq.frames[0] + 1).astype(np.float32)
    for D in (np.zeros((nD, 3)), acq.D_true[0].copy()):
        if nz == 1:
            D[:, 2] = 0.0
        f64, g64 = O.fp64_error_jacobian(ow, acq.reference + 1, ow.gradient(), fr, D)
        f, e = ow.get_error(fr, D, want_image=True)
        g = ow.get_jacobian_from_error(e)
        assert abs(f64 - f) <= 1e-6 * f
        assert np.max(np.abs(g64 - g)) <= 1e-5 * np.max(np.abs(g))


def test_round_bf16():
    """round_bf16: round to nearest, ties to even, on the 16 dropped bits."""
    bits = np.array([0x3F800000, 0x3F808000, 0x3F818000, 0x3F807FFF, 0x3F808001, 0xBF80C000], np.uint32)
    want = np.array([0x3F800000, 0x3F800000, 0x3F820000, 0x3F800000, 0x3F810000, 0xBF810000], np.uint32)
    assert np.array_equal(O.round_bf16(bits.view(np.float32)).view(np.uint32), want)

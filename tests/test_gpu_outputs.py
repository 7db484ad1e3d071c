"""Outputs after the solve: the forward splat (AbstractFrameWarper::warpImage) and the per-frame
metrics and images of FrameWarpAligner::addFrame's end (FrameWarpAligner.cpp:221-247, 317-346).

Tolerances (stated per quantity):
  * splat image and coverage: |a - b| <= 1e-5 * max(|b|, 1) per voxel (the same FP64 weights; the
    float sums add the same terms in a different order), and the coverage > 0 masks identical;
  * correlations: |a - b| <= 1e-9 (FP64 sums in a different order) against the oracle's statement;
    coverage fraction exact;
  * uint16 images: equal except where the float value lies within 1e-5 relative of a rounding
    boundary (a value that rounds differently there may differ by 1).
"""
import numpy as np
import pytest

import fa_b200 as fa
import fa_synth as S
import oracle_py as O
from conftest import golden_cases, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    ok, msg = fa.gpu_support()
    assert ok, msg
    return fa.Context()


def _scan(g):
    nz, ny, nx = g["reference"].shape
    line, il, ifr = g["scan"]
    return fa.scan_params(line, il, ifr, nx, ny, nz, bool(g["bidirectional"]))


def _close(a, b, rel=1e-5):
    return np.all(np.abs(a - b) <= rel * np.maximum(np.abs(b), 1.0))


@pytest.mark.parametrize("name", golden_cases())
@pytest.mark.parametrize("tag", ["a", "b"])
def test_splat_matches_reference(ctx, name, tag):
    g = load_golden(name)
    ref = fa.Reference(ctx, g["reference"], int(g["nD"]), _scan(g), fa.PREC_F32)
    wimg, cov = ref.warp_image(g["frame"], g[f"D_{tag}"])
    ref.close()
    assert _close(wimg, g[f"splat_{tag}"]), np.max(np.abs(wimg - g[f"splat_{tag}"]))
    assert _close(cov, g[f"coverage_{tag}"]), np.max(np.abs(cov - g[f"coverage_{tag}"]))
    assert np.array_equal(cov > 0, g[f"coverage_{tag}"] > 0)


def _u16_ok(got, value):
    """got == round-half-even(value) saturated, except next to rounding boundaries."""
    v = np.nan_to_num(value.astype(np.float64), nan=0.0)
    want = np.clip(np.rint(v), 0, 65535)
    near = np.abs(v - np.floor(v) - 0.5) <= 1e-5 * np.maximum(np.abs(v), 1.0)
    bad = (got.astype(np.float64) != want) & ~near
    return not bad.any()


@pytest.mark.parametrize("shape,nD,precision", [((1, 128, 128), 8, fa.PREC_MIXED), ((4, 48, 64), 9, fa.PREC_F32)])
def test_aligner_results_against_oracle(ctx, shape, nD, precision):
    acq = S.make_acquisition(shape, nD, 3, S.BlobSpec(60, (2.0, 6.0), (1.0, 2.0), mean=20.0),
                             S.WalkSpec(1.0, 3.0, 0.2 if shape[0] > 1 else 0.0, 1.0 if shape[0] > 1 else 0.0),
                             seed=91)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    raw = np.ascontiguousarray(acq.frames.astype(np.uint16))
    al = fa.Aligner(ctx, nD=nD, precision=precision)
    al.set_reference(acq.reference, fa.scan_params(line, il, ifr, nx, ny, nz))
    D, _ = al.add_frames([raw[k] for k in range(3)])
    res, imgs = al.results([raw[k] for k in range(3)], D, images=True)
    res2 = al.results([raw[k] for k in range(3)], D)
    al.close()
    assert res == res2  # deterministic, and the same with or without the images
    ow = O.OracleWarper(acq.reference + 1, nD, O.scan_init(line, il, ifr, nx, ny, nz))
    refp1 = (acq.reference + 1).astype(np.float32)
    for k in range(3):
        frame = raw[k].astype(np.float32)
        wimg, cov = ow.warp_image(frame, D[k])
        assert np.array_equal(imgs["mask"][k] > 0, cov > 0)
        assert _close(imgs["mask"][k], cov)
        m = (cov > 0).astype(np.uint8).ravel()
        warped = ow.warp_interpolated(frame + 1, D[k], 0.0)
        corr = O.correlation(warped.ravel(), refp1.ravel(), m)
        unal = O.correlation((frame + 1).ravel(), refp1.ravel(), m)
        # the warped image itself is the FP32 fused warp (within 1e-5 of the reference's), so the
        # correlation carries that difference: 1e-6 absolute
        assert abs(res[k]["correlation"] - corr) <= 1e-6, (res[k]["correlation"], corr)
        assert abs(res[k]["unaligned_correlation"] - unal) <= 1e-9
        assert res[k]["coverage"] == float(np.count_nonzero(cov)) / cov.size
        assert res[k]["use_frame"] == 1  # thresholds 0
        with np.errstate(invalid="ignore", divide="ignore"):
            assert _u16_ok(imgs["realigned_preserving"][k], wimg / cov)
        assert _u16_ok(imgs["realigned"][k], ow.warp_interpolated(frame, D[k], 0.0))


@pytest.mark.parametrize("name", golden_cases())
def test_shift_pixels_against_oracle(ctx, name):
    """FrameWarpAligner::shiftPixel: coordinates truncated to int for warpPoint, points outside the
    volume unchanged; displacements from the oracle's warpPoint (pinned to the reference build)."""
    g = load_golden(name)
    nz, ny, nx = g["reference"].shape
    line, il, ifr = g["scan"]
    ref = fa.Reference(ctx, g["reference"], int(g["nD"]), _scan(g), fa.PREC_F32)
    ow = O.OracleWarper(g["reference"], int(g["nD"]), O.scan_init(line, il, ifr, nx, ny, nz, bool(g["bidirectional"])))
    rng = np.random.default_rng(5)
    n = 500
    x = rng.uniform(-1.5, nx + 0.5, n)
    y = rng.uniform(-1.5, ny + 0.5, n)
    z = rng.uniform(-0.9, nz + 0.5, n) if nz > 1 else np.zeros(n)
    D = g["D_a"]
    sx, sy, sz = ref.shift_pixels(D, x, y, z)
    ref.close()
    for k in range(n):
        xi, yi, zi = int(x[k]), int(y[k]), int(z[k])  # C++ double -> int truncation
        if 0 <= xi < nx and 0 <= yi < ny and 0 <= zi < nz:
            d = ow.warp_point(D, xi, yi, zi)
            want = (x[k] - d[0], y[k] - d[1], z[k] - d[2] if nz > 1 else z[k])
        else:
            want = (x[k], y[k], z[k])
        assert (sx[k], sy[k], sz[k]) == want, (k, (sx[k], sy[k], sz[k]), want)

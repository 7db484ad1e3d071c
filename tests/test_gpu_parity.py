"""GPU parity: the CUDA library through its C ABI against the oracle and the reference's golden
outputs (tests/golden, produced by the reference's own FrameWarper/Sobel3d/VolumePhaseCorrelator
sources).

Tolerances (stated per quantity):
  * interval tables (D_range), Sobel gradients, phase-correlation peaks: bit-exact;
  * Hessian H = J^T J: |dH| <= 1e-12 * max|H| (FP64 sums in a different order);
  * warped images: |a - b| <= 1e-5 * max(|b|, 1) per voxel (1e-5 relative; values carry the +1
    offset so valid voxels are >= 1 away from partial-coverage edges);
  * error sum f: relative 2e-6; J^T e: |dg| <= 2e-5 * max|g| (FP32 trilinear and FP32 partial sums
    vs the reference's double weights and sequential double sums);
  * recovered displacements: RMS over control points <= 0.01 px against the CPU solve.
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


def _rms(a, b, n_dim):
    d = (np.asarray(a) - np.asarray(b))[..., :n_dim]
    return float(np.sqrt((d ** 2).sum(-1).mean()))


def _warp_ok(a, b):
    return np.all(np.abs(a - b) <= 1e-5 * np.maximum(np.abs(b), 1.0))


@pytest.mark.parametrize("name", golden_cases())
def test_reference_setup(ctx, name):
    g = load_golden(name)
    ref = fa.Reference(ctx, g["reference"], int(g["nD"]), _scan(g))
    assert np.array_equal(ref.ranges(), g["ranges"])
    gx, gy, gz = ref.gradient()
    assert np.array_equal(gx, g["gx"]) and np.array_equal(gy, g["gy"]) and np.array_equal(gz, g["gz"])
    H = ref.hessian()
    assert np.max(np.abs(H - g["H"])) <= 1e-12 * np.max(np.abs(g["H"]))
    assert np.array_equal(H, H.T)


@pytest.mark.parametrize("name", golden_cases())
@pytest.mark.parametrize("tag", ["a", "b"])
def test_error_jacobian_warp(ctx, name, tag):
    g = load_golden(name)
    ref = fa.Reference(ctx, g["reference"], int(g["nD"]), _scan(g))
    fr = fa.Frame(ref, g["frame"])
    D = g[f"D_{tag}"]
    f = fr.get_error(D)
    assert abs(f - g[f"f_{tag}"]) <= 2e-6 * abs(g[f"f_{tag}"])
    jac = fr.get_jacobian(D)
    want = g[f"jac_{tag}"]
    assert np.max(np.abs(jac - want)) <= 2e-5 * np.max(np.abs(want))
    assert _warp_ok(fr.warp(D, 0.0), g[f"warp0_{tag}"])
    assert _warp_ok(fr.warp(D, -1.0), g[f"warpm1_{tag}"])


@pytest.mark.parametrize("name", golden_cases())
def test_phase_shift(ctx, name):
    g = load_golden(name)
    c = fa.Correlator(ctx, g["raw_reference"])
    assert np.array_equal(c.compute_shift(g["raw_frame"]), g["phase_shift"])


def test_phase_shift_known_cases(ctx):
    d = load_golden("phase_shifts")
    for k in [k[len("shift_"):] for k in d if k.startswith("shift_")]:
        c = fa.Correlator(ctx, d[f"ref_{k}"])
        assert np.array_equal(c.compute_shift(d[f"vol_{k}"]), d[f"shift_{k}"]), k


@pytest.mark.parametrize("name", golden_cases())
def test_full_solve(ctx, name):
    g = load_golden(name)
    ref = fa.Reference(ctx, g["reference"], int(g["nD"]), _scan(g))
    fr = fa.Frame(ref, g["frame"])
    D, st = fr.align(g["phase_shift"], 100)
    assert _rms(D, g["D_solve"], ref.n_dim) <= 0.01
    assert st["iterations"] >= 1


def test_subproblem_matches_oracle_bitwise(ctx):
    rng = np.random.Generator(np.random.PCG64(5))
    for n_dim, nD in [(2, 10), (3, 32), (3, 7)]:
        P = n_dim * nD
        J = np.zeros((4 * P, P))
        for i in range(nD):
            rows = slice(4 * i * n_dim, 4 * (i + 1) * n_dim)
            J[rows, i * n_dim:(i + 1) * n_dim] = rng.normal(size=(4 * n_dim, n_dim))
            if i + 1 < nD:
                J[rows, (i + 1) * n_dim:(i + 2) * n_dim] = rng.normal(size=(4 * n_dim, n_dim))
        H = J.T @ J
        # keep the block-tridiagonal pattern exactly
        for i in range(P):
            for j in range(P):
                if abs(i // n_dim - j // n_dim) > 1:
                    H[i, j] = 0.0
        g = rng.normal(size=P) * 10
        for radius in [1e-3, 0.5, 5.0, 40.0, 1e4]:
            p_dev, b_dev = fa.test_tr_subproblem(ctx, nD, n_dim, H, g, radius)
            p_cpu, b_cpu = O.tr_subproblem(H, g, radius)
            assert b_dev == b_cpu
            assert np.array_equal(p_dev, p_cpu), (n_dim, nD, radius, np.max(np.abs(p_dev - p_cpu)))


def test_batch_equals_single(ctx):
    names = [n for n in golden_cases() if load_golden(n)["reference"].shape[0] == 1]
    refs, frames, rigid, single = [], [], [], []
    for n in names:
        g = load_golden(n)
        ref = fa.Reference(ctx, g["reference"], int(g["nD"]), _scan(g))
        fr = fa.Frame(ref, g["frame"])
        refs.append(ref)
        frames.append(fr)
        rigid.append(g["phase_shift"])
        single.append(fr.align(g["phase_shift"], 100)[0])
    # mixed batch of frames of different sizes and references, in one launch per iteration
    nDs = {r.nD for r in refs}
    for nD in nDs:
        idx = [i for i, r in enumerate(refs) if r.nD == nD]
        D, stats = fa.align_batch([frames[i] for i in idx], np.array([rigid[i] for i in idx]), 100)
        for k, i in enumerate(idx):
            assert np.array_equal(D[k], single[i])


def _acq(shape, nD, n_frames, seed):
    return S.make_acquisition(shape, nD, n_frames, S.BlobSpec(int(200 * np.prod(shape[1:]) / 65536) + 10,
                                                              (2.0, 8.0), (1.0, 2.0)),
                              S.WalkSpec(1.5, 6.0, 0.3, 1.5), seed=seed)


@pytest.mark.parametrize("precision", [fa.PREC_F32, fa.PREC_MIXED])
def test_plane_256_against_oracle(ctx, precision):
    acq = S.make_config(S.CONFIG0, n_frames=3)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
    ref = fa.Reference(ctx, acq.reference + 1, acq.nD, fa.scan_params(line, il, ifr, nx, ny, nz), precision)
    corr = fa.Correlator(ctx, acq.reference)
    frames = [fa.Frame(ref, acq.frames[k] + 1) for k in range(3)]
    shifts = np.array([corr.compute_shift(acq.frames[k]) for k in range(3)])
    D_b, _ = fa.align_batch(frames, shifts, 100)
    for k in range(3):
        assert np.array_equal(shifts[k], O.phase_shift(acq.reference, acq.frames[k]))
        D_cpu, _ = ow.align_frame(acq.frames[k] + 1, shifts[k], 100)
        D_gpu, _ = frames[k].align(shifts[k], 100)
        assert _rms(D_gpu, D_cpu, 2) <= 0.01, (k, _rms(D_gpu, D_cpu, 2))
        assert np.array_equal(D_b[k], D_gpu)


def test_stack_512x512x16_against_oracle(ctx):
    """The 512x512x16, nD = 32 workload at full size: one frame, CPU solve vs plain GPU solve."""
    acq = S.make_config(S.CONFIG1, n_frames=1)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
    ref = fa.Reference(ctx, acq.reference + 1, acq.nD, fa.scan_params(line, il, ifr, nx, ny, nz))
    H = ref.hessian()
    Hc = ow.hessian()
    assert np.max(np.abs(H - Hc)) <= 1e-10 * np.max(np.abs(Hc))
    fr = fa.Frame(ref, acq.frames[0] + 1)
    D = acq.D_true[0]
    f_cpu, err = ow.get_error(acq.frames[0] + 1, D, want_image=True)
    assert abs(fr.get_error(D) - f_cpu) <= 2e-6 * f_cpu
    j_cpu = ow.get_jacobian_from_error(err)
    assert np.max(np.abs(fr.get_jacobian(D) - j_cpu)) <= 2e-5 * np.max(np.abs(j_cpu))
    shift = fa.Correlator(ctx, acq.reference).compute_shift(acq.frames[0])
    D_cpu, _ = ow.align_frame(acq.frames[0] + 1, shift, 100)
    D_gpu, _ = fr.align(shift, 100)
    assert _rms(D_gpu, D_cpu, 3) <= 0.01


def test_errors_are_reported(ctx):
    scan = fa.scan_params(1.0, 1.01, 8 * 1.01, 8, 8, 3)
    with pytest.raises(fa.FaError, match="Something went wrong"):
        fa.Reference(ctx, np.ones((3, 8, 8), np.float32), 500, scan)
    with pytest.raises(fa.FaError) as e:
        fa.Reference(ctx, np.ones((1, 8, 1), np.float32), 3, fa.scan_params(1.0, 1.01, 8.08, 1, 8, 1))
    assert e.value.status == 1
    acq = _acq((1, 32, 32), 4, 1, 9)
    line, il, ifr = acq.scan
    ref = fa.Reference(ctx, acq.reference + 1, 4, fa.scan_params(line, il, ifr, 32, 32, 1))
    fr = fa.Frame(ref, acq.frames[0] + 1)
    D = np.zeros((4, 3))
    D[1, 0] = np.nan
    with pytest.raises(fa.FaError) as e:
        fr.get_error(D)
    assert e.value.status == 1


@pytest.mark.parametrize("precision", [fa.PREC_F32, fa.PREC_MIXED])
def test_aligner_raw_frames_against_oracle(ctx, precision):
    """fa_aligner_*: raw uint16 frames in (host and device), +1 offset, phase-correlation start and
    the batched solve on the device; D within 0.01 px RMS of the CPU solve of the same frames."""
    import torch

    acq = S.make_config(S.CONFIG0, n_frames=5)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
    al = fa.Aligner(ctx, nD=acq.nD, precision=precision)
    al.set_reference(acq.reference, fa.scan_params(line, il, ifr, nx, ny, nz))
    raw = np.ascontiguousarray(acq.frames.astype(np.uint16))
    D_host, st = al.add_frames([raw[k] for k in range(5)])
    dev = torch.from_numpy(raw.view(np.int16)).to("cuda:0")
    torch.cuda.synchronize()
    D_dev, _ = al.add_frames_device([dev[k].data_ptr() for k in range(5)], fa.U16, 5)
    assert np.array_equal(D_host, D_dev)
    for k in range(5):
        shift = O.phase_shift(acq.reference, acq.frames[k])
        D_cpu, _ = ow.align_frame(acq.frames[k] + 1, shift, 100)
        assert _rms(D_host[k], D_cpu, 2) <= 0.01, (k, _rms(D_host[k], D_cpu, 2))


def test_tile_shapes_agree(ctx):
    """Every tile shape the autotuner may pick gives the same f and J^T e (the partial sums only
    change grouping): relative 1e-6 for f, 1e-5 of max|J^T e|."""
    acq = _acq((4, 64, 128), 13, 1, 17)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    D = acq.D_true[0]
    results = []
    for tile, mb in [(512, 2), (2048, 3), (8192, 4), (32768, 2)]:
        ref = fa.Reference(ctx, acq.reference + 1, 13, fa.scan_params(line, il, ifr, nx, ny, nz), fa.PREC_MIXED)
        ref.retune(tile, mb)
        fr = fa.Frame(ref, acq.frames[0] + 1)
        results.append((fr.get_error(D), fr.get_jacobian(D), fr.align(None, 100)[0]))
        fr.close()
    f0, j0, d0 = results[0]
    for f, j, d in results[1:]:
        assert abs(f - f0) <= 1e-6 * f0
        assert np.max(np.abs(j - j0)) <= 1e-5 * np.max(np.abs(j0))
        assert _rms(d, d0, 3) <= 0.01


def test_autotuned_context(ctx):
    tuned = fa.Context(autotune=True)
    acq = _acq((2, 64, 128), 9, 1, 18)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    ref = fa.Reference(tuned, acq.reference + 1, 9, fa.scan_params(line, il, ifr, nx, ny, nz), fa.PREC_MIXED)
    tile, mb = ref.tuning()
    assert tile % nx == 0 and 2 <= mb <= 4
    fr = fa.Frame(ref, acq.frames[0] + 1)
    ref_plain = fa.Reference(ctx, acq.reference + 1, 9, fa.scan_params(line, il, ifr, nx, ny, nz), fa.PREC_MIXED)
    fr_plain = fa.Frame(ref_plain, acq.frames[0] + 1)
    f1, f2 = fr.get_error(acq.D_true[0]), fr_plain.get_error(acq.D_true[0])
    assert abs(f1 - f2) <= 1e-6 * f2

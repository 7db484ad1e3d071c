"""The drop-in boundary, compiled and run: B200FrameWarper (frame-aligner_b200/adaptor/
B200FrameWarper.h) built against the reference's own FrameWarper.h and driven by the reference's
AbstractFrameWarper::setReference (FrameWarper.cpp:186-205) and OptimisationModel
(OptimisationModel.cpp:45-62), against the reference's CpuFrameWarper on the golden cases.

Tolerances: f 2e-6 relative; J^T e 2e-5 of max|J^T e|; the Hessian the model reads 1e-12 of
max|H|; warped images 1e-5 x max(|value|, 1); the solve the model drives (the project's trust
region, dlib being absent from the reference tree) 0.01 px RMS from the CPU warper's solve."""
import numpy as np
import pytest

import oracle_py as O
from conftest import golden_cases, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_adaptor():
    if not O.adaptor_available():
        pytest.fail("oracle/_ref/libfa_adaptor.so missing: build with make -C oracle (needs the reference tree)")
    msg = __import__("ctypes").create_string_buffer(256)
    assert O.adaptorlib().fa_adaptor_gpu_support(msg, 256) == 1, msg.value


@pytest.mark.parametrize("name", golden_cases())
def test_adaptor_matches_cpu_warper(name):
    g = load_golden(name)
    line, il, ifr = g["scan"]
    bidir = bool(g["bidirectional"])
    nD = int(g["nD"])
    aw = O.AdaptorWarper(g["reference"], nD, line, il, ifr, bidir)
    aw.set_frame(g["frame"])
    nd = aw.n_dim
    for tag in ("a", "b"):
        D = g[f"D_{tag}"]
        f, der, hess = aw.model(D)
        assert abs(f - g[f"f_{tag}"]) <= 2e-6 * abs(g[f"f_{tag}"])
        want = g[f"jac_{tag}"]
        assert np.max(np.abs(der - want)) <= 2e-5 * np.max(np.abs(want))
        assert np.max(np.abs(hess - g["H"])) <= 1e-12 * np.max(np.abs(g["H"]))
        for inv in (0, -1):
            w = aw.warp_interpolated(D, inv)
            ref_w = g[f"warp0_{tag}"] if inv == 0 else g[f"warpm1_{tag}"]
            assert np.all(np.abs(w - ref_w) <= 1e-5 * np.maximum(np.abs(ref_w), 1.0))
    D, iters = aw.align(g["phase_shift"], 100)
    rms = float(np.sqrt(((D - g["D_solve"])[:, :nd] ** 2).sum(-1).mean()))
    assert rms <= 0.01 and iters >= 1, (rms, iters)


def test_adaptor_reports_errors_as_exceptions():
    # the reference's own set-up throws first: the scan never reaches interval nD - 2
    # (FrameWarper.cpp:280-281)
    with pytest.raises(RuntimeError, match="Something went wrong"):
        O.AdaptorWarper(np.ones((3, 8, 8), np.float32), 500, 1.0, 1.01, 8 * 1.01)
    # the reference accepts it, the library does not (control intervals shorter than one image row):
    # the library's error reaches the caller as the same exception type
    g = load_golden(golden_cases()[0])
    line, il, ifr = g["scan"]
    with pytest.raises(RuntimeError, match="shorter than one image row"):
        O.AdaptorWarper(g["reference"], 500, line, il, ifr)

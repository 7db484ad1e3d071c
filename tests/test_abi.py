"""The C ABI library loads on a CPU-only host and exports every entry point that
include/fa_b200.h declares (no compute calls: those need the GPU and live in the -m gpu tests)."""
import os
import re

import numpy as np
import pytest

import fa_b200 as fa
import oracle_py as O

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_entry_points():
    text = open(os.path.join(ROOT, "include", "fa_b200.h")).read()
    return sorted(set(re.findall(r"^(?:fa_status|const char\*)\s+(fa_\w+)\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_entry_points()
    assert "fa_get_error" in names and "fa_get_jacobian" in names and "fa_align_batch" in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol():
    lib = fa.lib()
    missing = [n for n in declared_entry_points() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert set(declared_entry_points()) <= set(fa.SIGNATURES)


@pytest.mark.parametrize("args", [(1.0, 1.01, 512 * 1.01, 512, 512, 16, 0), (100.0, 50.0, 102.0, 0, 7, 3, 1),
                                  (2.0, 3.0, 700.0, 33, 21, 1, 0)])
def test_scan_params_match_reference_constructor(args):
    line, il, ifr, nx, ny, nz, bidir = args
    s = fa.scan_params(line, il, ifr, nx, ny, nz, bidir)
    o = O.scan_init(line, il, ifr, nx, ny, nz, bidir)
    for k in ("line_duration", "interline_duration", "pixel_duration", "frame_duration", "interframe_duration",
              "stack_duration", "n_x", "n_y", "n_z", "bidirectional"):
        assert getattr(s, k) == getattr(o, k), k


def test_status_strings():
    lib = fa.lib()
    assert lib.fa_status_string(0) == b"ok"
    assert lib.fa_status_string(2) == b"out of memory"


def test_gpu_support_reports_without_a_device():
    ok, msg = fa.gpu_support()
    if not ok:
        assert msg  # "No compatible GPU" / "Insufficient Driver" (GpuFrameWarper.cpp:16-44)


def test_realignment_info_csv(tmp_path):
    """fa_write_realignment_info writes FrameWarpAligner::writeRealignmentInfo's format
    (FrameWarpAligner.cpp:288-314; C++ default stream formatting = printf %g)."""
    import fa_b200 as fa

    scan = fa.ScanParams()
    fa.check(fa.lib().fa_scan_params_init(1.0, 1.01, 51.7, 32, 48, 3, 0, scan))
    rng = np.random.default_rng(3)
    D = rng.normal(0, 2, (2, 4, 3))
    res = [{"correlation": 0.91234567, "unaligned_correlation": 0.5, "coverage": 1.0},
           {"correlation": 1e-7, "unaligned_correlation": -0.25, "coverage": 0.875}]
    f = tmp_path / "info.csv"
    fa.write_realignment_info(str(f), scan, D, res)
    g = lambda v: "%g" % v  # noqa: E731
    want = ["Realignment Information Version, 2", "Line Duration," + g(scan.line_duration),
            "Interline Duration," + g(scan.interline_duration), "Frame Duration," + g(scan.frame_duration),
            "Interframe Duration," + g(scan.interframe_duration), "Lines,48", "Frames Per Stack,3",
            "Frame, UnalignedCorrelation, Correlation, Coverage" + "".join(
                ", dx_%d, dy_%d, dz_%d" % (j, j, j) for j in range(4))]
    for i, r in enumerate(res):
        want.append("%d,%s,%s, %s" % (i, g(r["unaligned_correlation"]), g(r["correlation"]), g(r["coverage"])) +
                    "".join(", %s, %s, %s" % tuple(g(v) for v in D[i, j]) for j in range(4)))
    assert f.read_text() == "\n".join(want) + "\n"

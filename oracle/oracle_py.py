"""ctypes bindings for the oracle (TEST INFRASTRUCTURE ONLY).

Loads ``liboracle.so`` (the C restatement of frame-aligner's warper path, fa_oracle.c) and, when
present, ``_ref/libfa_ref.so`` (the reference's own FrameWarper.cpp, Sobel3d.cpp,
VolumePhaseCorrelator.cpp and OptimisationModel.cpp compiled unchanged against container
stand-ins). Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may import
this module; it is the checker, never the product path.

Phase correlation (FrameAligner/VolumePhaseCorrelator.cpp:57-166) is restated here with numpy's
FP64 FFT (pocketfft); window, normalisation, first-maximum argmax and wrap follow the reference
lines cited in ``phase_shift``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


class OrScan(C.Structure):
    _fields_ = [
        ("line_duration", C.c_double),
        ("interline_duration", C.c_double),
        ("pixel_duration", C.c_double),
        ("frame_duration", C.c_double),
        ("interframe_duration", C.c_double),
        ("stack_duration", C.c_double),
        ("n_x", C.c_int),
        ("n_y", C.c_int),
        ("n_z", C.c_int),
        ("bidirectional", C.c_int),
    ]


class OrStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("evaluations", C.c_int),
        ("accepted", C.c_int),
        ("f_final", C.c_double),
        ("radius_final", C.c_double),
    ]


_lib = None
_ref = {}


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} (run make -C oracle)")
        L = C.CDLL(path)
        L.or_scan_init.argtypes = [C.POINTER(OrScan), C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                   C.c_int, C.c_int]
        L.or_process_scan.argtypes = [C.POINTER(OrScan), C.c_int, C.c_int, C.POINTER(OrScan)]
        L.or_warper_create.restype = C.c_void_p
        L.or_warper_create.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(OrScan), C.c_char_p]
        L.or_warper_destroy.argtypes = [C.c_void_p]
        L.or_warper_n_dim.argtypes = [C.c_void_p]
        L.or_warper_precomp.argtypes = [C.c_void_p, _u16p, _f32p, _i32p]
        L.or_warper_hessian.argtypes = [C.c_void_p, _f64p]
        L.or_warper_gradient.argtypes = [C.c_void_p, _f32p, _f32p, _f32p]
        L.or_warp_interpolated.argtypes = [C.c_void_p, _f32p, _f64p, C.c_float, _f32p]
        L.or_get_error.restype = C.c_double
        L.or_get_error.argtypes = [C.c_void_p, _f32p, _f64p, _f32p]
        L.or_get_jacobian.argtypes = [C.c_void_p, _f32p, _f64p]
        L.or_warp_image.argtypes = [C.c_void_p, _f32p, _f64p, _f32p, _f32p]
        L.or_warp_point.argtypes = [C.c_void_p, _f64p, C.c_int, C.c_int, C.c_int, C.c_int, _f64p]
        L.or_sobel3d.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f32p, _f32p, _f32p]
        L.or_downsample.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p]
        L.or_smooth_stack.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_double, _f32p]
        L.or_gaussian_kernel.argtypes = [C.c_double, _f32p, C.c_int]
        L.or_correlation.restype = C.c_double
        L.or_correlation.argtypes = [_f32p, _f32p, _u8p, C.c_long]
        L.or_tr_subproblem.argtypes = [C.c_int, _f64p, _f64p, C.c_double, C.c_double, C.c_int, _f64p]
        L.or_align_frame.argtypes = [C.c_void_p, _f32p, _f64p, C.c_int, _f64p, C.POINTER(OrStats)]
        L.or_align_frame_warm.argtypes = [C.c_void_p, _f32p, _f64p, C.c_void_p, C.c_int, _f64p, C.POINTER(OrStats)]
        L.or_align_frames_mt.argtypes = [C.c_void_p, _f32p, C.c_int, _f64p, C.c_int, C.c_int, _f64p, _i32p]
        _lib = L
    return _lib


def _ref_path(fast=False):
    return os.path.join(HERE, "_ref", "libfa_ref_fast.so" if fast else "libfa_ref.so")


def ref_available(fast=False) -> bool:
    """The reference build is present: the parity build (-O2, no fused multiply-add) or, with
    fast=True, the timing build with the reference's release flags."""
    return os.path.exists(_ref_path(fast))


def reflib(fast=False):
    if fast not in _ref:
        path = _ref_path(fast)
        if not os.path.exists(path):
            raise RuntimeError(f"reference build missing: {path}")
        R = C.CDLL(path)
        R.fr_warper_create.restype = C.c_void_p
        R.fr_warper_create.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                       C.c_double, C.c_int, C.c_char_p]
        R.fr_warper_destroy.argtypes = [C.c_void_p]
        R.fr_n_dim.argtypes = [C.c_void_p]
        R.fr_set_frame.argtypes = [C.c_void_p, _f32p]
        R.fr_get_error.restype = C.c_double
        R.fr_get_error.argtypes = [C.c_void_p, _f64p]
        R.fr_get_jacobian.argtypes = [C.c_void_p, _f64p, _f64p]
        R.fr_hessian.argtypes = [C.c_void_p, _f64p]
        R.fr_model_f.restype = C.c_double
        R.fr_model_f.argtypes = [C.c_void_p, _f64p]
        R.fr_precomp.argtypes = [C.c_void_p, _u16p, _f32p, _i32p]
        R.fr_warp_interpolated.argtypes = [C.c_void_p, _f64p, C.c_int, _f32p]
        R.fr_warp_image.argtypes = [C.c_void_p, _f64p, _f32p, _f32p]
        R.fr_warp_point.argtypes = [C.c_void_p, _f64p, C.c_int, C.c_int, C.c_int, C.c_int, _f64p]
        R.fr_sobel3d.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f32p, _f32p, _f32p]
        R.fr_phase_shift.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, _f64p]
        R.fr_align_frame.argtypes = [C.c_void_p, _f32p, _f64p, C.c_int, _f64p, _i32p]
        R.fr_mt_create.restype = C.c_void_p
        R.fr_mt_create.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                   C.c_int, C.c_int, C.c_char_p]
        R.fr_mt_destroy.argtypes = [C.c_void_p]
        R.fr_mt_align.argtypes = [C.c_void_p, _f32p, C.c_int, _f64p, C.c_int, _f64p, _i32p]
        _ref[fast] = R
    return _ref[fast]


def scan_init(line, interline, interframe, nx, ny, nz, bidirectional=False) -> OrScan:
    s = OrScan()
    lib().or_scan_init(C.byref(s), line, interline, interframe, nx, ny, nz, int(bidirectional))
    return s


def _c32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class OracleWarper:
    """The restated AbstractFrameWarper/CpuFrameWarper (FrameAligner/FrameWarper.h:95-160)."""

    def __init__(self, reference, nD, scan: OrScan):
        ref = _c32(reference)
        assert ref.ndim == 3
        self.dims = ref.shape
        self.nD = int(nD)
        err = C.create_string_buffer(256)
        self._h = lib().or_warper_create(ref, ref.shape[0], ref.shape[1], ref.shape[2], self.nD, C.byref(scan), err)
        if not self._h:
            raise RuntimeError(err.value.decode())
        self.n_dim = lib().or_warper_n_dim(self._h)
        self.N = int(np.prod(self.dims))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_warper_destroy(self._h)
            self._h = None

    @property
    def P(self):
        return self.nD * self.n_dim

    def precomp(self):
        Di = np.empty(self.N, np.uint16)
        Df = np.empty(self.N, np.float32)
        r = np.empty(2 * self.nD, np.int32)
        lib().or_warper_precomp(self._h, Di, Df, r)
        return Di.reshape(self.dims), Df.reshape(self.dims), r.reshape(self.nD, 2)

    def hessian(self):
        H = np.empty((self.P, self.P), np.float64)
        lib().or_warper_hessian(self._h, H)
        return H

    def gradient(self):
        g = [np.empty(self.N, np.float32) for _ in range(3)]
        lib().or_warper_gradient(self._h, *g)
        return [x.reshape(self.dims) for x in g]

    def warp_interpolated(self, frame, D, invalid_value=0.0):
        out = np.empty(self.N, np.float32)
        lib().or_warp_interpolated(self._h, _c32(frame).ravel(), _c64(D).ravel(), float(invalid_value), out)
        return out.reshape(self.dims)

    def get_error(self, frame, D, want_image=False):
        err = np.empty(self.N, np.float32)
        f = lib().or_get_error(self._h, _c32(frame).ravel(), _c64(D).ravel(), err)
        return (f, err.reshape(self.dims)) if want_image else f

    def get_jacobian_from_error(self, err):
        jac = np.empty(self.P, np.float64)
        lib().or_get_jacobian(self._h, _c32(err).ravel(), jac)
        return jac

    def get_jacobian(self, frame, D):
        _, e = self.get_error(frame, D, want_image=True)
        return self.get_jacobian_from_error(e)

    def warp_image(self, frame, D):
        w = np.empty(self.N, np.float32)
        c = np.empty(self.N, np.float32)
        lib().or_warp_image(self._h, _c32(frame).ravel(), _c64(D).ravel(), w, c)
        return w.reshape(self.dims), c.reshape(self.dims)

    def warp_point(self, D, x, y, z, spatial_binning=1):
        out = np.empty(3, np.float64)
        lib().or_warp_point(self._h, _c64(D).ravel(), x, y, z, spatial_binning, out)
        return out

    def align_frame(self, frame, rigid_shift=(0.0, 0.0, 0.0), max_iter=100, warm=None):
        """or_align_frame; warm (nD x 3) adds the previous frame's solution as a fourth start."""
        D = np.empty((self.nD, 3), np.float64)
        st = OrStats()
        if warm is None:
            lib().or_align_frame(self._h, _c32(frame).ravel(), _c64(rigid_shift), max_iter, D, C.byref(st))
        else:
            w = _c64(warm).ravel()
            lib().or_align_frame_warm(self._h, _c32(frame).ravel(), _c64(rigid_shift), w.ctypes.data, max_iter, D,
                                      C.byref(st))
        return D, st

    def align_frames_mt(self, frames, rigid_shifts, n_threads, max_iter=100):
        frames = _c32(frames)
        n = frames.shape[0]
        D = np.empty((n, self.nD, 3), np.float64)
        iters = np.empty(n, np.int32)
        lib().or_align_frames_mt(self._h, frames.ravel(), n, _c64(rigid_shifts).ravel(), max_iter, n_threads, D,
                                 iters)
        return D, iters


class RefWarper:
    """The reference's own CpuFrameWarper, built from its sources (oracle/_ref/libfa_ref.so)."""

    def __init__(self, reference, nD, line, interline, interframe, bidirectional=False):
        ref = _c32(reference)
        self.dims = ref.shape
        self.nD = int(nD)
        err = C.create_string_buffer(256)
        R = reflib()
        self._h = R.fr_warper_create(ref, ref.shape[0], ref.shape[1], ref.shape[2], self.nD, line, interline,
                                     interframe, int(bidirectional), err)
        if not self._h:
            raise RuntimeError(err.value.decode())
        self.n_dim = R.fr_n_dim(self._h)
        self.N = int(np.prod(self.dims))

    def __del__(self):
        if getattr(self, "_h", None):
            reflib().fr_warper_destroy(self._h)
            self._h = None

    @property
    def P(self):
        return self.nD * self.n_dim

    def set_frame(self, frame):
        reflib().fr_set_frame(self._h, _c32(frame).ravel())

    def get_error(self, D):
        return reflib().fr_get_error(self._h, _c64(D).ravel())

    def get_jacobian(self, D):
        j = np.empty(self.P, np.float64)
        reflib().fr_get_jacobian(self._h, _c64(D).ravel(), j)
        return j

    def hessian(self):
        H = np.empty((self.P, self.P), np.float64)
        reflib().fr_hessian(self._h, H)
        return H

    def precomp(self):
        Di = np.empty(self.N, np.uint16)
        Df = np.empty(self.N, np.float32)
        r = np.empty(2 * self.nD, np.int32)
        reflib().fr_precomp(self._h, Di, Df, r)
        return Di.reshape(self.dims), Df.reshape(self.dims), r.reshape(self.nD, 2)

    def warp_interpolated(self, D, invalid_value=0):
        out = np.empty(self.N, np.float32)
        reflib().fr_warp_interpolated(self._h, _c64(D).ravel(), int(invalid_value), out)
        return out.reshape(self.dims)

    def warp_image(self, D):
        w = np.empty(self.N, np.float32)
        c = np.empty(self.N, np.float32)
        reflib().fr_warp_image(self._h, _c64(D).ravel(), w, c)
        return w.reshape(self.dims), c.reshape(self.dims)

    def warp_point(self, D, x, y, z, spatial_binning=1):
        out = np.empty(3, np.float64)
        reflib().fr_warp_point(self._h, _c64(D).ravel(), x, y, z, spatial_binning, out)
        return out

    def align_frame(self, frame, rigid_shift=(0.0, 0.0, 0.0), max_iter=100):
        D = np.empty((self.nD, 3), np.float64)
        it = np.zeros(1, np.int32)
        reflib().fr_align_frame(self._h, _c32(frame).ravel(), _c64(rigid_shift), max_iter, D, it)
        return D, int(it[0])


_adaptor = None


def adaptor_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libfa_adaptor.so"))


def adaptorlib():
    """_ref/libfa_adaptor.so: the drop-in B200FrameWarper driven by the reference's own
    FrameWarper.cpp / OptimisationModel.cpp (ref_adaptor.cpp)."""
    global _adaptor
    if _adaptor is None:
        path = os.path.join(HERE, "_ref", "libfa_adaptor.so")
        if not os.path.exists(path):
            raise RuntimeError(f"adaptor build missing: {path}")
        A = C.CDLL(path)
        A.fa_adaptor_gpu_support.argtypes = [C.c_char_p, C.c_int]
        A.fa_adaptor_create.restype = C.c_void_p
        A.fa_adaptor_create.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                        C.c_double, C.c_int, C.c_int, C.c_char_p]
        A.fa_adaptor_destroy.argtypes = [C.c_void_p]
        A.fa_adaptor_n_dim.argtypes = [C.c_void_p]
        A.fa_adaptor_set_frame.argtypes = [C.c_void_p, _f32p, C.c_char_p]
        A.fa_adaptor_model.argtypes = [C.c_void_p, _f64p, C.POINTER(C.c_double), _f64p, _f64p, C.c_char_p]
        A.fa_adaptor_warp.argtypes = [C.c_void_p, _f64p, C.c_int, _f32p, C.c_char_p]
        A.fa_adaptor_align.argtypes = [C.c_void_p, _f64p, C.c_int, _f64p, C.POINTER(C.c_int), C.c_char_p]
        _adaptor = A
    return _adaptor


class AdaptorWarper:
    """B200FrameWarper (frame-aligner_b200/adaptor/B200FrameWarper.h) behind the reference's
    AbstractFrameWarper::setReference and OptimisationModel."""

    def __init__(self, reference, nD, line, interline, interframe, bidirectional=False, precision=0):
        ref = _c32(reference)
        self.dims = ref.shape
        self.nD = nD
        err = C.create_string_buffer(256)
        self._h = adaptorlib().fa_adaptor_create(ref, ref.shape[0], ref.shape[1], ref.shape[2], nD, line, interline,
                                                 interframe, int(bidirectional), int(precision), err)
        if not self._h:
            raise RuntimeError(err.value.decode())
        self.n_dim = adaptorlib().fa_adaptor_n_dim(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            adaptorlib().fa_adaptor_destroy(self._h)
            self._h = None

    def _ok(self, rc, err):
        if rc != 0:
            raise RuntimeError(err.value.decode())

    def set_frame(self, frame):
        err = C.create_string_buffer(256)
        self._ok(adaptorlib().fa_adaptor_set_frame(self._h, _c32(frame).ravel(), err), err)

    def model(self, D):
        """(f, der, hess) as OptimisationModel reads them through the adaptor."""
        P = self.nD * self.n_dim
        f = C.c_double()
        der = np.empty(P, np.float64)
        hess = np.empty((P, P), np.float64)
        err = C.create_string_buffer(256)
        self._ok(adaptorlib().fa_adaptor_model(self._h, _c64(D).ravel(), C.byref(f), der, hess, err), err)
        return f.value, der, hess

    def warp_interpolated(self, D, invalid_value=0):
        out = np.empty(int(np.prod(self.dims)), np.float32)
        err = C.create_string_buffer(256)
        self._ok(adaptorlib().fa_adaptor_warp(self._h, _c64(D).ravel(), int(invalid_value), out, err), err)
        return out.reshape(self.dims)

    def align(self, rigid_shift=(0.0, 0.0, 0.0), max_iter=100):
        D = np.zeros((self.nD, 3), np.float64)
        it = C.c_int()
        err = C.create_string_buffer(256)
        self._ok(adaptorlib().fa_adaptor_align(self._h, _c64(rigid_shift), max_iter, D, C.byref(it), err), err)
        return D, it.value


class RefPool:
    """One reference warper per worker thread (fr_mt_create / fr_mt_align); fast=True uses the timing
    build (the reference's release flags)."""

    def __init__(self, reference, nD, line, interline, interframe, n_threads, bidirectional=False, fast=False):
        ref = _c32(reference)
        self.dims = ref.shape
        self.nD = nD
        self.fast = fast
        err = C.create_string_buffer(256)
        self._h = reflib(fast).fr_mt_create(ref, ref.shape[0], ref.shape[1], ref.shape[2], nD, line, interline,
                                            interframe, int(bidirectional), n_threads, err)
        if not self._h:
            raise RuntimeError(err.value.decode())

    def __del__(self):
        if getattr(self, "_h", None):
            reflib(self.fast).fr_mt_destroy(self._h)
            self._h = None

    def align(self, frames, rigid_shifts, max_iter=100):
        frames = _c32(frames)
        n = frames.shape[0]
        D = np.empty((n, self.nD, 3), np.float64)
        iters = np.empty(n, np.int32)
        reflib(self.fast).fr_mt_align(self._h, frames.ravel(), n, _c64(rigid_shifts).ravel(), max_iter, D, iters)
        return D, iters


def ref_sobel3d(m):
    m = _c32(m)
    out = [np.empty(m.size, np.float32) for _ in range(3)]
    reflib().fr_sobel3d(m.ravel(), m.shape[0], m.shape[1], m.shape[2], *out)
    return [o.reshape(m.shape) for o in out]


def ref_phase_shift(ref, vol):
    ref = _c32(ref)
    s = np.empty(3, np.float64)
    reflib().fr_phase_shift(ref.ravel(), _c32(vol).ravel(), ref.shape[0], ref.shape[1], ref.shape[2], s)
    return s


def sobel3d(m):
    m = _c32(m)
    out = [np.empty(m.size, np.float32) for _ in range(3)]
    lib().or_sobel3d(m.ravel(), m.shape[0], m.shape[1], m.shape[2], *out)
    return [o.reshape(m.shape) for o in out]


def downsample(vol, factor):
    v = _c32(vol)
    nz, ny, nx = v.shape
    nh = -(-ny // factor)
    nw = -(-nx // factor)
    out = np.empty(nz * nh * nw, np.float32)
    lib().or_downsample(v.ravel(), nz, ny, nx, factor, out)
    return out.reshape(nz, nh, nw)


def correlation(a, b, mask):
    a = _c32(a).ravel()
    return lib().or_correlation(a, _c32(b).ravel(), np.ascontiguousarray(mask, np.uint8).ravel(), a.size)


def round_bf16(a):
    """float32 -> bfloat16 -> float32, round to nearest even (the conversion the device uses for the
    mixed-precision reference and gradient copies); finite inputs only."""
    b = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def fp64_error_jacobian(ow, reference, gradient, frame, D):
    """One evaluation of the warper's objective and gradient with every product and sum in double,
    on explicitly given stored values (reference, gradient (gx, gy, gz) and frame, e.g. rounded to
    BF16 / FP16), for measuring the error of a reduced-precision evaluation:

      * d(x) = Df D[Di+1] + (1 - Df) D[Di] from the restated interval tables (warpPoint,
        FrameWarper.cpp:397-419);
      * the zero-padded trilinear (bilinear for one plane) sample at x + d (warpImageInterpolated,
        FrameWarper.cpp:31-69; getZeroPadded, FrameWarper.h:39-47);
      * e = sample - reference where the sample is positive, else 0 (computeErrorImage,
        FrameWarper.cpp:4-29; the GPU mask v != 0, GpuFrameWarperKernels.cu:216-218); f = sum e^2;
      * g[k] = sum over storage range k-1 of grad Df e + sum over range k of grad (1 - Df) e, each range
        without its last voxel (computeSteepestDecentImages, FrameWarper.cpp:296-345, and
        computeJacobian, FrameWarper.cpp:147-167).

    Returns (f, g) with g in OptimisationModel's parameter order (P doubles)."""
    nz, ny, nx = ow.dims
    nd = ow.n_dim
    Di, Df, rng = ow.precomp()
    Di = Di.astype(np.int64).ravel()
    Df = Df.astype(np.float64).ravel()
    D = np.asarray(D, np.float64).reshape(ow.nD, 3)
    d = Df[:, None] * D[Di + 1] + (1.0 - Df[:, None]) * D[Di]
    z, y, x = (a.ravel() for a in np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij"))
    lx, ly = x + d[:, 0], y + d[:, 1]
    lz = z + d[:, 2] if nd == 3 else z.astype(np.float64)
    x0, y0, z0 = np.floor(lx), np.floor(ly), np.floor(lz)
    fx, fy, fz = lx - x0, ly - y0, lz - z0
    x0, y0, z0 = x0.astype(np.int64), y0.astype(np.int64), z0.astype(np.int64)
    img = np.asarray(frame, np.float64).reshape(nz, ny, nx)

    def tap(zz, yy, xx):
        ok = (xx >= 0) & (xx < nx) & (yy >= 0) & (yy < ny) & ((zz >= 0) & (zz < nz) if nd == 3 else True)
        v = img[np.clip(zz, 0, nz - 1), np.clip(yy, 0, ny - 1), np.clip(xx, 0, nx - 1)]
        return np.where(ok, v, 0.0)

    def plane(zz):
        return ((tap(zz, y0, x0) * (1 - fx) + tap(zz, y0, x0 + 1) * fx) * (1 - fy) +
                (tap(zz, y0 + 1, x0) * (1 - fx) + tap(zz, y0 + 1, x0 + 1) * fx) * fy)

    val = plane(z0) if nd == 2 else plane(z0) * (1 - fz) + plane(z0 + 1) * fz
    e = np.where(val > 0, val - np.asarray(reference, np.float64).ravel(), 0.0)
    f = float(np.sum(e * e))
    grads = [np.asarray(g_, np.float64).ravel() for g_ in gradient[:nd]]
    g = np.zeros(ow.nD * nd)
    for k in range(ow.nD):
        for kk, w in ((k - 1, Df), (k, 1.0 - Df)):
            if kk < 0 or kk >= ow.nD - 1:
                continue
            b, en = int(rng[kk, 0]), int(rng[kk, 1])
            sl = slice(b, en)
            we = w[sl] * e[sl]
            for c in range(nd):
                g[k * nd + c] += float(np.dot(grads[c][sl], we))
    return f, g


def tr_subproblem(H, g, radius, eps=0.1, max_iter=20):
    H = _c64(H)
    p = np.empty(H.shape[0], np.float64)
    b = lib().or_tr_subproblem(H.shape[0], H, _c64(g), radius, eps, max_iter, p)
    return p, bool(b)


def hann(n):
    """VolumePhaseCorrelator::hann, VolumePhaseCorrelator.cpp:155-166 (square-root Hann)."""
    w = np.ones(n, np.float64)
    if n > 1:
        f = 2.0 * 3.14159265358979323846 / (n - 1)
        w = np.sqrt(0.5 * (1 - np.cos(f * np.arange(n))))
    return w


def phase_window(nz, ny, nx):
    """VolumePhaseCorrelator::computeWindow, VolumePhaseCorrelator.cpp:141-153 (1 along z)."""
    return (np.ones(nz)[:, None, None] * hann(ny)[None, :, None] * hann(nx)[None, None, :])


def phase_correlation_surface(ref, vol):
    """Steps 1-4 of VolumePhaseCorrelator::computeShift (VolumePhaseCorrelator.cpp:57-78)."""
    ref = np.asarray(ref, np.float32).astype(np.float64)
    vol = np.asarray(vol, np.float32).astype(np.float64)
    w = phase_window(*ref.shape)
    R = np.conj(np.fft.rfftn(ref * w))
    X = np.fft.rfftn(vol * w)
    prod = X * R
    prod = prod / (np.abs(prod) + np.finfo(np.float64).tiny)
    return np.fft.irfftn(prod, s=ref.shape, axes=(0, 1, 2)) * ref.size  # unnormalised like FFTW c2r


def phase_shift(ref, vol):
    """Integer shift (x, y, z): first maximum, wrapped at > n/2 (VolumePhaseCorrelator.cpp:81-103)."""
    surf = phase_correlation_surface(ref, vol)
    nz, ny, nx = surf.shape
    idx = int(np.argmax(surf.ravel()))  # numpy returns the first maximum
    x = idx % nx
    y = (idx // nx) % ny
    z = idx // (nx * ny)
    if x > nx // 2:
        x -= nx
    if y > ny // 2:
        y -= ny
    if z > nz // 2:
        z -= nz
    return np.array([x, y, z], np.float64)


def smooth_stack(vol, sigma):
    """or_smooth_stack: smoothStack's per-plane Gaussian (sigma along x, 1 along y)."""
    v = _c32(vol)
    if v.ndim == 2:
        v = v[None]
    out = np.empty_like(v)
    if lib().or_smooth_stack(v.ravel(), v.shape[0], v.shape[1], v.shape[2], float(sigma), out.ravel()) != 0:
        raise ValueError("kernel too large")
    return out


def gaussian_kernel(sigma):
    k = np.empty(257, np.float32)
    n = lib().or_gaussian_kernel(float(sigma), k, 257)
    return k[:n]

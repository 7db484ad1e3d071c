"""Python binding of the C ABI in include/fa_b200.h (ctypes over the in-tree libfa_b200.so).

The classes mirror the reference's warper interface (FrameAligner/FrameWarper.h:95-143 and
FrameAligner/GpuFrameWarper.h:31-72) so that tests read like the reference's own call sequence:

    w = B200FrameWarper(ctx)
    w.setReference(reference, nD, scan_params)       # AbstractFrameWarper::setReference
    w.registerFrame(frame)                           # GpuFrameWarper::registerFrame
    f = w.getError(frame, D)                         # getError -> sum of squared errors
    jac = w.getJacobian(frame, D)                    # getJacobian -> J^T e
    wimg = w.warpImageInterpolated(frame, D, -1)     # warpImageInterpolated
    w.deregisterFrame(frame)

There is no CPU fallback: if libfa_b200.so is missing or no sm_100 device is present, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfa_b200.so")

FA_OK = 0
(FA_ERR_BAD_ARG, FA_ERR_OOM, FA_ERR_CUDA, FA_ERR_TIMEOUT, FA_ERR_UNSUPPORTED, FA_ERR_NOT_FOUND, FA_ERR_STATE,
 FA_ERR_BUSY) = range(1, 9)
STATUS = {0: "ok", 1: "bad argument", 2: "out of memory", 3: "CUDA error", 4: "timeout", 5: "unsupported",
          6: "not found", 7: "bad state", 8: "busy"}
F32, F16, BF16, U16 = 0, 1, 2, 3
PREC_F32, PREC_MIXED = 0, 1
_DTYPES = {np.dtype(np.float32): F32, np.dtype(np.float16): F16, np.dtype(np.uint16): U16}


class FaError(RuntimeError):
    def __init__(self, status, message):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {message}")


class ScanParams(C.Structure):
    """ImageScanParameters fields (FrameAligner/ImageScanParameters.h:22-31)."""
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


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("memory_budget", C.c_size_t), ("autotune", C.c_int)]


class AlignerParams(C.Structure):
    """RealignmentParameters fields read by the aligner (FrameAligner/AbstractFrameAligner.h:31-48)."""
    _fields_ = [
        ("spatial_binning", C.c_int),
        ("n_resampling_points", C.c_int),
        ("nD", C.c_int),
        ("smoothing", C.c_double),
        ("precision", C.c_int),
        ("max_iterations", C.c_int),
        ("correlation_threshold", C.c_double),
        ("coverage_threshold", C.c_double),
    ]


class ServerConfig(C.Structure):
    _fields_ = [("memory_budget", C.c_size_t), ("max_in_flight", C.c_int), ("iterations_per_launch", C.c_int),
                ("warm_start", C.c_int), ("shared_launches", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [
        ("submitted", C.c_longlong), ("completed", C.c_longlong), ("failed", C.c_longlong),
        ("in_flight", C.c_longlong), ("peak_in_flight", C.c_longlong),
        ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double), ("max_ms", C.c_double),
        ("frames_per_s", C.c_double),
        ("slot_bytes", C.c_size_t), ("peak_slot_bytes", C.c_size_t),
        ("graph_launches", C.c_longlong),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class FrameResult(C.Structure):
    _fields_ = [("correlation", C.c_double), ("unaligned_correlation", C.c_double), ("coverage", C.c_double),
                ("use_frame", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AlignStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("evaluations", C.c_int),
        ("accepted", C.c_int),
        ("status", C.c_int),
        ("f_final", C.c_double),
        ("radius_final", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_vp = C.c_void_p

# (name, argtypes) for every entry point declared in include/fa_b200.h
SIGNATURES = {
    "fa_gpu_support": [C.POINTER(C.c_int), C.c_char_p, C.c_size_t],
    "fa_create": [C.POINTER(Config), C.POINTER(_vp)],
    "fa_destroy": [_vp],
    "fa_last_error": [],
    "fa_status_string": [C.c_int],
    "fa_scan_params_init": [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                            C.POINTER(ScanParams)],
    "fa_set_reference": [_vp, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(ScanParams), C.c_int,
                         C.POINTER(_vp)],
    "fa_set_reference_device": [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(ScanParams), C.c_int,
                                C.POINTER(_vp)],
    "fa_reference_destroy": [_vp],
    "fa_reference_info": [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "fa_reference_tuning": [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "fa_reference_retune": [_vp, C.c_int, C.c_int],
    "fa_get_hessian": [_vp, _f64p],
    "fa_get_gradient": [_vp, _vp, _vp, _vp],
    "fa_get_ranges": [_vp, _i32p],
    "fa_register_frame": [_vp, _vp, C.c_int, C.POINTER(_vp)],
    "fa_register_frame_device": [_vp, _vp, C.c_int, C.POINTER(_vp)],
    "fa_update_frame": [_vp, _vp, C.c_int],
    "fa_deregister_frame": [_vp],
    "fa_get_error": [_vp, _f64p, C.POINTER(C.c_double)],
    "fa_get_jacobian": [_vp, _f64p, _f64p],
    "fa_warp": [_vp, _f64p, C.c_float, _f32p],
    "fa_align_frame": [_vp, _vp, C.c_int, _f64p, C.POINTER(AlignStats)],
    "fa_align_batch": [_vp, C.c_int, _vp, C.c_int, _f64p, _vp],
    "fa_correlator_create": [_vp, _f32p, C.c_int, C.c_int, C.c_int, C.POINTER(_vp)],
    "fa_correlator_destroy": [_vp],
    "fa_correlator_shift": [_vp, _f32p, _f64p],
    "fa_correlator_shift_device": [_vp, _vp, _f64p],
    "fa_aligner_create": [_vp, C.c_void_p, C.POINTER(_vp)],
    "fa_aligner_destroy": [_vp],
    "fa_aligner_set_reference": [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(ScanParams)],
    "fa_aligner_info": [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "fa_aligner_reference": [_vp, C.POINTER(_vp)],
    "fa_aligner_add_frames": [_vp, _vp, C.c_int, C.c_int, _f64p, _vp],
    "fa_aligner_add_frames_device": [_vp, _vp, C.c_int, C.c_int, _f64p, _vp],
    "fa_warp_image": [_vp, _f32p, _f64p, _vp, _f32p],
    "fa_aligner_results": [_vp, _vp, C.c_int, C.c_int, _f64p, _vp, _vp, _vp, _vp],
    "fa_shift_pixels": [_vp, _f64p, C.c_longlong, _f64p, _f64p, _f64p],
    "fa_write_realignment_info": [C.c_char_p, C.POINTER(ScanParams), C.c_int, C.c_int, _f64p, _vp],
    "fa_server_create": [_vp, C.POINTER(ServerConfig), C.POINTER(_vp)],
    "fa_server_destroy": [_vp],
    "fa_server_add_acquisition": [_vp, C.POINTER(AlignerParams), _vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(ScanParams), C.c_int, C.POINTER(C.c_int)],
    "fa_server_acquisition_info": [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "fa_server_reserve": [_vp, C.c_int, C.c_int],
    "fa_server_submit": [_vp, C.c_int, _vp, C.c_int, C.POINTER(C.c_ulonglong)],
    "fa_server_wait": [_vp, C.c_ulonglong, C.c_double, _vp, _vp, C.POINTER(C.c_double)],
    "fa_server_get_stats": [_vp, C.POINTER(ServerStats)],
    "fa_server_reset_stats": [_vp],
    "fa_get_error_jacobian_static": [_vp, _vp, C.c_int, _f64p, C.POINTER(C.c_double), _f64p],
    "fa_kernel_launches": [],
    "fa_aligner_last_device_ms": [_vp, C.POINTER(C.c_double)],
    "fa_aligner_last_phase_ms": [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double)],
    "fa_profile_eval": [_vp, C.c_int, _f64p, C.c_int, C.POINTER(C.c_double)],
    "fa_test_tr_subproblem": [_vp, C.c_int, C.c_int, _f64p, _f64p, C.c_double, _f64p, C.POINTER(C.c_int)],
    "fa_test_correlation_surface": [_vp, _f32p, C.c_int, _f64p],
    "fa_test_downsample": [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f32p],
    "fa_test_plane_tables": [C.c_int, C.c_int, C.c_int, _f64p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                             _f64p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)],
}


def lib():
    """Loads libfa_b200.so. Raises if it is missing: there is no fallback path."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                               "(make -C frame-aligner_b200)")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.fa_kernel_launches.restype = C.c_longlong
        L.fa_last_error.restype = C.c_char_p
        L.fa_status_string.restype = C.c_char_p
        _lib = L
    return _lib


def check(status):
    if status != FA_OK:
        raise FaError(status, lib().fa_last_error().decode(errors="replace"))


def gpu_support():
    ok = C.c_int(0)
    msg = C.create_string_buffer(256)
    check(lib().fa_gpu_support(C.byref(ok), msg, 256))
    return bool(ok.value), msg.value.decode()


def scan_params(line, interline, interframe, nx, ny, nz, bidirectional=False) -> ScanParams:
    """ImageScanParameters constructor (FrameAligner/ImageScanParameters.h:7-20)."""
    s = ScanParams()
    check(lib().fa_scan_params_init(line, interline, interframe, nx, ny, nz, int(bidirectional), C.byref(s)))
    return s


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    def __init__(self, device=0, memory_budget=0, autotune=False):
        self._h = _vp()
        # Handles made from this context (frames, references, correlators, aligners, servers) must
        # not outlive it: the context counts its live handles and destroys itself only when the
        # count is zero, when asked to close or after the last handle closed. close() first closes
        # the handles still reachable (frames, then aligners, servers and correlators, then
        # references); handles the garbage collector finalises in the same cycle as the context are
        # unreachable for it, and the last of them to close destroys the context. Handles no longer
        # referenced are collected as usual.
        self._children = weakref.WeakSet()
        self._live = 0
        self._closing = False
        cfg = Config(device, memory_budget, int(autotune))
        check(lib().fa_create(C.byref(cfg), C.byref(self._h)))

    def _adopt(self, obj, rank):
        obj._close_rank = rank
        obj._owner = self
        self._children.add(obj)
        self._live += 1

    def _release(self, obj):
        self._children.discard(obj)
        self._live -= 1
        if self._closing and self._live == 0:
            self._destroy()

    def _destroy(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().fa_destroy(self._h)
            self._h = _vp()

    def close(self):
        if not (getattr(self, "_h", None) and self._h.value) or getattr(self, "_closing", False):
            return
        self._closing = True
        for obj in sorted(list(getattr(self, "_children", ())), key=lambda o: o._close_rank):
            try:
                obj.close()
            except Exception:
                pass
        if getattr(self, "_live", 0) == 0:
            self._destroy()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _released(obj):
    """Takes obj off its context's list of live handles (after obj closed its handle)."""
    owner = getattr(obj, "_owner", None)
    if owner is not None:
        owner._release(obj)
        obj._owner = None


class Reference:
    """A reference volume with its device-resident gradient and Hessian."""

    def __init__(self, ctx: Context, reference, nD, scan: ScanParams, precision=PREC_F32, device_ptr=None,
                 shape=None):
        self.ctx = ctx
        self._h = _vp()
        if device_ptr is not None:
            nz, ny, nx = shape
            check(lib().fa_set_reference_device(ctx._h, device_ptr, nz, ny, nx, int(nD), C.byref(scan), precision,
                                                C.byref(self._h)))
        else:
            ref = np.ascontiguousarray(reference, dtype=np.float32)
            if ref.ndim == 2:
                ref = ref[None]
            nz, ny, nx = ref.shape
            check(lib().fa_set_reference(ctx._h, ref, nz, ny, nx, int(nD), C.byref(scan), precision,
                                         C.byref(self._h)))
        ctx._adopt(self, 2)
        self.dims = (nz, ny, nx)
        self.nD = int(nD)
        self.precision = precision
        nd, P = C.c_int(), C.c_int()
        check(lib().fa_reference_info(self._h, C.byref(nd), C.byref(P)))
        self.n_dim, self.P = nd.value, P.value
        self.N = nz * ny * nx

    def hessian(self):
        H = np.empty((self.P, self.P), np.float64)
        check(lib().fa_get_hessian(self._h, H))
        return H

    def gradient(self):
        g = [np.empty(self.dims, np.float32) for _ in range(3)]
        check(lib().fa_get_gradient(self._h, *[x.ctypes.data for x in g]))
        return g

    def tuning(self):
        t, m = C.c_int(), C.c_int()
        check(lib().fa_reference_tuning(self._h, C.byref(t), C.byref(m)))
        return t.value, m.value

    def retune(self, tile_voxels, ctas_per_sm):
        check(lib().fa_reference_retune(self._h, tile_voxels, ctas_per_sm))

    def warp_image(self, frame, D, want_image=True):
        """fa_warp_image: forward intensity-preserving splat and coverage (AbstractFrameWarper::warpImage)."""
        fr = np.ascontiguousarray(frame, dtype=np.float32).reshape(self.dims)
        cov = np.empty(self.dims, np.float32)
        wimg = np.empty(self.dims, np.float32) if want_image else None
        check(lib().fa_warp_image(self._h, fr, np.ascontiguousarray(D, dtype=np.float64).reshape(-1, 3),
                                  wimg.ctypes.data if want_image else None, cov))
        return wimg, cov

    def shift_pixels(self, D, x, y, z):
        """fa_shift_pixels: FrameWarpAligner::shiftPixel for arrays of photon coordinates (copies)."""
        xs, ys, zs = (np.array(v, dtype=np.float64).ravel() for v in (x, y, z))
        check(lib().fa_shift_pixels(self._h, np.ascontiguousarray(D, dtype=np.float64).reshape(-1, 3), xs.size,
                                    xs, ys, zs))
        return xs, ys, zs

    def ranges(self):
        r = np.empty(2 * self.nD, np.int32)
        check(lib().fa_get_ranges(self._h, r))
        return r.reshape(self.nD, 2)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            check(lib().fa_reference_destroy(self._h))
            self._h = _vp()
            _released(self)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Frame:
    """A registered frame (device copy in the reference's storage precision)."""

    def __init__(self, ref: Reference, data=None, device_ptr=None, dtype=F32):
        self.ref = ref
        self._h = _vp()
        if device_ptr is not None:
            check(lib().fa_register_frame_device(ref._h, device_ptr, dtype, C.byref(self._h)))
        else:
            arr = np.ascontiguousarray(data)
            if arr.dtype not in _DTYPES:
                arr = arr.astype(np.float32)
            self._keep = arr
            check(lib().fa_register_frame(ref._h, arr.ctypes.data, _DTYPES[arr.dtype], C.byref(self._h)))
            self._keep = None
        ref.ctx._adopt(self, 0)

    def update(self, data):
        arr = np.ascontiguousarray(data)
        if arr.dtype not in _DTYPES:
            arr = arr.astype(np.float32)
        check(lib().fa_update_frame(self._h, arr.ctypes.data, _DTYPES[arr.dtype]))

    def get_error(self, D):
        f = C.c_double()
        check(lib().fa_get_error(self._h, _c64(D).ravel(), C.byref(f)))
        return f.value

    def get_jacobian(self, D):
        j = np.empty(self.ref.P, np.float64)
        check(lib().fa_get_jacobian(self._h, _c64(D).ravel(), j))
        return j

    def warp(self, D, invalid_value=0.0):
        out = np.empty(self.ref.N, np.float32)
        check(lib().fa_warp(self._h, _c64(D).ravel(), float(invalid_value), out))
        return out.reshape(self.ref.dims)

    def align(self, rigid_shift=None, max_iterations=100):
        D = np.empty((self.ref.nD, 3), np.float64)
        st = AlignStats()
        rs = None if rigid_shift is None else _c64(rigid_shift)
        check(lib().fa_align_frame(self._h, None if rs is None else rs.ctypes.data, max_iterations, D,
                                   C.byref(st)))
        return D, st.as_dict()

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            check(lib().fa_deregister_frame(self._h))
            self._h = _vp()
            _released(self)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def align_batch(frames, rigid_shifts=None, max_iterations=100):
    n = len(frames)
    handles = (_vp * n)(*[f._h.value for f in frames])
    nD = frames[0].ref.nD
    D = np.empty((n, nD, 3), np.float64)
    stats = (AlignStats * n)()
    rs = None if rigid_shifts is None else _c64(rigid_shifts)
    check(lib().fa_align_batch(C.cast(handles, _vp), n, None if rs is None else rs.ctypes.data, max_iterations, D,
                               C.cast(stats, _vp)))
    return D, [s.as_dict() for s in stats]


class Correlator:
    """VolumePhaseCorrelator (FrameAligner/VolumePhaseCorrelator.h:29-43) on the device."""

    def __init__(self, ctx: Context, reference):
        ref = np.ascontiguousarray(reference, dtype=np.float32)
        if ref.ndim == 2:
            ref = ref[None]
        self.dims = ref.shape
        self._h = _vp()
        check(lib().fa_correlator_create(ctx._h, ref, *ref.shape, C.byref(self._h)))
        ctx._adopt(self, 1)

    def compute_shift(self, volume):
        s = np.empty(3, np.float64)
        vol = np.ascontiguousarray(volume, dtype=np.float32).reshape(self.dims)
        check(lib().fa_correlator_shift(self._h, vol, s))
        return s

    def compute_shift_device(self, ptr):
        s = np.empty(3, np.float64)
        check(lib().fa_correlator_shift_device(self._h, ptr, s))
        return s

    def surface(self, volume, planes=True):
        """Correlation surface of one volume (test hook): fused kx-plane passes or cuFFT."""
        out = np.empty(self.dims, np.float64)
        vol = np.ascontiguousarray(volume, dtype=np.float32).reshape(self.dims)
        check(lib().fa_test_correlation_surface(self._h, vol, 1 if planes else 0, out))
        return out

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().fa_correlator_destroy(self._h)
            self._h = _vp()
            _released(self)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Aligner:
    """FrameWarpAligner's setReference / addFrame flow, batched (fa_aligner_*)."""

    def __init__(self, ctx: Context, spatial_binning=1, n_resampling_points=30, nD=0, precision=PREC_MIXED,
                 max_iterations=100, smoothing=0.0):
        self.ctx = ctx
        self._h = _vp()
        prm = AlignerParams(spatial_binning, n_resampling_points, nD, smoothing, precision, max_iterations)
        check(lib().fa_aligner_create(ctx._h, C.byref(prm), C.byref(self._h)))
        ctx._adopt(self, 1)

    def set_reference(self, reference, scan: ScanParams):
        ref = np.ascontiguousarray(reference)
        if ref.dtype not in (np.float32, np.uint16):
            ref = ref.astype(np.float32)
        if ref.ndim == 2:
            ref = ref[None]
        self.dims = ref.shape
        check(lib().fa_aligner_set_reference(self._h, ref.ctypes.data, _DTYPES[ref.dtype], *ref.shape, C.byref(scan)))
        nD, nd = C.c_int(), C.c_int()
        check(lib().fa_aligner_info(self._h, C.byref(nD), C.byref(nd)))
        self.nD, self.n_dim = nD.value, nd.value

    def add_frames(self, frames):
        """frames: sequence of host arrays (float32 or uint16), one per frame."""
        arrs = [np.ascontiguousarray(f) for f in frames]
        dt = arrs[0].dtype
        if dt not in (np.float32, np.uint16):
            arrs = [a.astype(np.float32) for a in arrs]
            dt = np.dtype(np.float32)
        n = len(arrs)
        ptrs = (_vp * n)(*[a.ctypes.data for a in arrs])
        D = np.empty((n, self.nD, 3), np.float64)
        stats = (AlignStats * n)()
        check(lib().fa_aligner_add_frames(self._h, C.cast(ptrs, _vp), _DTYPES[dt], n, D, C.cast(stats, _vp)))
        return D, [s.as_dict() for s in stats]

    def last_device_ms(self):
        ms = C.c_double()
        check(lib().fa_aligner_last_device_ms(self._h, C.byref(ms)))
        return ms.value

    def last_phase_ms(self):
        """(correlation ms, total ms) of the last add_frames call (fa_aligner_last_phase_ms)."""
        c, t = C.c_double(), C.c_double()
        check(lib().fa_aligner_last_phase_ms(self._h, C.byref(c), C.byref(t)))
        return c.value, t.value

    def reference_gradient(self):
        """The Sobel gradient of the aligner's warper reference (its smoothed reference + 1)."""
        r = _vp()
        check(lib().fa_aligner_reference(self._h, C.byref(r)))
        g = [np.empty(self.dims, np.float32) for _ in range(3)]
        check(lib().fa_get_gradient(r, *[x.ctypes.data for x in g]))
        return g

    def results(self, frames, D, images=False):
        """fa_aligner_results: per frame the metrics dict, and with images=True also the realigned and
        intensity-preserving realigned uint16 images and the coverage mask."""
        arrs = [np.ascontiguousarray(f) for f in frames]
        dt = arrs[0].dtype
        if dt not in (np.float32, np.uint16):
            arrs = [a.astype(np.float32) for a in arrs]
            dt = np.dtype(np.float32)
        n = len(arrs)
        ptrs = (_vp * n)(*[a.ctypes.data for a in arrs])
        D = np.ascontiguousarray(D, dtype=np.float64).reshape(n, self.nD, 3)
        res = (FrameResult * n)()
        if images:
            out = {k: [np.empty(self.dims, t) for _ in range(n)]
                   for k, t in (("realigned", np.uint16), ("realigned_preserving", np.uint16), ("mask", np.float32))}
            pa = {k: (_vp * n)(*[o.ctypes.data for o in v]) for k, v in out.items()}
            check(lib().fa_aligner_results(self._h, C.cast(ptrs, _vp), _DTYPES[dt], n, D, C.cast(res, _vp),
                                           C.cast(pa["realigned"], _vp), C.cast(pa["realigned_preserving"], _vp),
                                           C.cast(pa["mask"], _vp)))
            return [r.as_dict() for r in res], out
        check(lib().fa_aligner_results(self._h, C.cast(ptrs, _vp), _DTYPES[dt], n, D, C.cast(res, _vp), None, None,
                                       None))
        return [r.as_dict() for r in res]

    def add_frames_device(self, ptrs, dtype, n):
        arr = (_vp * n)(*ptrs)
        D = np.empty((n, self.nD, 3), np.float64)
        stats = (AlignStats * n)()
        check(lib().fa_aligner_add_frames_device(self._h, C.cast(arr, _vp), dtype, n, D, C.cast(stats, _vp)))
        return D, [s.as_dict() for s in stats]

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().fa_aligner_destroy(self._h)
            self._h = _vp()
            _released(self)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The serving loop (fa_server_*): several acquisitions, frames submitted asynchronously and
    solved with continuous batching on the device."""

    def __init__(self, ctx: Context, memory_budget=0, max_in_flight=0, iterations_per_launch=0, warm_start=True,
                 shared_launches=False):
        self.ctx = ctx
        self._h = _vp()
        lag = int(warm_start)  # True -> 1 (the previous frame), False -> 0, d -> frame k - d
        cfg = ServerConfig(memory_budget, max_in_flight, iterations_per_launch, lag, 1 if shared_launches else 0)
        check(lib().fa_server_create(ctx._h, C.byref(cfg), C.byref(self._h)))
        ctx._adopt(self, 1)
        self.acqs = {}
        self._keep = {}  # host frames referenced by outstanding tickets

    def add_acquisition(self, reference, scan: ScanParams, frame_dtype=np.uint16, spatial_binning=1, nD=0,
                        n_resampling_points=30, precision=PREC_MIXED, max_iterations=100, smoothing=0.0):
        ref = np.ascontiguousarray(reference)
        if ref.dtype not in (np.float32, np.uint16):
            ref = ref.astype(np.float32)
        if ref.ndim == 2:
            ref = ref[None]
        prm = AlignerParams(spatial_binning, n_resampling_points, nD, smoothing, precision, max_iterations)
        a = C.c_int()
        check(lib().fa_server_add_acquisition(self._h, C.byref(prm), ref.ctypes.data, _DTYPES[ref.dtype], *ref.shape,
                                              C.byref(scan), _DTYPES[np.dtype(frame_dtype)], C.byref(a)))
        nD_, nd = C.c_int(), C.c_int()
        check(lib().fa_server_acquisition_info(self._h, a.value, C.byref(nD_), C.byref(nd)))
        self.acqs[a.value] = {"dims": ref.shape, "nD": nD_.value, "n_dim": nd.value,
                              "dtype": np.dtype(frame_dtype)}
        return a.value

    def reserve(self, acquisition, n_slots):
        """fa_server_reserve: pre-creates frame slots for an acquisition."""
        check(lib().fa_server_reserve(self._h, acquisition, n_slots))

    def submit(self, acquisition, frame):
        """Queues a host frame (kept referenced until its result is collected); returns the ticket."""
        info = self.acqs[acquisition]
        arr = np.ascontiguousarray(frame, dtype=info["dtype"])
        if arr.size != int(np.prod(info["dims"])):
            raise ValueError(f"frame has {arr.size} elements, the acquisition's volume {info['dims']}")
        t = C.c_ulonglong()
        check(lib().fa_server_submit(self._h, acquisition, arr.ctypes.data, 0, C.byref(t)))
        self._keep[t.value] = (acquisition, arr)
        return t.value

    def submit_ptr(self, acquisition, ptr, on_device):
        """Queues a frame at a raw address (device memory when on_device); the caller keeps it valid."""
        t = C.c_ulonglong()
        check(lib().fa_server_submit(self._h, acquisition, ptr, 1 if on_device else 0, C.byref(t)))
        self._keep[t.value] = (acquisition, None)
        return t.value

    def wait(self, ticket, timeout_s=-1.0):
        """Returns (D (nD x 3), stats dict, latency ms) of a ticket."""
        acq, _ = self._keep[ticket]
        D = np.empty((self.acqs[acq]["nD"], 3), np.float64)
        st = AlignStats()
        lat = C.c_double()
        check(lib().fa_server_wait(self._h, ticket, timeout_s, D.ctypes.data, C.cast(C.byref(st), _vp),
                                   C.byref(lat)))
        del self._keep[ticket]
        return D, st.as_dict(), lat.value

    def stats(self):
        s = ServerStats()
        check(lib().fa_server_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    def reset_stats(self):
        check(lib().fa_server_reset_stats(self._h))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().fa_server_destroy(self._h)
            self._h = _vp()
            self._keep.clear()
            _released(self)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def get_error_jacobian_static(ref: Reference, frame_ptr, dtype, D):
    """fa_get_error_jacobian_static: evaluation of a frame in the caller's device memory with the
    library's fixed static scratch (no allocation inside the call)."""
    f = C.c_double()
    jac = np.empty(ref.P, np.float64)
    check(lib().fa_get_error_jacobian_static(ref._h, frame_ptr, dtype, _c64(D).ravel(), C.byref(f), jac))
    return f.value, jac


def kernel_launches():
    return int(lib().fa_kernel_launches())


def profile_eval(frames, D, launches=20):
    n = len(frames)
    handles = (_vp * n)(*[f._h.value for f in frames])
    ms = C.c_double()
    check(lib().fa_profile_eval(C.cast(handles, _vp), n, _c64(D).ravel(), launches, C.byref(ms)))
    return ms.value


def test_tr_subproblem(ctx: Context, nD, n_dim, H, g, radius):
    P = nD * n_dim
    p = np.empty(P, np.float64)
    b = C.c_int()
    check(lib().fa_test_tr_subproblem(ctx._h, nD, n_dim, _c64(H), _c64(g), radius, p, C.byref(b)))
    return p, bool(b.value)


def test_downsample(ctx: Context, volume, factor):
    """fa_test_downsample: the device downsample (AbstractFrameAligner.cpp:37-56) of a float32 or
    uint16 volume (nz, ny, nx)."""
    v = np.ascontiguousarray(volume)
    if v.dtype not in (np.float32, np.uint16):
        v = v.astype(np.float32)
    nz, ny, nx = v.shape
    out = np.empty(nz * (-(-ny // factor)) * (-(-nx // factor)), np.float32)
    check(lib().fa_test_downsample(ctx._h, v.ctypes.data, _DTYPES[v.dtype], nz, ny, nx, factor, out))
    return out.reshape(nz, -(-ny // factor), -(-nx // factor))


def plane_tables(nz, ny, nx):
    """Host-only test hook: twiddle tables and launch shape of the fused phase-correlation passes
    (fa_test_plane_tables). Raises FaError (FA_ERR_UNSUPPORTED) for dimensions that use cuFFT."""
    tx = np.empty(2 * max(nx, 1), np.float64)
    ty = np.empty(2 * max(ny, 1), np.float64)
    n_x, x_post, n_y, g, pp = (C.c_int() for _ in range(5))
    check(lib().fa_test_plane_tables(nz, ny, nx, tx, nx, C.byref(n_x), C.byref(x_post), ty, ny, C.byref(n_y),
                                     C.byref(g), C.byref(pp)))
    as_c = lambda a, n: a[: 2 * n].reshape(n, 2) @ np.array([1.0, 1.0j])
    return {"tw_x": as_c(tx, n_x.value), "x_post": x_post.value, "tw_y": as_c(ty, n_y.value),
            "rows_per_cta": g.value, "planes_per_cta": pp.value}


class B200FrameWarper:
    """AbstractFrameWarper-shaped facade (FrameAligner/FrameWarper.h:95-143) over the C ABI.

    Frames are identified by the identity of the numpy array passed to registerFrame, the way the
    reference identifies cv::Mat frames by their data pointer (GpuFrameWarper.h:55)."""

    def __init__(self, ctx: Context, precision=PREC_F32):
        self.ctx = ctx
        self.precision = precision
        self.reference = None
        self.frames = {}

    def setReference(self, reference, nD, scan: ScanParams):
        self.reference = Reference(self.ctx, reference, nD, scan, self.precision)
        self.n_dim = self.reference.n_dim
        self.dims = list(self.reference.dims)
        self.H = self.reference.hessian()

    def registerFrame(self, frame):
        self.frames[id(frame)] = Frame(self.reference, frame)

    def deregisterFrame(self, frame):
        fr = self.frames.pop(id(frame))
        fr.close()

    def _frame(self, frame):
        if id(frame) not in self.frames:
            raise FaError(6, "Unrecognised frame")  # GpuFrameWarper.cpp:162-167
        return self.frames[id(frame)]

    def getError(self, frame, D):
        return self._frame(frame).get_error(D)

    def getJacobian(self, frame, D):
        return self._frame(frame).get_jacobian(D)

    def warpImageInterpolated(self, frame, D, invalid_value=0):
        return self._frame(frame).warp(D, invalid_value)


def write_realignment_info(filename, scan: ScanParams, D, results):
    """fa_write_realignment_info: D (n, nD, 3), results: list of FrameResult dicts."""
    D = np.ascontiguousarray(D, dtype=np.float64)
    n, nD = D.shape[0], D.shape[1]
    res = (FrameResult * max(n, 1))()
    for i, r in enumerate(results):
        res[i] = FrameResult(r["correlation"], r["unaligned_correlation"], r["coverage"], r.get("use_frame", 1))
    check(lib().fa_write_realignment_info(filename.encode(), C.byref(scan), n, nD, D.reshape(-1) if n else
                                          np.zeros(3), C.cast(res, _vp)))

"""CPU: host logic of the fused phase-correlation passes (csrc/fa_plane_corr.cu), through the host-only
test hook fa_test_plane_tables -- which dimensions take the fused path, the launch shape, and the
twiddle tables the kernels index.

The second test restates the three passes in numpy with exactly those tables and the kernels' stage
order (in-place Stockham stages: radix 8 while three octaves are left, then 4 or 2; stage twiddles
at (r - 1) Ns + k; the nx/2-point packing of each real row, the half-spectrum split and fold, and the
kx-plane layout spec[kx][z][y]), and compares the resulting correlation surface with numpy's FP64
DFT of VolumePhaseCorrelator.cpp:57-103: |model - cpu| <= 1e-9 * max|cpu|. The GPU tests compare the
kernels themselves with the same CPU DFT (tests/test_gpu_plane_corr.py).
"""
import numpy as np
import pytest

import fa_b200 as fa

SHAPES = [(1, 8, 16), (2, 16, 16), (1, 64, 64), (4, 64, 128), (16, 32, 64), (8, 8, 32), (1, 256, 512),
          (2, 16, 1024), (4, 2048, 16), (1, 8, 4096)]
# planes of more than 8192 points or nz > 16: the (z, y) pass split into y lines and z columns
SPLIT_SHAPES = [(32, 16, 16), (64, 32, 32), (16, 1024, 32), (8, 2048, 16), (128, 16, 64)]


def _stages(L):
    """(R, Ns) of every stage of an L-point transform, in the kernels' order."""
    out, log2L, log2Ns = [], L.bit_length() - 1, 0
    while log2Ns < log2L:
        log2R = min(3, log2L - log2Ns)
        out.append((1 << log2R, 1 << log2Ns))
        log2Ns += log2R
    return out


def _root(m, n):
    """exp(-2 pi i m / n) computed in long double and rounded to double (as the library does)."""
    ang = np.longdouble("6.283185307179586476925286766559") * np.asarray(m, np.longdouble) / np.longdouble(n)
    return np.cos(ang).astype(np.float64) - 1j * np.sin(ang).astype(np.float64)


def _stage_table(L):
    t = []
    for R, Ns in _stages(L):
        if Ns > 1:
            for r in range(1, R):
                t.extend(_root(r * np.arange(Ns), Ns * R))
    return np.array(t, np.complex128)


def _fft_rows(x, tw, inverse):
    """The kernels' in-place Stockham stages over the last axis of x, twiddles from tw."""
    L = x.shape[-1]
    sign = 1.0 if inverse else -1.0
    off = 0
    for R, Ns in _stages(L):
        q = L // R
        j = np.arange(q)
        k = j % Ns
        a = np.stack([x[..., j + r * q] for r in range(R)], axis=-2)  # (..., R, q)
        if Ns > 1:
            for r in range(1, R):
                w = tw[off + (r - 1) * Ns + k]
                a[..., r, :] *= np.conj(w) if inverse else w
            off += (R - 1) * Ns
        n = np.arange(R)
        dft = np.exp(sign * 2j * np.pi * np.outer(n, n) / R)
        a = np.einsum("rs,...sq->...rq", dft, a)
        y = np.empty_like(x)
        o = (j - k) * R + k
        for r in range(R):
            y[..., o + r * Ns] = a[..., r, :]
        x = y
    return x


def _hann(n):
    if n == 1:
        return np.ones(1)
    return np.sqrt(0.5 * (1 - np.cos(2 * np.pi / (n - 1) * np.arange(n))))


def _model_surface(t, reference, volume):
    nz, ny, nx = reference.shape
    M = nx // 2
    tw_stage_x, W = t["tw_x"][: t["x_post"]], t["tw_x"][t["x_post"]:]
    wy, wx = _hann(ny), _hann(nx)

    def pass_rows_fwd(vol):  # window + real DFT along x, planes spec[kx][r], r = z * ny + y
        rows = (vol.astype(np.float64) * (wy[None, :, None] * wx[None, None, :])).reshape(nz * ny, nx)
        Z = _fft_rows(rows[:, 0::2] + 1j * rows[:, 1::2], tw_stage_x, False)
        k = np.arange(M + 1)
        zk, zm = Z[:, k % M], np.conj(Z[:, (M - k) % M])
        X = 0.5 * (zk + zm) - 0.5j * W[k] * (zk - zm)
        return X.T.reshape(M + 1, nz, ny)

    split = t["planes_per_cta"] == 0
    tw_z = _stage_table(nz)

    def along_z(a, inverse):  # z by the stage tables (split pass) or any exact DFT (z in registers)
        if split:
            return np.swapaxes(_fft_rows(np.swapaxes(a, 1, 2), tw_z, inverse), 1, 2)
        return np.fft.ifft(a, axis=1) * nz if inverse else np.fft.fft(a, axis=1)

    def pass_yz(spec, ref_conj):
        F = along_z(_fft_rows(spec, t["tw_y"], False), False)  # y by the tables
        if ref_conj is None:
            return np.conj(F)
        c = F * ref_conj
        q = np.abs(c) ** 2
        c = np.where(q > 0, c / np.sqrt(np.where(q > 0, q, 1.0)), 0)
        return _fft_rows(along_z(c, True), t["tw_y"], True)

    def pass_rows_inv(spec):
        X = spec.reshape(M + 1, nz * ny).T
        k = np.arange(M)
        xa, xb = X[:, k], np.conj(X[:, M - k])
        Z = (xa + xb) + 1j * ((xa - xb) * np.conj(W[k]))
        z = _fft_rows(Z, tw_stage_x, True)
        out = np.empty((nz * ny, nx))
        out[:, 0::2], out[:, 1::2] = z.real, z.imag
        return out.reshape(nz, ny, nx)

    ref_conj = pass_yz(pass_rows_fwd(reference), None)
    return pass_rows_inv(pass_yz(pass_rows_fwd(volume), ref_conj))


def _cpu_surface(reference, volume):
    nz, ny, nx = reference.shape
    w = _hann(ny)[None, :, None] * _hann(nx)[None, None, :]
    c = np.fft.fftn(volume.astype(np.float64) * w) * np.conj(np.fft.fftn(reference.astype(np.float64) * w))
    c = c / (np.abs(c) + np.finfo(np.float64).tiny)
    return np.fft.ifftn(c).real * c.size


@pytest.mark.parametrize("shape", SHAPES + SPLIT_SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_tables_and_launch_shape(shape):
    nz, ny, nx = shape
    t = fa.plane_tables(*shape)
    M = nx // 2
    # the tables are W^m rounded from long double: equal to a long-double statement within 2 ulp
    assert t["x_post"] == len(_stage_table(M))
    assert np.abs(t["tw_x"][: t["x_post"]] - _stage_table(M)).max(initial=0) <= 2.3e-16
    assert np.abs(t["tw_x"][t["x_post"]:] - _root(np.arange(M + 1), nx)).max() <= 2.3e-16
    assert np.abs(t["tw_y"] - _stage_table(ny)).max(initial=0) <= 2.3e-16
    assert len(t["tw_x"]) <= nx and len(t["tw_y"]) < ny  # the kernels' twiddle slots
    assert t["rows_per_cta"] == min(8, nz * ny, 2048 // M)
    split = nz > 16 or nz * ny > 8192
    assert t["planes_per_cta"] == (0 if split else max(1, 8192 // (nz * ny)))


@pytest.mark.parametrize("shape", SHAPES[:8] + SPLIT_SHAPES[:3], ids=lambda s: "x".join(map(str, s)))
def test_pass_structure_matches_dft(shape):
    nz, ny, nx = shape
    rng = np.random.default_rng(nz * 7 + ny * 3 + nx)
    ref = (rng.random(shape) * 1000).astype(np.float32)
    vol = (np.roll(ref, (1 % nz, -3 % ny, 5 % nx), axis=(0, 1, 2)) + rng.random(shape) * 50).astype(np.float32)
    got = _model_surface(fa.plane_tables(*shape), ref, vol)
    want = _cpu_surface(ref, vol)
    assert np.abs(got - want).max() <= 1e-9 * np.abs(want).max()
    assert int(np.argmax(got)) == int(np.argmax(want))


@pytest.mark.parametrize("shape", [(3, 20, 30), (2, 8, 8192), (1, 4, 64), (1, 64, 12), (1, 4096, 16), (1, 8, 8192),
                                   (2048, 16, 16), (32, 8, 16)],
                         ids=lambda s: "x".join(map(str, s)))
def test_other_dimensions_take_cufft(shape):
    with pytest.raises(fa.FaError):
        fa.plane_tables(*shape)

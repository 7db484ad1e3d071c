"""The serving loop (fa_server_*): continuous batching of frames from several acquisitions.

Tolerances (stated per check):
  * served frames without warm start vs fa_aligner_add_frames on the same raw frames: the same
    kernels and per-frame arithmetic, |dD| <= 1e-9 px;
  * a frame's result alone vs in a mix with other acquisitions' frames: identical, bit for bit
    (tolerance 0) -- a frame's fused passes and steps use only its own tiles, sums and state;
  * a warm-started chain (each frame also starts from the previous frame's solution) vs the
    oracle's warm-started chain over the same frames: RMS over control points <= 0.01 px per frame.
"""
import threading

import numpy as np
import pytest

import fa_b200 as fa
import fa_synth as S
import oracle_py as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    ok, msg = fa.gpu_support()
    assert ok, msg
    return fa.Context()


def _scan(acq):
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    return fa.scan_params(line, il, ifr, nx, ny, nz)


def _rms(a, b, n_dim):
    d = (np.asarray(a) - np.asarray(b))[..., :n_dim]
    return float(np.sqrt((d ** 2).sum(-1).mean()))


def _acq(shape, nD, n_frames, seed, step=1.0, bound=4.0):
    nblobs = int(200 * shape[1] * shape[2] / 65536) + 10
    walk = S.WalkSpec(step, bound, 0.2 if shape[0] > 1 else 0.0, 1.0 if shape[0] > 1 else 0.0)
    return S.make_acquisition(shape, nD, n_frames, S.BlobSpec(nblobs, (2.0, 6.0), (1.0, 2.0), mean=20.0), walk,
                              seed=seed, continue_walk=True)


@pytest.fixture(scope="module")
def acqs():
    """Three acquisitions of different sizes and kinds: a 3-D stack, a plane, and a plane whose row
    width is not a multiple of 4 (the scalar fused-pass class)."""
    return {
        "stack": _acq((4, 64, 128), 13, 6, 71),
        "plane": _acq((1, 256, 256), 10, 6, 72),
        "odd": _acq((1, 96, 98), 8, 6, 73),
    }


def _raw(acq):
    return np.ascontiguousarray(acq.frames.astype(np.uint16))


def _server(ctx, acqs, names, precision=fa.PREC_MIXED, **kw):
    srv = fa.Server(ctx, **kw)
    ids = {}
    for name in names:
        a = acqs[name]
        ids[name] = srv.add_acquisition(a.reference, _scan(a), frame_dtype=np.uint16, nD=a.nD, precision=precision)
    return srv, ids


def _run_sequence(srv, acq_id, frames):
    tickets = [srv.submit(acq_id, f) for f in frames]
    return [srv.wait(t, 120.0) for t in tickets]


@pytest.mark.parametrize("shared", [False, True])
def test_served_equals_aligner_without_warm_start(ctx, acqs, shared):
    names = ["stack", "plane", "odd"]
    srv, ids = _server(ctx, acqs, names, warm_start=False, shared_launches=shared)
    tickets = {n: [] for n in names}
    for k in range(6):  # interleaved submissions: the acquisitions share launches
        for n in names:
            tickets[n].append(srv.submit(ids[n], _raw(acqs[n])[k]))
    served = {n: np.array([srv.wait(t, 120.0)[0] for t in tickets[n]]) for n in names}
    st = srv.stats()
    srv.close()
    assert st["completed"] == 18 and st["failed"] == 0
    for n in names:
        a = acqs[n]
        al = fa.Aligner(ctx, nD=a.nD, precision=fa.PREC_MIXED)
        al.set_reference(a.reference, _scan(a))
        D, _ = al.add_frames([_raw(a)[k] for k in range(6)])
        al.close()
        assert np.max(np.abs(served[n] - D)) <= 1e-9, (n, np.max(np.abs(served[n] - D)))


@pytest.mark.parametrize("lag,shared", [(1, False), (1, True), (3, True)])
def test_alone_equals_mix_with_warm_start(ctx, acqs, lag, shared):
    names = ["stack", "plane", "odd"]
    alone = {}
    srv, ids = _server(ctx, acqs, names, warm_start=lag, shared_launches=shared)
    for n in names:  # one acquisition at a time
        alone[n] = np.array([r[0] for r in _run_sequence(srv, ids[n], _raw(acqs[n]))])
    srv.close()

    srv, ids = _server(ctx, acqs, names, warm_start=lag, shared_launches=shared)
    out, errors = {}, []

    def feed(n):
        try:
            out[n] = np.array([r[0] for r in _run_sequence(srv, ids[n], _raw(acqs[n]))])
        except Exception as e:  # reported below
            errors.append((n, e))

    threads = [threading.Thread(target=feed, args=(n,)) for n in names]
    for t in threads:
        t.start()
    for t in threads:
        t.join(300)
    st = srv.stats()
    srv.close()
    assert not errors, errors
    assert st["completed"] == 18
    for n in names:
        assert np.array_equal(alone[n], out[n]), (n, np.max(np.abs(alone[n] - out[n])))


@pytest.mark.parametrize("lag", [1, 2])
def test_warm_chain_against_oracle(ctx, acqs, lag):
    """F32 storage; the oracle chain feeds frame k the oracle's own solution of frame k - lag."""
    a = acqs["stack"]
    nz, ny, nx = a.reference.shape
    line, il, ifr = a.scan
    srv = fa.Server(ctx, warm_start=lag)
    aid = srv.add_acquisition(a.reference, _scan(a), frame_dtype=np.uint16, nD=a.nD, precision=fa.PREC_F32)
    served = _run_sequence(srv, aid, _raw(a))
    srv.close()
    ow = O.OracleWarper(a.reference + 1, a.nD, O.scan_init(line, il, ifr, nx, ny, nz))
    cpu = []
    for k in range(a.frames.shape[0]):
        shift = O.phase_shift(a.reference, a.frames[k])
        D_cpu, _ = ow.align_frame(a.frames[k] + 1, shift, 100, warm=cpu[k - lag] if k >= lag else None)
        cpu.append(D_cpu)
        assert _rms(served[k][0], D_cpu, 3) <= 0.01, (k, _rms(served[k][0], D_cpu, 3))


def test_memory_budget_admission(ctx, acqs):
    """A budget of about two frame slots: frames queue for slots, results are unchanged."""
    a = acqs["stack"]
    srv, ids = _server(ctx, acqs, ["stack"], warm_start=False)
    ref = _run_sequence(srv, ids["stack"], _raw(a))
    st = srv.stats()
    srv.close()
    per_slot = st["peak_slot_bytes"] / max(1, st["peak_in_flight"])
    budget = int(2.5 * per_slot)
    srv, ids = _server(ctx, acqs, ["stack"], warm_start=False, memory_budget=budget)
    got = _run_sequence(srv, ids["stack"], _raw(a))
    st2 = srv.stats()
    srv.close()
    assert st2["peak_slot_bytes"] <= budget
    assert st2["peak_in_flight"] <= 2
    for r, g in zip(ref, got):
        assert np.array_equal(r[0], g[0])


def test_device_submissions(ctx, acqs):
    import torch

    a = acqs["plane"]
    raw = _raw(a)
    srv, ids = _server(ctx, acqs, ["plane"], warm_start=True)
    host = [r[0] for r in _run_sequence(srv, ids["plane"], raw)]
    srv.close()
    dev = torch.from_numpy(raw.view(np.int16)).to("cuda:0")
    torch.cuda.synchronize()
    srv, ids = _server(ctx, acqs, ["plane"], warm_start=True)
    tickets = [srv.submit_ptr(ids["plane"], dev[k].data_ptr(), True) for k in range(raw.shape[0])]
    got = [srv.wait(t, 120.0)[0] for t in tickets]
    srv.close()
    for h, g in zip(host, got):
        assert np.array_equal(h, g)


def test_server_errors(ctx, acqs):
    a = acqs["plane"]
    srv = fa.Server(ctx, memory_budget=1 << 16)  # smaller than one slot (~280 KB)
    with pytest.raises(fa.FaError) as e:
        srv.add_acquisition(a.reference, _scan(a), frame_dtype=np.uint16, nD=a.nD)
    assert e.value.status == fa.FA_ERR_OOM
    srv.close()
    srv, ids = _server(ctx, acqs, ["plane"])
    with pytest.raises(fa.FaError) as e:
        srv.submit_ptr(7, 1, False)
    assert e.value.status == fa.FA_ERR_NOT_FOUND
    with pytest.raises(fa.FaError) as e:
        fa.check(fa.lib().fa_server_wait(srv._h, 12345, 0.0, None, None, None))
    assert e.value.status == fa.FA_ERR_NOT_FOUND
    srv.close()


def test_reserve_slots(ctx, acqs):
    """fa_server_reserve creates the slots up front (results unchanged); a budget that cannot hold
    them is reported."""
    a = acqs["stack"]
    srv, ids = _server(ctx, acqs, ["stack"], warm_start=False)
    ref = _run_sequence(srv, ids["stack"], _raw(a))
    per_slot = srv.stats()["peak_slot_bytes"] / 6
    srv.close()
    srv, ids = _server(ctx, acqs, ["stack"], warm_start=False)
    srv.reserve(ids["stack"], 4)
    held = srv.stats()["slot_bytes"]
    assert abs(held - 4 * per_slot) <= 1e-6 * held
    got = _run_sequence(srv, ids["stack"], _raw(a))
    srv.close()
    for r, g in zip(ref, got):
        assert np.array_equal(r[0], g[0])
    srv, ids = _server(ctx, acqs, ["stack"], warm_start=False, memory_budget=int(2.5 * per_slot))
    with pytest.raises(fa.FaError) as e:
        srv.reserve(ids["stack"], 4)
    assert e.value.status == fa.FA_ERR_OOM
    assert srv.stats()["slot_bytes"] <= 2.5 * per_slot
    srv.close()

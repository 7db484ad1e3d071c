"""The N > 1 path of bench.py on CPU: two `gloo` ranks, each aligning its own seeded frames with the
CPU oracle (the data path has no collective), then the max-over-ranks reduction the bench uses for
its timings. Each rank's result must equal the same shard computed in a single process."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import fa_synth as S  # noqa: E402

SMALL = dict(shape=(1, 64, 96), nD=6, n_frames=2, blobs=S.BlobSpec(30, (2.0, 5.0), (1.0, 1.0), mean=20.0),
             walk=S.WalkSpec(1.0, 3.0), seed=11)


def _shard(rank):
    import bench
    import oracle_py as O

    acq = bench.make_data(2, rank, cfg=SMALL)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
    out = []
    for k in range(acq.frames.shape[0]):
        shift = O.phase_shift(acq.reference, acq.frames[k])
        D, _ = ow.align_frame(acq.frames[k] + 1, shift, 100)
        out.append(D)
    return np.array(out)


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        D = _shard(rank)
        slowest = bench.max_over_ranks(float(rank + 1), dist, "cpu")
        gathered = [None] * world
        dist.all_gather_object(gathered, D)
        q.put((rank, slowest, gathered))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_sharding_and_max():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    single = [_shard(r) for r in range(world)]
    assert not np.array_equal(single[0], single[1])  # ranks really hold different frames
    for rank, slowest, gathered in results:
        assert slowest == float(world)
        for r in range(world):
            assert np.array_equal(gathered[r], single[r])

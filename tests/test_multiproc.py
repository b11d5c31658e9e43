"""Multi-rank host logic on CPU: world_size-2 gloo process groups run the
frame sharding and the gather; the per-shard compute is the CPU oracle here
(on GPUs it is the CUDA library)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from warp_md import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    import oracle
    from warp_md import synth

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        fr, ref = synth.make_trajectory(64, 13, 0.4, seed=5)  # every rank builds the same data
        got = shard.run_sharded(lambda a, b: oracle.rmsd_frames(fr[a:b], ref)[1], fr.shape[0])
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_frame_range_partitions():
    for n in (0, 1, 7, 13, 100):
        for w in (1, 2, 3, 8):
            spans = [shard.frame_range(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a <= b for a, b in spans)
            assert all(spans[i][1] == spans[i + 1][0] for i in range(w - 1))
            assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1
    with pytest.raises(ValueError):
        shard.frame_range(5, 2, 2)


def test_two_gloo_ranks_gather_the_full_series():
    import oracle
    from warp_md import synth

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    fr, ref = synth.make_trajectory(64, 13, 0.4, seed=5)
    _, exp = oracle.rmsd_frames(fr, ref)
    for r in (0, 1):
        np.testing.assert_array_equal(results[r], exp)

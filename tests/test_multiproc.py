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


def _oracle_part(frames, part, parts, rows=8):
    """CPU stand-in for one GPU's wmd_pairwise_rmsd_part: the oracle's matrix
    (plan.rs:593-674) restricted to the pairs i < j whose row block of `rows`
    frames is part (mod parts), mirrored, zeros elsewhere."""
    import torch

    import oracle

    _, full = oracle.pairwise(frames.numpy(), "rms")
    i, j = np.triu_indices(full.shape[0], k=1)
    keep = (i // rows) % parts == part
    out = np.zeros(full.shape, np.float32)
    out[i[keep], j[keep]] = full[i[keep], j[keep]]
    out[j[keep], i[keep]] = full[i[keep], j[keep]]
    return torch.from_numpy(out)


def _pair_worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    from warp_md import synth

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        full = synth.make_drift_trajectory(50, 37, 0.1, seed=9)  # every rank builds the same data
        f0, f1 = shard.frame_range(full.shape[0], rank, world)
        local = torch.from_numpy(full[f0:f1].copy())
        gathered = shard.gather_frames(local, full.shape[0])
        everyone = shard.pairwise_sharded(local, full.shape[0], compute_part=_oracle_part)
        at_root = shard.pairwise_sharded(local, full.shape[0], compute_part=_oracle_part, dst=0)
        q.put((rank, gathered.numpy(), everyone.numpy(), None if at_root is None else at_root.numpy()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_assemble_the_all_pairs_matrix_from_tile_rows():
    """Frames split 18/19 over two ranks: the all_gather restores the whole
    trajectory on both, each rank computes its tile rows, and the summed parts
    equal the oracle's one-process matrix exactly (all_reduce on every rank,
    reduce to rank 0)."""
    import oracle
    from warp_md import synth

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_pair_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    for _ in procs:
        rank, gathered, everyone, at_root = q.get(timeout=300)
        results[rank] = (gathered, everyone, at_root)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = synth.make_drift_trajectory(50, 37, 0.1, seed=9)
    _, exp = oracle.pairwise(full, "rms")
    exp32 = exp.astype(np.float32)
    for r in (0, 1):
        gathered, everyone, at_root = results[r]
        np.testing.assert_array_equal(gathered, full)
        np.testing.assert_array_equal(everyone, exp32)
    np.testing.assert_array_equal(results[0][2], exp32)
    assert results[1][2] is None

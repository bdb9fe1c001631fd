"""Sample-sharded replicas (swiftimpute_b200.replicas) with two gloo ranks on
the CPU: each rank takes its shard of the targets, the shards gathered at rank 0
equal the whole batch, and a step's time is the slowest rank's. The oracle
stands in for each rank's device work (no GPU here)."""
import os
import socket

import numpy as np
import pytest

from swiftimpute_b200.replicas import gather_rows, max_over_ranks, shard


def test_shards_cover_rows_in_order():
    for n in (0, 1, 7, 10, 1001):
        for world in (1, 2, 3, 8):
            spans = [shard(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard(10, 2, 2)


def _workload():
    from swiftimpute_b200 import synth
    panel, pos, _ = synth.make_panel(240, 128, 8, seed=77, spacing=1000)
    codes, _, _ = synth.make_targets(panel, 11, synth.typed_every(240, 4), seed=78)
    return panel, pos, codes


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        panel, pos, codes = _workload()
        pairs = oracle.select_pairs(oracle.pbwt_build(panel), 8)   # every rank holds the panel and index
        a, b = shard(codes.shape[0], world, rank)
        local = oracle.fb_batch(codes[a:b], pairs, panel, pos, 8, 10000.0, threads=1)["dosage"]
        whole = gather_rows(local, dist)
        slowest = max_over_ranks(10.0 + rank, dist)
        if rank == 0:
            np.save(os.path.join(out_dir, "whole.npy"), whole)
            np.save(os.path.join(out_dir, "slowest.npy"), np.array([slowest]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_gather_the_whole_batch(tmp_path):
    import torch.multiprocessing as mp
    import oracle
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    panel, pos, codes = _workload()
    pairs = oracle.select_pairs(oracle.pbwt_build(panel), 8)
    want = oracle.fb_batch(codes, pairs, panel, pos, 8, 10000.0, threads=1)["dosage"]
    got = np.load(tmp_path / "whole.npy")
    assert np.array_equal(got, want)  # same FP64 computation, row by row
    assert np.load(tmp_path / "slowest.npy")[0] == 10.0 + (world - 1)

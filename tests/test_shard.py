"""Shot sharding across processes (the multi-GPU path) on CPU: two gloo ranks
each run one contiguous range of global shots through the oracle with the
device's Philox streams, rank 0 gathers; the merged records must equal one
process running every shot."""

from __future__ import annotations

import datetime
import os
import socket

import numpy as np
import pytest

from clifft_b200 import shard

PROG = os.path.join(os.path.dirname(__file__), "golden", "programs", "cfg1.npz")


def test_shard_range_partitions_every_shot():
    for total in (0, 1, 7, 1000, 1001):
        for world in (1, 2, 3, 8):
            spans = [shard.shard_range(total, world, r) for r in range(world)]
            covered = [i for first, n in spans for i in range(first, first + n)]
            assert covered == list(range(total))
            sizes = [n for _, n in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.shard_range(10, 2, 2)


def _oracle_sampler(program, shots, seed, first_shot, precision, survivors):
    from oracle import pyoracle as O
    r = O.run(program, shots, seed=seed, rng=O.RNG_PHILOX, first_shot=first_shot)
    return {"meas": r["meas"], "det": r["det"], "obs": r["obs"], "discarded": r["discarded"],
            "passed_shots": int((r["discarded"] == 0).sum())}


def _worker(rank, world, port, total, seed, out_path):
    import torch.distributed as dist
    from clifft_b200.program import Program
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = shard.sample_sharded(Program.load(PROG), total, seed, sampler=_oracle_sampler)
        if rank == 0:
            np.savez(out_path, **{k: np.asarray(v) for k, v in res.items()})
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_match_one_process(tmp_path):
    import torch.multiprocessing as mp
    from clifft_b200.program import Program
    from oracle import pyoracle as O
    total, seed = 3001, 17
    out = str(tmp_path / "merged.npz")
    mp.spawn(_worker, args=(2, _free_port(), total, seed, out), nprocs=2, join=True)
    merged = np.load(out)
    one = O.run(Program.load(PROG), total, seed=seed, rng=O.RNG_PHILOX)
    for key in ("meas", "det", "obs", "discarded"):
        assert np.array_equal(merged[key], one[key]), key
    assert int(merged["passed_shots"]) == int((one["discarded"] == 0).sum())

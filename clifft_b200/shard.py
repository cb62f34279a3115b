"""Shot sharding over GPUs: one process per GPU (torch.distributed), each
sampling a contiguous range of global shot indices.

Every shot draws from its own Philox stream, keyed by the seed and its global
index (`first_shot` + local index), so the union of the shards is the same set
of records a single GPU produces for the whole range, whatever the number of
ranks. There is no collective on the data path: each rank samples its range,
then the records are gathered once to rank 0 (concatenated in rank order) and
the counters summed. The reference loops over shots with no cross-shot state
other than its RNG stream (src/clifft/svm/svm.cc:218-252), which is what makes
this split exact.
"""

from __future__ import annotations

from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

# per-call totals that are summed over shards; every other array is per shot
SUM_KEYS = ("passed_shots", "logical_errors", "observable_ones", "dust_clamps")


def shard_range(total_shots: int, world: int, rank: int) -> Tuple[int, int]:
    """(first_shot, shots) of `rank`: contiguous, sizes differing by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    if total_shots < 0:
        raise ValueError("total_shots must be non-negative")
    base, extra = divmod(total_shots, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def gpu_sampler(program, shots: int, seed: int, first_shot: int, precision: str,
                survivors: bool) -> Dict[str, object]:
    """One shard on this process's current CUDA device (clifft_gpu_sample)."""
    from . import api
    r = api.run(program, shots, seed, precision=precision, survivors=survivors, first_shot=first_shot)
    keys = ("meas_words", "det_words", "obs_words", "exp_vals", "survived", "passed_shots",
            "logical_errors", "observable_ones", "dust_clamps")
    return {k: r[k] for k in keys}


def merge(parts: List[Dict[str, object]]) -> Dict[str, object]:
    """Records concatenated in rank (= global shot) order, totals summed."""
    out: Dict[str, object] = {}
    for key in parts[0]:
        vals = [p[key] for p in parts]
        if key in SUM_KEYS:
            out[key] = sum(np.asarray(v, dtype=np.int64) for v in vals)
            if np.ndim(out[key]) == 0:
                out[key] = int(out[key])
        else:
            out[key] = np.concatenate([np.asarray(v) for v in vals], axis=0)
    return out


def sample_sharded(program, total_shots: int, seed: int, *, precision: str = "fp32",
                   survivors: bool = False, sampler: Optional[Callable] = None,
                   group=None) -> Optional[Dict[str, object]]:
    """Sample `total_shots` shots split over the ranks of the default (or given)
    process group. Returns the merged result on rank 0 and None elsewhere
    (every rank returns the merged result when torch.distributed is not
    initialised). `sampler(program, shots, seed, first_shot, precision,
    survivors)` runs one shard (default: the GPU executor)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        world, rank = dist.get_world_size(group), dist.get_rank(group)
    else:
        world, rank = 1, 0
    first, count = shard_range(total_shots, world, rank)
    local = (sampler or gpu_sampler)(program, count, seed, first, precision, survivors)
    if world == 1:
        return merge([local])
    parts = [None] * world if rank == 0 else None
    dist.gather_object(local, parts, dst=0, group=group)
    return merge(parts) if rank == 0 else None

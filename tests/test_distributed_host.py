"""Sample sharding of one frame across ranks, on CPU: the shard partition,
the exact resolve of fixed-point sums, and a world-size-2 gloo all-reduce of
per-rank sums that must equal the single-process result bit for bit.  The
per-sample values are synthetic integers keyed by (pixel, sample), standing
in for the device's fixed-point path samples."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from ordinarylight_b200.distributed import ACCUM_SCALE, resolve_sums, sample_shard


def _synthetic_sums(h, w, first, count):
    """Fixed-point sums of samples [first, first + count) of every pixel."""
    pix = np.arange(h * w, dtype=np.uint64).reshape(h, w, 1)
    total = np.zeros((h, w, 3), np.uint64)
    for s in range(first, first + count):
        v = (pix * np.uint64(2654435761) + np.uint64(s) * np.uint64(40503) + np.arange(3, dtype=np.uint64))
        total += (v % np.uint64(1 << 34))          # up to 64 in fixed point (2^34 / 2^28)
    return total


@pytest.mark.parametrize("samples,world", [(16, 2), (7, 3), (1, 4), (65536, 8)])
def test_sample_shards_cover_the_frame_once(samples, world):
    shards = [sample_shard(samples, world, r) for r in range(world)]
    covered = [s for first, count in shards for s in range(first, first + count)]
    assert covered == list(range(samples))
    counts = [c for _, c in shards]
    assert max(counts) - min(counts) <= 1
    with pytest.raises(ValueError):
        sample_shard(samples, world, world)


def test_resolve_matches_the_device_formula_in_numpy_and_torch():
    import torch

    sums = np.array([[[0, 1, 268435456], [2 ** 40 + 12345, 2 ** 53 + 1, 2 ** 62]]], np.uint64)
    img = resolve_sums(sums, 16)
    scale = 1.0 / (ACCUM_SCALE * 16.0)
    expect = (sums.astype(np.float64) * scale).astype(np.float32)
    assert img.dtype == np.float32 and img.shape == (1, 2, 4)
    assert np.array_equal(img[..., :3], expect) and np.all(img[..., 3] == 0)
    timg = resolve_sums(torch.from_numpy(sums.astype(np.int64)), 16)
    assert np.array_equal(timg.numpy(), img)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, h, w, spp, out_dir):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        first, count = sample_shard(spp, world, rank)
        local = torch.from_numpy(_synthetic_sums(h, w, first, count).astype(np.int64))
        dist.all_reduce(local, op=dist.ReduceOp.SUM)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), resolve_sums(local, spp).numpy())
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_equal_one_process(tmp_path):
    import torch.multiprocessing as mp

    h, w, spp, world = 6, 5, 9, 2
    mp.spawn(_worker, args=(world, _free_port(), h, w, spp, str(tmp_path)), nprocs=world, join=True)
    single = resolve_sums(_synthetic_sums(h, w, 0, spp), spp)
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert got.tobytes() == single.tobytes()

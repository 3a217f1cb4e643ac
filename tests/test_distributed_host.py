"""Sample sharding of one frame across ranks, on CPU: the shard partition,
the exact resolve of fixed-point sums, the accumulator's overflow bound, a
world-size-2 gloo all-reduce of per-rank sums, and ``render_frame_sharded``
itself run by two gloo ranks with a stand-in renderer; both must equal the
single-process result bit for bit.  The per-sample values are synthetic
integers keyed by (pixel, sample), standing in for the device's fixed-point
path samples."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from ordinarylight_b200.distributed import (ACCUM_SCALE, MAX_FRAME_SAMPLES, SAMPLE_CLAMP, render_frame_sharded,
                                            resolve_sums, sample_shard)

HEADER = os.path.join(os.path.dirname(__file__), "..", "ordinarylight_b200", "csrc", "olc_common.cuh")


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


def _header_constant(name):
    import re

    text = open(HEADER).read()
    return float(re.search(rf"#define {name} ([0-9.e]+)u?f?", text).group(1))


def test_the_accumulator_cannot_wrap_for_the_largest_frame():
    """Each channel of a sample is clamped before it is scaled by 2^28; the
    largest frame (65,536 samples, however it is split into shards) must
    keep a pixel's sum below 2^63, the limit of the signed 64-bit tensors
    the all-reduce adds (and a fortiori of the device's unsigned words)."""
    clamp, scale = _header_constant("OLC_SAMPLE_CLAMP"), _header_constant("OLC_ACCUM_SCALE")
    frame = _header_constant("OLC_MAX_FRAME_SAMPLES")
    assert (clamp, scale, frame) == (SAMPLE_CLAMP, ACCUM_SCALE, MAX_FRAME_SAMPLES)
    per_sample = int(np.float32(clamp) * np.float32(scale))     # float32 product, rounded like __float2ull_rn
    assert per_sample * int(frame) < 2 ** 63
    # the worst case resolves without wrapping and gives the clamp back
    worst = np.full((1, 1, 3), per_sample * int(frame), np.uint64)
    assert resolve_sums(worst.astype(np.int64), int(frame))[0, 0, 0] == np.float32(clamp)


class _StandInRenderer:
    """Fills a job's sums like the device would for samples
    [first_sample, first_sample + samples) of each pixel."""

    device = "cpu"

    class config:
        samples_per_pixel = 9

    def render_batch(self, requests, outs, sums):
        import torch

        (req,), (dst,) = requests, sums
        h, w = dst.shape[:2]
        dst.copy_(torch.from_numpy(_synthetic_sums(h, w, req.first_sample, req.samples).astype(np.int64)))
        return outs


def _sharded_worker(rank, world, port, h, w, spp, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        image = render_frame_sharded(_StandInRenderer(), None, None, w, h, samples=spp, frame_index=3)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), image.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("spp", [9, 1])
def test_render_frame_sharded_on_two_gloo_ranks_equals_one_process(tmp_path, spp):
    """The function a user calls, across two processes: each rank renders its
    sample shard (one rank gets none when spp is 1), the sums are all-reduced
    and resolved; every rank's image equals the single-process frame."""
    import torch.multiprocessing as mp

    h, w, world = 4, 7, 2
    mp.spawn(_sharded_worker, args=(world, _free_port(), h, w, spp, str(tmp_path)), nprocs=world, join=True)
    single = render_frame_sharded(_StandInRenderer(), None, None, w, h, samples=spp).numpy()
    assert single.tobytes() == resolve_sums(_synthetic_sums(h, w, 0, spp), spp).tobytes()
    for r in range(world):
        assert np.load(tmp_path / f"rank{r}.npy").tobytes() == single.tobytes()


def test_render_frame_sharded_rejects_frames_beyond_the_exact_range():
    with pytest.raises(ValueError):
        render_frame_sharded(_StandInRenderer(), None, None, 4, 4, samples=MAX_FRAME_SAMPLES + 1)

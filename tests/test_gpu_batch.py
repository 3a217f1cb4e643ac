"""Batched and served forms against the plain path.

A job's random numbers are keyed by (pixel, sample, bounce, seed +
frame_index) and its samples accumulate in order-independent fixed point, so
the batched form (many jobs and scenes per wavefront chunk), the served form
(continuous batching across steps) and every chunk size must reproduce the
plain ``render_frame`` image bit for bit.  Plain frames here use no temporal
history (each plain render runs on a fresh sequence), as the batched and
served jobs do.
"""

from __future__ import annotations

import numpy as np
import pytest

from ordinarylight_b200 import CudaWavefrontRenderer, scenes
from ordinarylight_b200.renderers.cuda import RenderRequest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene_set():
    room, room_cam = scenes.box_room()
    spheres, spheres_cam = scenes.instanced_spheres(seed=7, instances=6, segments=24, bands=13, emitters=32,
                                                    extent=5.0)
    spheres2, spheres2_cam = scenes.instanced_spheres(seed=9, instances=3, segments=16, bands=9, emitters=0,
                                                      extent=4.0)
    return [(room, room_cam), (spheres, spheres_cam), (spheres2, spheres2_cam)]


def _requests(scene_set):
    (room, rc), (sph, sc), (sph2, s2c) = scene_set
    return [
        RenderRequest(room, rc, 64, 48, samples=4, frame_index=0, max_bounces=4),
        RenderRequest(sph, sc, 96, 64, samples=2, frame_index=3, max_bounces=8),
        RenderRequest(sph2, s2c, 40, 40, samples=1, frame_index=1, max_bounces=4),
        RenderRequest(room, rc, 32, 32, samples=8, frame_index=5, max_bounces=2),
        RenderRequest(sph, sc, 128, 72, samples=1, frame_index=0, max_bounces=3),
    ]


def _plain(request, **cfg):
    """Plain per-request image on a fresh renderer (no temporal history)."""
    with CudaWavefrontRenderer(max_bounces=request.max_bounces, seed=1, **cfg) as r:
        return r.render_frame(request.scene, request.camera, request.width, request.height,
                              samples=request.samples, frame_index=request.frame_index)


@pytest.mark.parametrize("restir", [False, True])
def test_batch_equals_plain_bit_for_bit(native_library, cuda_device, scene_set, restir):
    requests = _requests(scene_set)
    with CudaWavefrontRenderer(seed=1, restir=restir) as r:
        images = r.render_batch(requests)
        t = r.last_timings
        assert t["traversal_errors"] == 0 and t["queue_overflow"] == 0
        assert t["camera_rays"] == sum(q.width * q.height * q.samples for q in requests)
        again = r.render_batch(requests)   # replayed from the captured graph
    for request, image, image2 in zip(requests, images, again):
        plain = _plain(request, restir=restir)
        assert image.shape == plain.shape
        assert image.tobytes() == plain.tobytes()
        assert image2.tobytes() == image.tobytes()


def test_a_medium_scene_in_the_chunk_keeps_the_other_images(native_library, cuda_device, scene_set):
    """Chunks whose scenes have no participating medium run the shading
    kernel built without the medium code; a chunk that also holds a job over
    a scene with a medium runs the full kernel for all of its jobs.  The
    medium-free jobs must come out bit for bit as their plain renders do
    (which ran the medium-free kernel), and the medium job as its own."""
    terrain, terrain_cam = scenes.terrain(size=64, volume_size=16)
    requests = _requests(scene_set)[:3] + [RenderRequest(terrain, terrain_cam, 48, 32, samples=2, frame_index=2,
                                                         max_bounces=4)]
    with CudaWavefrontRenderer(seed=1) as r:
        images = r.render_batch(requests)
        assert r.last_timings["chunks"] == 1   # one chunk: every job is shaded by the full kernel
    for request, image in zip(requests, images):
        assert image.tobytes() == _plain(request).tobytes()


@pytest.mark.parametrize("chunk_paths", [4096, 20000])
def test_batch_chunking_does_not_change_images(native_library, cuda_device, scene_set, chunk_paths):
    requests = _requests(scene_set)
    with CudaWavefrontRenderer(seed=1, restir=True) as r:
        base = r.render_batch(requests)
        r.reconfigure(chunk_paths=chunk_paths, block_size=128, trace_block=64, stack_depth=16, sort_rays=True)
        chunked = r.render_batch(requests)
        assert r.last_timings["chunks"] > 1
    for a, b in zip(base, chunked):
        assert a.tobytes() == b.tobytes()


def test_served_result_is_the_same_alone_and_in_the_mix(native_library, cuda_device, scene_set):
    requests = _requests(scene_set)
    target = requests[1]
    with CudaWavefrontRenderer(seed=1, restir=True, chunk_paths=16384) as r:
        ticket = r.submit(target)
        alone = None
        for _ in range(1000):
            done = r.serve_step()
            if done:
                assert [t for t, _ in done] == [ticket]
                alone = done[0][1]
                break
        assert alone is not None
        # the same request among others; more arrive between steps
        tickets = {r.submit(q): k for k, q in enumerate(requests[:3])}
        results = {}
        late = False
        for _ in range(1000):
            for t, image in r.serve_step():
                results[tickets[t]] = image
            if not late:
                tickets[r.submit(requests[3])] = 3
                tickets[r.submit(requests[4])] = 4
                late = True
            if len(results) == len(requests):
                break
        assert r.queued_tickets() == []
    assert results[1].tobytes() == alone.tobytes()
    for k, request in enumerate(requests):
        assert results[k].tobytes() == _plain(request, restir=True).tobytes()


def test_served_small_request_finishes_before_a_large_one(native_library, cuda_device, scene_set):
    (room, rc), (sph, sc), _ = scene_set
    big = RenderRequest(sph, sc, 256, 256, samples=8, max_bounces=4)
    small = RenderRequest(room, rc, 16, 16, samples=1, max_bounces=4)
    with CudaWavefrontRenderer(seed=1, chunk_paths=65536) as r:
        t_big = r.submit(big)
        t_small = r.submit(small)
        first = []
        while not first:
            first = r.serve_step()
        assert [t for t, _ in first] == [t_small]
        assert t_big in r.queued_tickets()
        rest = []
        while r.queued_tickets():
            rest += r.serve_step()
        assert [t for t, _ in rest] == [t_big]
        assert rest[0][1].tobytes() == _plain(big).tobytes()
        assert first[0][1].tobytes() == _plain(small).tobytes()


def test_cancel_and_scene_pool_reuse(native_library, cuda_device, scene_set):
    (room, rc), (sph, sc), (sph2, s2c) = scene_set
    with CudaWavefrontRenderer(seed=1, max_bounces=4) as r:
        plain = r.render_frame(room, rc, 48, 48, samples=2)
        ticket = r.submit(RenderRequest(sph, sc, 64, 64, samples=2))
        r.cancel(ticket)
        assert r.queued_tickets() == []
        with pytest.raises(ValueError):
            r.cancel(ticket)
        h1 = r.resident_scene(sph)
        h2 = r.resident_scene(sph2)
        assert h1 != h2 and r.resident_scene(sph) == h1
        before = r.pool_info()
        r.release_scene(sph)
        r.resident_scene(sph)        # re-added into the freed ranges
        after = r.pool_info()
        assert after["pool_bytes"] == before["pool_bytes"]
        assert after["resident_scenes"] == before["resident_scenes"]
        # the default scene renders the same bits with other scenes resident
        assert r.render_frame(room, rc, 48, 48, samples=2).tobytes() == plain.tobytes()
        img = r.render_batch([RenderRequest(sph, sc, 64, 64, samples=2)])[0]
        assert img.tobytes() == _plain(RenderRequest(sph, sc, 64, 64, samples=2, max_bounces=4)).tobytes()


def test_render_server_stream(native_library, cuda_device, scene_set):
    from ordinarylight_b200.serving import RenderServer, poisson_arrivals, run_stream

    requests = _requests(scene_set) * 2
    with CudaWavefrontRenderer(seed=1, restir=True) as r:
        server = RenderServer(r, budget_bytes=8 * 10**9).start()
        futures = run_stream(server, requests, poisson_arrivals(200.0, len(requests), seed=3))
        server.stop()
        summary = server.stats.summary()
    assert summary["completed"] == len(requests) and summary["rejected"] == 0
    assert np.isfinite(summary["p50_ms"]) and summary["p99_ms"] >= summary["p50_ms"]
    for request, f in zip(requests, futures):
        assert f.result().tobytes() == _plain(request, restir=True).tobytes()


def test_render_server_rejects_what_cannot_fit(native_library, cuda_device, scene_set):
    from ordinarylight_b200.serving import AdmissionRejected, RenderServer

    (room, rc), _, _ = scene_set
    with CudaWavefrontRenderer(seed=1) as r:
        server = RenderServer(r, budget_bytes=1024).start()
        f = server.submit(RenderRequest(room, rc, 64, 64))
        with pytest.raises(AdmissionRejected):
            f.result(timeout=60)
        server.stop()
        assert server.stats.rejected == 1


def test_autotuner_keeps_images(native_library, cuda_device, scene_set):
    from ordinarylight_b200.autotune import autotune

    requests = _requests(scene_set)[:3]
    with CudaWavefrontRenderer(seed=1) as r:
        base = r.render_batch(requests)
        result = autotune(r, requests, chunks=(8192, 1 << 20), blocks=((128, 128), (256, 64)), stacks=(16, 24),
                          sorts=(False, True), repeats=1, use_cache=False)
        assert len(result.trials) >= 4
        assert r.config.chunk_paths == result.chunk_paths and r.config.stack_depth == result.stack_depth
        tuned = r.render_batch(requests)
    for a, b in zip(base, tuned):
        assert a.tobytes() == b.tobytes()


@pytest.mark.parametrize("restir", [False, True])
def test_sample_shards_add_up_to_the_frame_bit_for_bit(native_library, cuda_device, scene_set, restir):
    import torch

    from ordinarylight_b200.distributed import render_frame_sharded, resolve_sums, sample_shard

    (room, rc), (sph, sc), _ = scene_set
    for scene, camera in ((room, rc), (sph, sc)):
        w, h, spp = 48, 40, 7
        full = _plain(RenderRequest(scene, camera, w, h, samples=spp, frame_index=2, max_bounces=5), restir=restir)
        with CudaWavefrontRenderer(seed=1, max_bounces=5, restir=restir) as r:
            # three shards as three ranks would render them, summed on the device
            total = torch.zeros((h, w, 3), dtype=torch.int64, device="cuda")
            for rank in range(3):
                first, count = sample_shard(spp, 3, rank)
                sums = torch.empty((h, w, 3), dtype=torch.int64, device="cuda")
                img = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
                r.render_batch([RenderRequest(scene, camera, w, h, samples=count, frame_index=2,
                                              first_sample=first)], outs=[img], sums=[sums])
                total += sums
            assert resolve_sums(total, spp).cpu().numpy().tobytes() == full.tobytes()
            # host sums, and the one-rank path of render_frame_sharded
            host = np.empty((h, w, 3), np.uint64)
            r.render_batch([RenderRequest(scene, camera, w, h, samples=spp, frame_index=2)], sums=[host])
            assert resolve_sums(host, spp).tobytes() == full.tobytes()
            single = render_frame_sharded(r, scene, camera, w, h, samples=spp, frame_index=2)
            assert single.cpu().numpy().tobytes() == full.tobytes()

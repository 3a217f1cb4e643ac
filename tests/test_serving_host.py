"""Host logic of the served and batched forms, on CPU: admission by an HBM
budget, LRU eviction of idle scenes, rejection, failure handling, latency
statistics and the autotuner's coordinate descent.  The device is replaced
by a fake renderer with the same methods, so nothing here needs a GPU."""

from __future__ import annotations

import time

import numpy as np
import pytest

from ordinarylight_b200.renderers.cuda import RenderRequest
from ordinarylight_b200.serving import AdmissionRejected, RenderServer, poisson_arrivals, run_stream


class FakeScene:
    def __init__(self, name, nbytes):
        self.name = name
        self.nbytes = nbytes
        self.revision = 0


class FakeRenderer:
    """Mimics CudaWavefrontRenderer's pool / serving surface.  Each step
    advances every queued job by `paths_per_step` paths of a shared chunk."""

    def __init__(self, paths_per_step=10_000, fail_on_step=None):
        self.resident = {}          # id -> (scene, handle)
        self.order = []             # LRU order of ids
        self.jobs = {}              # ticket -> [request, remaining paths]
        self.next_ticket = 1
        self.paths_per_step = paths_per_step
        self.fail_on_step = fail_on_step
        self.steps = 0
        self.uploads = 0
        self.evictions = []
        self.last_timings = {}

    # pool
    def resident_scene(self, scene):
        if id(scene) not in self.resident:
            self.resident[id(scene)] = (scene, len(self.resident) + 1)
            self.uploads += 1
        else:
            self.order.remove(id(scene))
        self.order.append(id(scene))
        return self.resident[id(scene)][1]

    def release_scene(self, scene):
        del self.resident[id(scene)]
        self.order.remove(id(scene))
        self.evictions.append(scene.name)

    def resident_scenes(self):
        return [(self.resident[i][0], self.resident[i][1], self.resident[i][0].nbytes) for i in self.order]

    def job_bytes(self, request):
        return request.width * request.height * 40

    def pool_info(self):
        used = sum(self.job_bytes(j[0]) for j in self.jobs.values())
        return {"scene_bytes": sum(s.nbytes for s, _ in self.resident.values()), "wavefront_bytes": 1000,
                "pixel_bytes_used": used, "pool_bytes": 0}

    # serving
    def submit(self, request):
        t = self.next_ticket
        self.next_ticket += 1
        self.jobs[t] = [request, request.width * request.height * (request.samples or 1)]
        return t

    def serve_step(self):
        self.steps += 1
        if self.fail_on_step == self.steps:
            victims = list(self.jobs)[:1]
            for t in victims:
                del self.jobs[t]
            raise RuntimeError("simulated device failure")
        budget = self.paths_per_step
        done = []
        # shortest remaining work first, as the native planner orders a step
        for t in sorted(self.jobs, key=lambda k: self.jobs[k][1]):
            take = min(budget, self.jobs[t][1])
            self.jobs[t][1] -= take
            budget -= take
            if self.jobs[t][1] == 0:
                req = self.jobs.pop(t)[0]
                done.append((t, np.full((req.height, req.width, 4), float(t), np.float32)))
            if budget == 0:
                break
        self.last_timings = {"rays": self.paths_per_step - budget, "gpu_ms": 1.0}
        time.sleep(0.001)
        return done

    def queued_tickets(self):
        return list(self.jobs)


def _req(scene, w=16, h=16, spp=1):
    return RenderRequest(scene, None, w, h, samples=spp)


def test_requests_complete_and_report_latency():
    r = FakeRenderer()
    a, b = FakeScene("a", 100), FakeScene("b", 200)
    reqs = [_req(a, 32, 32, 4), _req(b, 8, 8), _req(a, 16, 16, 2)] * 3
    server = RenderServer(r, budget_bytes=10**9).start()
    futures = run_stream(server, reqs, poisson_arrivals(500.0, len(reqs), seed=1))
    server.stop()
    s = server.stats.summary()
    assert s["completed"] == len(reqs) and s["rejected"] == 0 and s["failed"] == 0
    assert 0 < s["p50_ms"] <= s["p99_ms"]
    assert all(f.result().shape == (q.height, q.width, 4) for f, q in zip(futures, reqs))
    assert r.uploads == 2            # each scene uploaded once, then resident


def test_small_requests_finish_inside_big_ones():
    """Continuous batching: a small request submitted after a big one does
    not wait for the big one to finish."""
    r = FakeRenderer(paths_per_step=5_000)
    s = FakeScene("s", 10)
    server = RenderServer(r, budget_bytes=10**9).start()
    big = server.submit(_req(s, 256, 256, 4))      # ~52 steps
    time.sleep(0.01)
    small = server.submit(_req(s, 8, 8, 1))
    small.result(timeout=10)
    assert not big.done()
    big.result(timeout=30)
    server.stop()


def test_budget_evicts_idle_scenes_lru_first():
    r = FakeRenderer()
    scenes = [FakeScene(f"s{k}", 1000) for k in range(4)]
    # room for the wavefront (1000), two scenes and one small request
    server = RenderServer(r, budget_bytes=1000 + 2 * 1000 + 16 * 16 * 40).start()
    for sc in scenes:
        server.submit(_req(sc)).result(timeout=10)
    server.stop()
    assert r.evictions[:2] == ["s0", "s1"]
    assert len(r.resident) == 2


def test_request_that_cannot_fit_is_rejected_and_others_continue():
    r = FakeRenderer()
    sc = FakeScene("s", 10)
    server = RenderServer(r, budget_bytes=1000 + 10 + 64 * 64 * 40).start()
    too_big = server.submit(_req(sc, 512, 512))
    with pytest.raises(AdmissionRejected):
        too_big.result(timeout=10)
    ok = server.submit(_req(sc, 64, 64))
    assert ok.result(timeout=10).shape == (64, 64, 4)
    server.stop()
    assert server.stats.rejected == 1 and server.stats.completed == 1


def test_requests_wait_for_budget_instead_of_failing():
    r = FakeRenderer(paths_per_step=1_000)
    sc = FakeScene("s", 10)
    # two 64x64 requests do not fit together: the second waits for the first
    server = RenderServer(r, budget_bytes=1000 + 10 + 64 * 64 * 40 + 100).start()
    f1 = server.submit(_req(sc, 64, 64))
    f2 = server.submit(_req(sc, 64, 64))
    assert f1.result(timeout=10) is not None and f2.result(timeout=10) is not None
    server.stop()
    assert server.stats.queue_ms[1] > server.stats.queue_ms[0]


def test_step_failure_fails_only_the_dropped_jobs():
    r = FakeRenderer(paths_per_step=100, fail_on_step=2)
    sc = FakeScene("s", 10)
    server = RenderServer(r, budget_bytes=10**9).start()
    f1 = server.submit(_req(sc, 16, 16))
    f2 = server.submit(_req(sc, 16, 16))
    with pytest.raises(RuntimeError):
        f1.result(timeout=10)
    assert f2.result(timeout=10).shape == (16, 16, 4)
    server.stop()
    assert server.stats.failed == 1


def test_serial_server_is_fifo_one_at_a_time():
    from ordinarylight_b200.serving import SerialServer

    class Serial(FakeRenderer):
        def __init__(self):
            super().__init__()
            self.order = []

        def render_batch(self, requests, outs=None):
            assert len(requests) == 1
            q = requests[0]
            self.order.append(q.width)
            self.last_timings = {"rays": q.width * q.height, "gpu_ms": 0.5}
            time.sleep(0.002)
            return [np.zeros((q.height, q.width, 4), np.float32)]

    r = Serial()
    sc = FakeScene("s", 1)
    server = SerialServer(r).start()
    futures = [server.submit(_req(sc, w, 4)) for w in (64, 8, 32)]
    for f in futures:
        f.result(timeout=10)
    server.stop()
    assert r.order == [64, 8, 32]
    assert server.stats.completed == 3 and server.stats.latencies_ms[2] > server.stats.latencies_ms[0]


def test_submit_after_stop_raises():
    server = RenderServer(FakeRenderer(), budget_bytes=10**9).start()
    server.stop()
    with pytest.raises(RuntimeError):
        server.submit(_req(FakeScene("s", 1)))


def test_poisson_arrivals_rate():
    t = poisson_arrivals(100.0, 20000, seed=0)
    assert np.all(np.diff(t) > 0)
    assert abs(len(t) / t[-1] - 100.0) < 3.0


class FakeTunable:
    """Batch time is a known function of the knobs; the autotuner must find
    the minimum along each coordinate."""

    def __init__(self):
        from ordinarylight_b200.renderers.cuda import CudaRendererConfig
        self.config = CudaRendererConfig()
        self.calls = 0

    def reconfigure(self, **changes):
        from dataclasses import replace
        self.config = replace(self.config, **changes)

    def render_batch(self, requests, outs=None):
        c = self.config
        cost = abs(np.log2(max(c.chunk_paths, 1)) - 18) + abs(c.block_size - 128) / 64 + abs(c.stack_depth - 24) / 8
        time.sleep(0.002 + 0.002 * cost)
        self.calls += 1
        return outs


def test_autotuner_coordinate_descent():
    from ordinarylight_b200.autotune import autotune

    r = FakeTunable()
    reqs = [_req(FakeScene("s", 1))]
    result = autotune(r, reqs, repeats=1, use_cache=False)
    assert (result.chunk_paths, result.block_size, result.stack_depth) == (1 << 18, 128, 24)
    assert r.config.chunk_paths == 1 << 18
    assert len(result.trials) <= 1 + 4 + 4 + 3 + 2
    again = autotune(r, reqs, repeats=1)          # cached: no new trials
    calls = r.calls
    assert autotune(r, reqs, repeats=1) is again and r.calls == calls


# ---------------------------------------------------------------------------
# multi-GPU placement (ReplicaRouter): one RenderServer per device
# ---------------------------------------------------------------------------
class _StubServer:
    """Accepts submissions and leaves their futures pending until `finish`."""

    def __init__(self):
        self.requests = []
        self.futures = []

    def submit(self, request):
        from concurrent.futures import Future

        f = Future()
        self.requests.append(request)
        self.futures.append(f)
        return f

    def finish(self):
        for f in self.futures:
            if not f.done():
                f.set_result(None)


def test_router_keeps_a_scenes_requests_on_one_replica_and_spreads_new_scenes():
    from ordinarylight_b200.serving import ReplicaRouter

    a, b, c = FakeScene("a", 10), FakeScene("b", 10), FakeScene("c", 10)
    servers = [_StubServer(), _StubServer()]
    router = ReplicaRouter(servers, spill_factor=2.0, spill_paths=0)
    for scene in (a, b, a, b, a):
        router.submit(_req(scene, 8, 8))
    assert router.placements == [0, 1, 0, 1, 0]
    assert [r.scene for r in servers[0].requests] == [a, a, a]
    router.submit(_req(c, 8, 8))          # new scene: the less loaded replica
    assert router.placements[-1] == 1


def test_router_replicates_a_hot_scene_when_its_holder_is_overloaded():
    from ordinarylight_b200.serving import ReplicaRouter

    hot = FakeScene("hot", 10)
    servers = [_StubServer(), _StubServer()]
    router = ReplicaRouter(servers, spill_factor=1.0, spill_paths=0)
    placed = [router.place(_req(hot, 16, 16)) for _ in range(4)]
    # holder 0 takes requests while it is within one request's work of the
    # least-loaded replica, then the scene spills onto replica 1 as well,
    # and the less loaded of its two holders takes the next one
    assert placed == [0, 0, 1, 1]
    assert router.outstanding() == [512, 512]


def test_router_releases_work_on_completion_and_is_deterministic():
    from ordinarylight_b200.serving import ReplicaRouter

    scenes = [FakeScene(str(k), 10) for k in range(5)]
    runs = []
    for _ in range(2):
        servers = [_StubServer() for _ in range(3)]
        router = ReplicaRouter(servers, spill_factor=1.5, spill_paths=64)
        rng = np.random.default_rng(3)
        for k in range(40):
            router.submit(_req(scenes[int(rng.integers(5))], 8, 8, int(rng.integers(1, 4))))
        runs.append(list(router.placements))
        for s in servers:
            s.finish()
        assert router.outstanding() == [0, 0, 0]
        assert sum(len(s.requests) for s in servers) == 40
    assert runs[0] == runs[1]
    assert len(set(runs[0])) == 3          # every replica gets work


def test_router_over_two_servers_returns_every_image():
    """Two RenderServers stand in for two GPUs (each with its own fake
    renderer): every request completes with its own replica's image and the
    merged statistics count each once."""
    from ordinarylight_b200.serving import ReplicaRouter

    scenes = [FakeScene(str(k), 100) for k in range(4)]
    servers = [RenderServer(FakeRenderer(paths_per_step=5000), budget_bytes=10**9) for _ in range(2)]
    with ReplicaRouter(servers) as router:
        futures = [router.submit(_req(scenes[k % 4], 16, 8, 2)) for k in range(12)]
        images = [f.result(timeout=10) for f in futures]
    assert all(img.shape == (8, 16, 4) for img in images)
    s = router.summary()
    assert s["completed"] == 12 and s["replicas"] == 2 and sum(s["per_replica_requests"]) == 12
    assert min(s["per_replica_requests"]) > 0

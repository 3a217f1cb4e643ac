"""Served rendering: a request loop with continuous batching on one device,
and a router that places requests across one such loop per GPU.

The reference renders submissions one at a time on a renderer-owned worker
(``Renderer.render_async`` -> ``_render_serialized``,
ordinarylight/renderer/_core.py:614-651 and :709-717).  :class:`RenderServer`
keeps that API shape (``submit`` returns a future; results are the same
images) but runs a device loop that

* keeps scene hierarchies and materials resident in the device scene pool
  (a scene is uploaded once and reused by every request that names it);
* admits queued requests by an HBM budget: a request enters the wavefront
  only while the resident scenes, the fixed wavefront buffers and the pixels
  of every admitted request fit the budget; least-recently-used scenes that
  no admitted request needs are evicted to make room, and a request that
  could never fit is rejected;
* merges admitted requests into the shared ray queues chunk by chunk
  (``CudaWavefrontRenderer.serve_step``): requests that arrive while a chunk
  is on the GPU join the next chunk, and small requests finish inside the
  chunks of large ones instead of waiting behind them;
* reports p50/p99 latency (submission to completion), throughput and the
  rejected-request count.

Each image is bit-identical to ``render_frame`` of the same request on a
fresh sequence: the random numbers are keyed by (pixel, sample, bounce,
seed + frame_index) and accumulation is order independent, so neither the
chunking nor the mix changes a result.
"""

from __future__ import annotations

from collections import deque
from concurrent.futures import Future
from dataclasses import dataclass, field
import threading
import time

import numpy as np

from .renderers.cuda import CudaWavefrontRenderer, RenderRequest

DEFAULT_BUDGET_BYTES = 150 * 10**9


class AdmissionRejected(RuntimeError):
    """A request whose scene and pixels alone exceed the HBM budget."""


@dataclass
class _Pending:
    request: RenderRequest
    future: Future
    submitted: float
    admitted: float = 0.0
    ticket: int = 0


@dataclass
class ServerStatistics:
    completed: int = 0
    rejected: int = 0
    failed: int = 0
    rays: int = 0
    gpu_ms: float = 0.0
    steps: int = 0
    latencies_ms: list = field(default_factory=list)
    queue_ms: list = field(default_factory=list)
    started: float = 0.0
    finished: float = 0.0

    def percentile(self, q: float) -> float:
        if not self.latencies_ms:
            return float("nan")
        return float(np.percentile(np.asarray(self.latencies_ms), q))

    def summary(self) -> dict:
        wall = max(self.finished - self.started, 1e-9)
        return {
            "completed": self.completed,
            "rejected": self.rejected,
            "failed": self.failed,
            "p50_ms": self.percentile(50),
            "p99_ms": self.percentile(99),
            "mean_ms": float(np.mean(self.latencies_ms)) if self.latencies_ms else float("nan"),
            "throughput_req_s": self.completed / wall,
            "mrays_per_s": self.rays / wall / 1e6,
            "gpu_mrays_per_s": self.rays / (self.gpu_ms * 1e3) if self.gpu_ms > 0 else 0.0,
            "steps": self.steps,
            "wall_s": wall,
        }


class RenderServer:
    """Continuous-batching request loop over a :class:`CudaWavefrontRenderer`.

    ``submit`` is thread-safe and returns a ``concurrent.futures.Future``
    whose result is the (height, width, 4) float32 image.  All device work
    happens on the server's own thread.
    """

    def __init__(self, renderer: CudaWavefrontRenderer, *, budget_bytes: int = DEFAULT_BUDGET_BYTES):
        self.renderer = renderer
        self.budget_bytes = int(budget_bytes)
        self._draining = True
        self._lock = threading.Condition()
        self._waiting: deque[_Pending] = deque()
        self._admitted: dict[int, _Pending] = {}
        self._running = False
        self._thread = None
        self.stats = ServerStatistics()
        self._error = None

    # -- client side ----------------------------------------------------------------
    def submit(self, request: RenderRequest) -> Future:
        future: Future = Future()
        with self._lock:
            if not self._running:
                raise RuntimeError("server is not running")
            self._waiting.append(_Pending(request, future, time.perf_counter()))
            self._lock.notify()
        return future

    def start(self):
        with self._lock:
            if self._running:
                return self
            self._running = True
            self.stats = ServerStatistics(started=time.perf_counter())
        self._thread = threading.Thread(target=self._loop, name="olc-render-server", daemon=True)
        self._thread.start()
        return self

    def stop(self, *, drain: bool = True, timeout: float | None = None):
        """Stop the loop; with ``drain`` it first finishes every request."""
        with self._lock:
            self._draining = drain
            self._running = False
            self._lock.notify()
        if self._thread is not None:
            self._thread.join(timeout)
        self.stats.finished = time.perf_counter()
        if self._error is not None:
            raise self._error

    def __enter__(self):
        return self.start()

    def __exit__(self, *_exc):
        self.stop()

    # -- admission ------------------------------------------------------------------
    def _used_bytes(self) -> int:
        """Bytes charged to the budget: resident scenes, the wavefront buffers
        and the pixels of admitted requests (the pool's growth slack beyond
        the scenes' own ranges is not charged)."""
        info = self.renderer.pool_info()
        return info["scene_bytes"] + info["wavefront_bytes"] + info["pixel_bytes_used"]

    def _admit(self, pending: _Pending) -> bool:
        """Admit one waiting request if the budget allows, evicting resident
        scenes that no admitted request needs (least recently used first).
        Returns False to keep it waiting; raises AdmissionRejected when it
        cannot fit even with nothing else admitted."""
        r = self.renderer
        scene = pending.request.scene
        r.resident_scene(scene)   # uploads on first use; its bytes count from here
        need = r.job_bytes(pending.request)
        used = self._used_bytes()
        if used + need > self.budget_bytes:
            busy = {id(p.request.scene) for p in self._admitted.values()} | {id(scene)}
            for resident, _handle, nbytes in r.resident_scenes():
                if used + need <= self.budget_bytes:
                    break
                if id(resident) in busy:
                    continue
                r.release_scene(resident)
                used -= nbytes
            if used + need > self.budget_bytes:
                if not self._admitted:
                    r.release_scene(scene)
                    raise AdmissionRejected(
                        f"request needs {need} bytes with {used} in use; the budget is {self.budget_bytes}")
                return False
        pending.ticket = r.submit(pending.request)
        pending.admitted = time.perf_counter()
        self._admitted[pending.ticket] = pending
        return True

    # -- device loop ----------------------------------------------------------------
    def _loop(self):
        try:
            while True:
                with self._lock:
                    while self._running and not self._waiting and not self._admitted:
                        self._lock.wait()
                    if not self._running and not self._admitted and (not self._waiting or not self._draining):
                        break
                    waiting = list(self._waiting)
                    self._waiting.clear()
                # admission in arrival order; what does not fit waits
                keep = deque()
                for k, pending in enumerate(waiting):
                    if keep:
                        keep.append(pending)
                        continue
                    try:
                        if not self._admit(pending):
                            keep.append(pending)
                    except AdmissionRejected as exc:
                        self.stats.rejected += 1
                        pending.future.set_exception(exc)
                    except Exception as exc:  # invalid request
                        self.stats.failed += 1
                        pending.future.set_exception(exc)
                if keep:
                    with self._lock:
                        self._waiting.extendleft(reversed(keep))
                if not self._admitted:
                    continue
                try:
                    done = self.renderer.serve_step()
                except Exception as exc:
                    queued = set(self.renderer.queued_tickets())
                    for ticket in [t for t in self._admitted if t not in queued]:
                        self.stats.failed += 1
                        self._admitted.pop(ticket).future.set_exception(exc)
                    continue
                t = self.renderer.last_timings
                self.stats.rays += t.get("rays", 0)
                self.stats.gpu_ms += t.get("gpu_ms", 0.0)
                self.stats.steps += 1
                now = time.perf_counter()
                for ticket, image in done:
                    pending = self._admitted.pop(ticket)
                    self.stats.completed += 1
                    self.stats.latencies_ms.append((now - pending.submitted) * 1e3)
                    self.stats.queue_ms.append((pending.admitted - pending.submitted) * 1e3)
                    pending.future.set_result(image)
        except BaseException as exc:  # keep the failure for stop()
            self._error = exc
            with self._lock:
                for pending in list(self._waiting) + list(self._admitted.values()):
                    if not pending.future.done():
                        pending.future.set_exception(RuntimeError(f"render server failed: {exc}"))
                self._waiting.clear()
                self._admitted.clear()
                self._running = False


class SerialServer(RenderServer):
    """The plain path under the same request stream: one request at a time in
    arrival order, the way the reference serialises ``render_async``
    submissions on one worker (ordinarylight/renderer/_core.py:614-651,
    :709-717), with every scene resident.  Same ``submit``/``start``/``stop``
    and statistics as :class:`RenderServer`, for latency comparisons."""

    def _loop(self):
        try:
            while True:
                with self._lock:
                    while self._running and not self._waiting:
                        self._lock.wait()
                    if not self._waiting and (not self._running or not self._draining):
                        break
                    if not self._running and not self._draining:
                        break
                    pending = self._waiting.popleft()
                pending.admitted = time.perf_counter()
                try:
                    image = self.renderer.render_batch([pending.request])[0]
                except Exception as exc:
                    self.stats.failed += 1
                    pending.future.set_exception(exc)
                    continue
                t = self.renderer.last_timings
                self.stats.rays += t.get("rays", 0)
                self.stats.gpu_ms += t.get("gpu_ms", 0.0)
                self.stats.steps += 1
                now = time.perf_counter()
                self.stats.completed += 1
                self.stats.latencies_ms.append((now - pending.submitted) * 1e3)
                self.stats.queue_ms.append((pending.admitted - pending.submitted) * 1e3)
                pending.future.set_result(image)
        except BaseException as exc:
            self._error = exc
            with self._lock:
                for pending in list(self._waiting):
                    if not pending.future.done():
                        pending.future.set_exception(RuntimeError(f"render server failed: {exc}"))
                self._waiting.clear()
                self._running = False


class ReplicaRouter:
    """Serving across GPUs: one :class:`RenderServer` per device (each with
    its own renderer, scene pool and budget) behind one ``submit``.  The
    path shards by request, so the GPUs exchange nothing; the router only
    places requests.

    Placement is by scene affinity and outstanding work (the paths, width x
    height x samples, of a replica's unfinished requests):

    * a request whose scene is already placed goes to the replica that holds
      it, unless that replica's outstanding work exceeds the least-loaded
      replica's by more than ``spill_factor`` x the request's own work (plus
      ``spill_paths``); the request then goes to the least-loaded replica and
      the scene becomes resident there too (a hot scene is replicated);
    * a request with a new scene goes to the least-loaded replica (ties: the
      one holding the fewest scenes, then the lowest index).

    Each result is the image that replica's renderer produces, which is the
    image any device produces: random numbers are keyed by (pixel, sample,
    bounce, seed + frame_index), not by device or batch.
    """

    def __init__(self, servers, *, spill_factor: float = 2.0, spill_paths: int = 1 << 22):
        if not servers:
            raise ValueError("a router needs at least one server")
        self.servers = list(servers)
        self.spill_factor = float(spill_factor)
        self.spill_paths = int(spill_paths)
        self._lock = threading.Lock()
        self._outstanding = [0] * len(self.servers)
        self._holders: dict[int, list[int]] = {}    # scene key -> replicas it was placed on
        self._scenes_on = [0] * len(self.servers)
        self.placements: list[int] = []             # replica of every submitted request, in order

    @staticmethod
    def _scene_key(scene) -> int:
        return id(scene)

    @staticmethod
    def _work(request: RenderRequest) -> int:
        spp = request.samples if request.samples is not None else 1
        return int(request.width) * int(request.height) * int(spp)

    def place(self, request: RenderRequest) -> int:
        """The replica `request` goes to (and books its work there)."""
        work = self._work(request)
        key = self._scene_key(request.scene)
        with self._lock:
            least = min(range(len(self.servers)), key=lambda i: (self._outstanding[i], self._scenes_on[i], i))
            holders = self._holders.get(key, [])
            choice = least
            if holders:
                best = min(holders, key=lambda i: (self._outstanding[i], i))
                if self._outstanding[best] <= self._outstanding[least] + self.spill_factor * work + self.spill_paths:
                    choice = best
            if choice not in holders:
                self._holders.setdefault(key, []).append(choice)
                self._scenes_on[choice] += 1
            self._outstanding[choice] += work
            self.placements.append(choice)
            return choice

    def _done(self, replica: int, work: int):
        with self._lock:
            self._outstanding[replica] -= work

    def submit(self, request: RenderRequest) -> Future:
        replica = self.place(request)
        work = self._work(request)
        try:
            future = self.servers[replica].submit(request)
        except BaseException:
            self._done(replica, work)
            raise
        future.add_done_callback(lambda _f: self._done(replica, work))
        return future

    def outstanding(self) -> list:
        with self._lock:
            return list(self._outstanding)

    def start(self):
        for server in self.servers:
            server.start()
        return self

    def stop(self, *, drain: bool = True, timeout: float | None = None):
        errors = []
        for server in self.servers:
            try:
                server.stop(drain=drain, timeout=timeout)
            except BaseException as exc:   # stop every replica, then report
                errors.append(exc)
        if errors:
            raise errors[0]

    def __enter__(self):
        return self.start()

    def __exit__(self, *_exc):
        self.stop()

    def summary(self) -> dict:
        """Statistics over all replicas: latency percentiles of every
        completed request, throughput over the longest replica wall time."""
        lat, rays, gpu_ms, completed, rejected, failed, steps = [], 0, 0.0, 0, 0, 0, 0
        started = min(s.stats.started for s in self.servers)
        finished = max(s.stats.finished for s in self.servers)
        for s in self.servers:
            st = s.stats
            lat += st.latencies_ms
            rays += st.rays
            gpu_ms += st.gpu_ms
            completed += st.completed
            rejected += st.rejected
            failed += st.failed
            steps += st.steps
        wall = max(finished - started, 1e-9)
        return {"replicas": len(self.servers), "completed": completed, "rejected": rejected, "failed": failed,
                "p50_ms": float(np.percentile(lat, 50)) if lat else float("nan"),
                "p99_ms": float(np.percentile(lat, 99)) if lat else float("nan"),
                "throughput_req_s": completed / wall, "mrays_per_s": rays / wall / 1e6, "steps": steps,
                "per_replica_requests": [self.placements.count(i) for i in range(len(self.servers))]}


def poisson_arrivals(rate_per_s: float, count: int, seed: int = 0) -> np.ndarray:
    """Arrival times (seconds from 0) of a Poisson stream."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / float(rate_per_s), size=int(count)))


def run_stream(server: RenderServer, requests, arrivals) -> list:
    """Submit ``requests`` at their ``arrivals`` (seconds, real time) and
    wait for all of them; returns the futures in request order."""
    futures = []
    t0 = time.perf_counter()
    for request, at in zip(requests, arrivals):
        delay = t0 + float(at) - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        futures.append(server.submit(request))
    for f in futures:
        try:
            f.result()
        except Exception:
            pass
    return futures


__all__ = ["AdmissionRejected", "RenderServer", "ReplicaRouter", "SerialServer", "ServerStatistics", "poisson_arrivals",
           "run_stream", "DEFAULT_BUDGET_BYTES"]

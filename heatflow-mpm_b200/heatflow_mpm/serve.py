"""Serving air scenarios: continuous batching of independent scenes on one GPU.

Requests (``AirScenario`` with a horizon in substeps) arrive over time.  The server keeps every admitted scene's
fields and CG state resident on the device and advances all of them together, one batched substep per loop turn
(one launch per stage for the whole batch).  A request waiting in the queue is admitted as soon as a slot and its HBM
share are free, and a scene leaves the batch the moment its horizon is reached.  The batch plan (scene table, work
tables, workspace) is rebuilt only when the membership changes.

The GPU is never waited for between substeps: substeps are enqueued on the compute stream up to ``depth`` ahead of
the GPU; admitted scenes are built (statics on the device, initial temperature) and new plans uploaded on a side
stream while the queued substeps run, and the compute stream waits for that side stream only before the first
substep that uses them.  A finished scene's result fields and state block are copied to pinned host memory behind its
last substep; the request completes when that copy has landed.  Every ``status_every`` substeps the active scenes'
state blocks are copied back the same way, and a scene whose solver reports a failure (non-finite residual, maxiter,
barrier timeout) leaves the batch at once as a failed request.  Plans and scenes that queued substeps may still use
are released only after the compute stream has passed them.

Reported: aggregate scene-substeps/s (and 96^3-equivalent substeps/s, weighting each by n^3 / 96^3), the latency
of every request (arrival -> result on the host; p50/p99), the completed fraction and the ages of the requests still
unfinished when the trace window closes, and the GPU time of every batched substep (p50/p99).  Each scene's result
is bit-identical to running it alone (the kernels' reductions depend only on the scene).
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .batch import AirScenario, make_scene, upload_bytes
from .scene import ScenePlan


@dataclass
class Request:
    scenario: AirScenario
    arrival: float                      # seconds after the start of the trace
    rid: int = 0
    admitted: float | None = None
    done_at: float | None = None
    substeps_done: int = 0
    scene: object = None
    result: dict = field(default_factory=dict)


def poisson_trace(rate=20.0, duration=60.0, seed=0, edges=(48, 64, 96, 128), horizon=(200, 2000), power=(100, 800),
                  fan=(0, 3), sphere_prob=0.5, sphere_radius=(0.02, 0.06)):
    """The served workload: Poisson arrivals at `rate` per second over `duration` seconds; each request draws its grid
    edge, horizon (substeps), heater power, fan speed and, with probability sphere_prob, a static solid sphere."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        n = int(rng.choice(edges))
        sc = AirScenario(n=n, power=float(rng.uniform(*power)), fan=float(rng.uniform(*fan)),
                         horizon=int(rng.integers(horizon[0], horizon[1] + 1)), seed=int(rng.integers(1 << 30)),
                         sphere_radius=float(rng.uniform(*sphere_radius)) if rng.uniform() < sphere_prob else 0.0)
        out.append(Request(sc, t, rid=len(out)))
    return out


_FAILED = _lib.HF_SCENE_NONFINITE | _lib.HF_SCENE_HEAT_MAXITER | _lib.HF_SCENE_PRESSURE_MAXITER | \
    _lib.HF_SCENE_BARRIER_TIMEOUT


class AirServer:
    def __init__(self, device="cuda:0", dt=2e-3, hbm_budget=150e9, max_slots=256, persistent_blocks=0, group_cells=0,
                 lanes=0, keep_results=False, result_fields=("T",), setup="device", depth=2, status_every=10):
        self.device = torch.device(device)
        self.dt = dt
        self.budget = float(hbm_budget)
        self.max_slots = max_slots
        self.persistent_blocks = persistent_blocks
        self.group_cells = group_cells
        self.lanes = lanes
        self.keep_results = keep_results
        self.result_fields = ("T", "u", "v", "w") if keep_results else tuple(result_fields)
        self.setup = setup               # scene statics built on the device ("device") or on the host ("host")
        self.depth = max(1, int(depth))  # batched substeps enqueued ahead of the GPU
        self.status_every = int(status_every)
        self.admit_ms: list[float] = []  # host time of building each admitted scene (statics, upload, face fractions)
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        self.queue = collections.deque()
        self.active: list[Request] = []
        self.finished: list[Request] = []
        self.failed: list[Request] = []
        self.retiring = []               # (request, completion handle, host buffers) of result copies in flight
        self.checks = []                 # (requests, completion handle, host buffer) of status checks in flight
        self.inflight = collections.deque()   # (start, end) CUDA events of enqueued batched substeps not yet timed
        self.released = collections.deque()   # (event, objects) kept alive until the compute stream has passed event
        self.plan = None
        self.used = 0.0
        self.substep_ms: list[float] = []
        self.scene_substeps = 0
        self.weighted_substeps = 0.0
        self.plan_builds = 0
        self.steps = 0
        self._side = None

    # ------------------------------------------------------------------------------------------------ streams
    def _side_stream(self):
        if self._side is None:
            self._side = torch.cuda.Stream(self.device)
        return self._side

    def _release_later(self, *objs):
        """Keep objects (plans, scenes) alive until the compute stream has run everything enqueued so far."""
        if self.device.type != "cuda":
            return
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.device))
        self.released.append((ev, objs))

    # ------------------------------------------------------------------------------------------------ admission
    def submit(self, req: Request):
        self.queue.append(req)

    def _build_scene(self, scenario):
        """One admitted scene, built on the side stream: statics on the device, face fractions and conductivity."""
        if self.device.type != "cuda":
            scene = make_scene(scenario, self.device, setup=self.setup)
            ScenePlan([scene], self.device).prepare_statics()
            return scene
        with torch.cuda.stream(self._side_stream()):
            scene = make_scene(scenario, self.device, setup=self.setup)
            # the new scene's static obstacle fields, face fractions and conductivity, prepared on its own
            ScenePlan([scene], self.device).prepare_statics()
        return scene

    def _admit(self, now):
        changed = False
        while self.queue and len(self.active) < self.max_slots:
            req = self.queue[0]
            need = req.scenario.device_bytes()
            if self.used + need > self.budget:
                break
            self.queue.popleft()
            t0 = time.perf_counter()
            req.scene = self._build_scene(req.scenario)
            self.h2d_bytes += upload_bytes(req.scenario, self.setup)
            self.admit_ms.append(1e3 * (time.perf_counter() - t0))
            req.admitted = now
            self.used += need
            self.active.append(req)
            changed = True
        return changed

    # ------------------------------------------------------------------------------------------------ retirement
    def _copy_back(self, req, slot):
        """Enqueue, behind the scene's last substep, the copies of its result fields (current buffers, chosen on the
        device) and state block into pinned host memory.  Returns (handle, host buffers)."""
        import ctypes as C
        sc = req.scene
        stream = torch.cuda.current_stream(self.device)
        host = {}
        which = {"T": 0, "u": 1, "v": 2, "w": 3}
        for nm in self.result_fields:
            shape = tuple(getattr(sc, nm)[0].shape)
            dev = torch.empty(shape, dtype=torch.float32, device=self.device)
            _lib.check(self.plan.L.hf_current_field(C.byref(self.plan.plan), slot, which[nm], dev.data_ptr(),
                                                    C.c_void_p(stream.cuda_stream)), "hf_current_field")
            host[nm] = torch.empty(shape, dtype=torch.float32).pin_memory()
            host[nm].copy_(dev, non_blocking=True)
            self._release_later(dev)
        host["state"] = torch.empty(sc.state.numel(), dtype=torch.uint8).pin_memory()
        host["state"].copy_(sc.state, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(stream)
        return ev, host

    def _retire(self, now):
        """Scenes at their horizon, or failed, leave the batch: their results are copied back asynchronously."""
        keep, changed = [], False
        for slot, req in enumerate(self.active):
            if req.substeps_done >= req.scenario.horizon or req.result.get("failed"):
                handle, host = self._copy_back(req, slot)
                self.retiring.append((req, handle, host))
                self.used -= req.scenario.device_bytes()
                changed = True
            else:
                keep.append(req)
        self.active = keep
        self._collect(now)
        return changed

    def _done(self, handle):
        return handle.query()

    def _collect(self, now, wait=False):
        """Requests whose result copies have landed complete now (failed when their solver status says so)."""
        still = []
        for req, handle, host in self.retiring:
            if wait:
                handle.synchronize()
            if not self._done(handle):
                still.append((req, handle, host))
                continue
            req.done_at = now
            st = _lib.SceneState.from_buffer_copy(host["state"].numpy().tobytes()) if "state" in host else None
            for nm in self.result_fields:
                req.result[nm] = host[nm].numpy()
                self.d2h_bytes += req.result[nm].nbytes
            if self.keep_results and st is not None:
                req.result["state"] = st
            req.scene = None
            if st is not None and (st.status & _FAILED):
                req.result["failed"] = True
                req.result["status"] = int(st.status)
                self.failed.append(req)
            else:
                self.finished.append(req)
        self.retiring = still

    def _check_status(self):
        """Copy every active scene's state block back (asynchronously) to find failed solves early."""
        if not self.active:
            return
        reqs = list(self.active)
        nbytes = reqs[0].scene.state.numel()
        host = torch.empty((len(reqs), nbytes), dtype=torch.uint8).pin_memory()
        for i, r in enumerate(reqs):
            host[i].copy_(r.scene.state, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(self.device))
        self.checks.append((reqs, ev, host))

    def _poll(self):
        """Timings of finished substeps, landed status checks, released plans and scenes (never blocks)."""
        while self.inflight and self._done(self.inflight[0][1]):
            a, b = self.inflight.popleft()
            self.substep_ms.append(a.elapsed_time(b))
        keep = []
        for reqs, ev, host in self.checks:
            if not self._done(ev):
                keep.append((reqs, ev, host))
                continue
            for i, r in enumerate(reqs):
                st = _lib.SceneState.from_buffer_copy(host[i].numpy().tobytes())
                if st.status & _FAILED and r.scene is not None:
                    r.result["failed"] = True
        self.checks = keep
        while self.released and self._done(self.released[0][0]):
            self.released.popleft()

    # ------------------------------------------------------------------------------------------------ stepping
    def _rebuild(self):
        """A plan over the active scenes, built and uploaded on the side stream; the compute stream waits for it (and
        for the statics of newly admitted scenes) before its next substep.  The old plan is released once the compute
        stream has passed it."""
        if self.plan is not None:
            self._release_later(self.plan)
        if self.active:
            side = self._side_stream() if self.device.type == "cuda" else None
            if side is not None:
                with torch.cuda.stream(side):
                    self.plan = ScenePlan([r.scene for r in self.active], self.device,
                                          persistent_blocks=self.persistent_blocks, group_cells=self.group_cells,
                                          lanes=self.lanes)
                torch.cuda.current_stream(self.device).wait_stream(side)
            else:
                self.plan = ScenePlan([r.scene for r in self.active], self.device,
                                      persistent_blocks=self.persistent_blocks, group_cells=self.group_cells,
                                      lanes=self.lanes)
        else:
            self.plan = None
        self.plan_builds += 1

    def _throttle(self):
        """At most `depth` batched substeps in flight: wait for the oldest one beyond that."""
        while len(self.inflight) >= self.depth:
            self.inflight[0][1].synchronize()
            self._poll()

    def step(self, now):
        """Admit, enqueue one substep of every active scene, retire the finished and failed ones."""
        self._poll()
        changed = self._admit(now)
        if changed or (self.plan is None and self.active):
            self._rebuild()
        self._collect(now)
        if not self.active:
            return
        self._throttle()
        self._advance()
        self.steps += 1
        for r in self.active:
            r.substeps_done += 1
            self.scene_substeps += 1
            self.weighted_substeps += r.scenario.n ** 3 / 96.0 ** 3
        if self.status_every > 0 and self.steps % self.status_every == 0:
            self._check_status()
        if self._retire(now):
            self._rebuild()

    def _advance(self):
        """Enqueue one batched substep of every active scene between two CUDA events on the compute stream."""
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        self.plan.substep(self.dt)
        b.record()
        self.inflight.append((a, b))

    def serve(self, trace, time_limit=None, clock=time.perf_counter):
        """Replay `trace` against the wall clock: requests enter the queue at their arrival times.  Stops when every
        request is done or after time_limit seconds (the substeps already enqueued then finish and are counted).
        Returns the summary dict."""
        pending = collections.deque(sorted(trace, key=lambda r: r.arrival))
        self.submitted = len(pending)
        t0 = clock()
        while pending or self.queue or self.active or self.retiring:
            now = clock() - t0
            if time_limit is not None and now > time_limit:
                break
            while pending and pending[0].arrival <= now:
                self.submit(pending.popleft())
            if not self.active and not self.queue:
                self._collect(now)
                if self.retiring and not pending:
                    self._collect(clock() - t0, wait=True)
                elif pending:
                    time.sleep(max(0.0, min(pending[0].arrival - now, 0.01)))
                continue
            self.step(now)
        if self.device.type == "cuda":
            torch.cuda.synchronize(self.device)
        self.elapsed = clock() - t0
        self._poll()
        self._collect(self.elapsed, wait=True)
        self.unfinished_ages = [self.elapsed - r.arrival for r in list(pending) + list(self.queue) + self.active]
        self.unfinished = len(self.unfinished_ages)
        return self.summary()

    def summary(self):
        lat = [r.done_at - r.arrival for r in self.finished]
        q = lambda a, p: float(np.percentile(a, p)) if len(a) else None
        el = getattr(self, "elapsed", None) or 1e-9
        ages = getattr(self, "unfinished_ages", [])
        total = getattr(self, "submitted", None) or (len(self.finished) + len(self.failed) + len(ages)) or 1
        return {"requests_done": len(self.finished), "requests_failed": len(self.failed),
                "requests_unfinished": getattr(self, "unfinished", 0),
                "completed_fraction": len(self.finished) / total,
                "scene_substeps": self.scene_substeps, "substeps_per_s": self.scene_substeps / el,
                "substeps96_per_s": self.weighted_substeps / el,
                "request_latency_p50_s": q(lat, 50), "request_latency_p99_s": q(lat, 99),
                "unfinished_age_p50_s": q(ages, 50), "unfinished_age_p99_s": q(ages, 99),
                "substep_latency_p50_ms": q(self.substep_ms, 50), "substep_latency_p99_ms": q(self.substep_ms, 99),
                "batched_substeps": self.steps, "plan_builds": self.plan_builds, "elapsed_s": el,
                "setup": self.setup, "admit_ms_p50": q(self.admit_ms, 50), "admit_ms_p99": q(self.admit_ms, 99)}

"""Serving air scenarios: continuous batching of independent scenes on one GPU.

Requests (``AirScenario`` with a horizon in substeps) arrive over time.  The server keeps every admitted scene's
fields and CG state resident on the device and advances all of them together, one batched substep per loop turn
(one launch per stage for the whole batch).  A request waiting in the queue is admitted as soon as a slot and its HBM
share are free -- between two substeps, while the others keep running -- and a scene leaves the batch the moment its
horizon is reached.  The batch plan (scene table, work tables, workspace) is rebuilt only when the membership changes.

Reported: aggregate scene-substeps/s (and 96^3-equivalent substeps/s, weighting each by n^3 / 96^3), the latency
of every request (arrival -> last substep done; p50/p99), and the latency of every batched substep (p50/p99).
Each scene's result is bit-identical to running it alone (the kernels' reductions depend only on the scene).
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np
import torch

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


class AirServer:
    def __init__(self, device="cuda:0", dt=2e-3, hbm_budget=150e9, max_slots=256, persistent_blocks=0, group_cells=0,
                 lanes=0, keep_results=False, result_fields=("T",), setup="device"):
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
        self.admit_ms: list[float] = []  # host time of building each admitted scene (statics, upload, face fractions)
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        self.queue = collections.deque()
        self.active: list[Request] = []
        self.finished: list[Request] = []
        self.plan = None
        self.used = 0.0
        self.substep_ms: list[float] = []
        self.scene_substeps = 0
        self.weighted_substeps = 0.0
        self.plan_builds = 0

    # ------------------------------------------------------------------------------------------------ admission
    def submit(self, req: Request):
        self.queue.append(req)

    def _admit(self, now):
        changed = False
        while self.queue and len(self.active) < self.max_slots:
            req = self.queue[0]
            need = req.scenario.device_bytes()
            if self.used + need > self.budget:
                break
            self.queue.popleft()
            t0 = time.perf_counter()
            req.scene = make_scene(req.scenario, self.device, setup=self.setup)
            self.h2d_bytes += upload_bytes(req.scenario, self.setup)
            # the new scene's static obstacle fields, face fractions and conductivity, prepared on its own
            ScenePlan([req.scene], self.device).prepare_statics()
            self.admit_ms.append(1e3 * (time.perf_counter() - t0))
            req.admitted = now
            self.used += need
            self.active.append(req)
            changed = True
        return changed

    def _retire(self, now):
        keep, changed = [], False
        for req in self.active:
            if req.substeps_done >= req.scenario.horizon:
                req.done_at = now
                for nm in self.result_fields:
                    req.result[nm] = req.scene.current(nm).cpu().numpy()
                    self.d2h_bytes += req.result[nm].nbytes
                if self.keep_results:
                    req.result["state"] = req.scene.read_state()
                self.used -= req.scenario.device_bytes()
                req.scene = None
                self.finished.append(req)
                changed = True
            else:
                keep.append(req)
        self.active = keep
        return changed

    # ------------------------------------------------------------------------------------------------ stepping
    def _rebuild(self):
        self.plan = ScenePlan([r.scene for r in self.active], self.device, persistent_blocks=self.persistent_blocks,
                              group_cells=self.group_cells, lanes=self.lanes) if self.active else None
        self.plan_builds += 1

    def step(self, now):
        """Admit, advance every active scene one substep, retire the finished ones.  Returns the substep's ms."""
        changed = self._admit(now)
        if changed or (self.plan is None and self.active):
            self._rebuild()
        if not self.active:
            return 0.0
        ms = self._advance()
        self.substep_ms.append(ms)
        for r in self.active:
            r.substeps_done += 1
            self.scene_substeps += 1
            self.weighted_substeps += r.scenario.n ** 3 / 96.0 ** 3
        if self._retire(now):
            self._rebuild()
        return ms

    def _advance(self):
        """One batched substep of every active scene, timed with CUDA events on the current stream."""
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        self.plan.substep(self.dt)
        b.record()
        b.synchronize()
        return a.elapsed_time(b)

    def serve(self, trace, time_limit=None, clock=time.perf_counter):
        """Replay `trace` against the wall clock: requests enter the queue at their arrival times.  Stops when every
        request is done or after time_limit seconds.  Returns the summary dict."""
        pending = collections.deque(sorted(trace, key=lambda r: r.arrival))
        t0 = clock()
        while pending or self.queue or self.active:
            now = clock() - t0
            if time_limit is not None and now > time_limit:
                break
            while pending and pending[0].arrival <= now:
                self.submit(pending.popleft())
            if not self.active and not self.queue:
                if pending:
                    time.sleep(max(0.0, min(pending[0].arrival - now, 0.01)))
                continue
            self.step(now)
        self.elapsed = clock() - t0
        self.unfinished = len(pending) + len(self.queue) + len(self.active)
        return self.summary()

    def summary(self):
        lat = [r.done_at - r.arrival for r in self.finished]
        q = lambda a, p: float(np.percentile(a, p)) if len(a) else None
        el = getattr(self, "elapsed", None) or 1e-9
        return {"requests_done": len(self.finished), "requests_unfinished": getattr(self, "unfinished", 0),
                "scene_substeps": self.scene_substeps, "substeps_per_s": self.scene_substeps / el,
                "substeps96_per_s": self.weighted_substeps / el,
                "request_latency_p50_s": q(lat, 50), "request_latency_p99_s": q(lat, 99),
                "substep_latency_p50_ms": q(self.substep_ms, 50), "substep_latency_p99_ms": q(self.substep_ms, 99),
                "batched_substeps": len(self.substep_ms), "plan_builds": self.plan_builds, "elapsed_s": el,
                "setup": self.setup, "admit_ms_p50": q(self.admit_ms, 50), "admit_ms_p99": q(self.admit_ms, 99)}

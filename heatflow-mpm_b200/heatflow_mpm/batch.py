"""Batched air scenes: many independent scenes of uneven size advanced together, one launch per stage per substep.

``AirScenario`` describes one air-only scene (grid edge, heater, fan, optional static solid sphere).  ``AirBatch``
builds the device scenes, one plan over all of them (scene table + chunk and tile tables: the kernels walk the tables,
so scenes of different n share every launch), optionally captures K substeps in one CUDA graph, and reports per-scene
state.  The CG solves of a batch run in the streaming persistent kernels with per-scene convergence masking: a scene
that has converged stops iterating while the others continue.  Results are bit-identical to each scene run alone.

``autotune`` picks the launch shape of the CG solves for a batch -- blocks of the streaming kernel, the cells of one
scene group (a group's CG vectors should stay in L2) and the lanes that solve groups side by side -- by timing
candidates on the device; every candidate computes the same bits, so tuning never changes results.  Choices are cached
per GPU and batch signature in a JSON file.
"""
from __future__ import annotations

import functools
import json
import os
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .heater import FAN, K_SOLID, BoxHeater, Heater, face_masks, fan_momentum, source_rate
from .scene import DeviceScene, SceneSpec, ScenePlan
from .solver import wall_fixed
from .voxelize import device_statics, sphere_bounds


@dataclass
class AirScenario:
    """One air-only scene: a cube of edge L with n cells per edge, a heater, and optionally a static solid sphere."""
    n: int
    L: float = 0.48
    power: float = 400.0
    t_cap: float = 120.0
    fan: float = 0.0
    heater_x: float | None = None        # box heater at this x [m]; None: the reference trough heater
    sphere_radius: float = 0.0           # static solid sphere at the box centre, on the floor (0: none)
    sphere_t: float = 20.0               # the sphere's cells are held at this temperature
    t_amb: float = 25.0
    cg_tol: float = 1e-4
    heat_tol: float = 1e-6
    horizon: int = 0                     # substeps requested (serving)
    seed: int = 0
    noise: float = 0.01                  # seeded uniform +-noise K on the initial temperature
    tag: dict = field(default_factory=dict)

    @property
    def h(self):
        return self.L / self.n

    def heater(self):
        if self.heater_x is not None:
            return BoxHeater(x=self.heater_x, power=self.power, t_cap=self.t_cap, fan=self.fan)
        return Heater(power=self.power, t_cap=self.t_cap, fan=self.fan)

    def spec(self) -> SceneSpec:
        """The scene's SceneSpec: equal, array for array, to building it from heater.masks and wall_fixed directly
        (the geometry that does not depend on power or fan speed is cached per grid and heater placement)."""
        n, h = self.n, self.h
        g = _geometry(n, self.L, self.heater_x, self.fan > 0, self.t_amb)
        rate = source_rate(self.power, 1.2, g["n_source"], h)
        kf = list(g["k_faces"])
        mf = fan_momentum(g["touch_fan"], self.fan, g["facing"]) if self.fan > 0 else list(g["zero_faces"])
        solid, fixed, tfix = g["solid"], g["fixed"], g["tfix"]
        if self.sphere_radius > 0:
            # a cold solid sphere resting on the floor at the box centre: alpha_s = 1, K_SOLID and no momentum on its
            # faces, cells held at sphere_t
            R, c = self.sphere_radius, self.L / 2
            x = (np.arange(n) + 0.5) * h
            lo, hi, top = sphere_bounds(n, h, self.L, R)
            ball = np.zeros((n, n, n), bool)
            ball[lo:hi, lo:hi, :top] = ((x[lo:hi, None, None] - c) ** 2 + (x[None, lo:hi, None] - c) ** 2
                                        + (x[None, None, :top] - R) ** 2 <= R * R)
            solid = np.maximum(solid, ball.astype(np.float32))
            fixed = fixed | ball
            tfix = np.where(ball, np.float32(self.sphere_t), tfix).astype(np.float32)
            on_ball, _ = face_masks(ball, ball)
            for axis in range(3):
                kf[axis] = np.where(on_ball[axis], np.float32(K_SOLID), kf[axis]).astype(np.float32)
                mf[axis] = np.where(on_ball[axis], np.float32(0.0), mf[axis]).astype(np.float32)
        return SceneSpec(n=n, h=h, t_amb=self.t_amb, cg_tol=self.cg_tol, heat_tol=self.heat_tol, fixed=fixed, tfix=tfix,
                         source=g["source"], rate=rate, t_cap=self.t_cap, static_alpha=solid, static_k=kf, static_m=mf)

    def device_spec(self, device="cuda:0") -> SceneSpec:
        """spec() with the heater, walls and sphere voxelised on the device (voxelize.device_statics): the same
        arrays bit for bit, without building or uploading them on the host."""
        sphere = (self.sphere_radius, self.sphere_t, self.L) if self.sphere_radius > 0 else None
        st = device_statics(self.heater(), self.n, self.h, (self.L / 2, self.L / 2), 1.2, self.t_amb, sphere=sphere,
                            device=device)
        return SceneSpec(n=self.n, h=self.h, t_amb=self.t_amb, cg_tol=self.cg_tol, heat_tol=self.heat_tol, rate=st.rate,
                         t_cap=self.t_cap, statics=st)

    def initial_T(self):
        rng = np.random.default_rng(self.seed)
        return (self.t_amb + rng.uniform(-self.noise, self.noise, (self.n,) * 3)).astype(np.float32)

    def device_bytes(self) -> int:
        """HBM a resident scene of this size takes (fields, statics, CG vectors), for admission control."""
        n = self.n
        N, NF = n ** 3, (n + 1) * n * n
        return int(4 * (20 * N + 16 * NF) + N)


@functools.lru_cache(maxsize=64)
def _geometry(n, L, heater_x, fan_on, t_amb):
    """Heater cells, masks, static conduction faces and fixed cells of a grid: everything of a scenario's spec that
    depends only on the grid, the heater placement and whether the fan runs.  Arrays are read-only (shared)."""
    fan = 1.0 if fan_on else 0.0
    heater = BoxHeater(x=heater_x, fan=fan) if heater_x is not None else Heater(fan=fan)
    cells, solid, source, _, kf, _, geom = heater.masks(n, L / n, (L / 2, L / 2), 1.2)
    _, touch_fan = face_masks(solid, cells == FAN)
    fixed, tfix = wall_fixed(n, cells, heater.t_rod, t_amb)
    g = dict(solid=solid.astype(np.float32), source=source, n_source=int(source.sum()), k_faces=tuple(kf),
             touch_fan=tuple(touch_fan), facing=tuple(geom["facing"]), fixed=fixed, tfix=tfix.astype(np.float32),
             zero_faces=tuple(np.zeros(a.shape, np.float32) for a in kf))
    for v in g.values():
        for a in (v if isinstance(v, tuple) else (v,)):
            if isinstance(a, np.ndarray):
                a.setflags(write=False)
    return g


def make_scene(sc: AirScenario, device="cuda:0", setup="device") -> DeviceScene:
    """A resident scene of the scenario, its statics built on the device (setup="device") or on the host ("host")."""
    if setup not in ("device", "host"):
        raise ValueError("setup must be 'device' or 'host'")
    ds = DeviceScene(sc.device_spec(device) if setup == "device" else sc.spec(), device)
    ds.set_current("T", sc.initial_T())
    ds.apply_fixed_to_T()
    return ds


class AirBatch:
    """Scenes advanced together by one plan; see the module docstring."""

    def __init__(self, scenarios, device="cuda:0", persistent_blocks=0, scenes=None, group_cells=0, lanes=0):
        self.device = torch.device(device)
        self.scenarios = list(scenarios)
        self.scenes = scenes if scenes is not None else [make_scene(s, device) for s in self.scenarios]
        self.plan = ScenePlan(self.scenes, device, persistent_blocks=persistent_blocks, group_cells=group_cells,
                              lanes=lanes)
        self.plan.prepare_statics()
        self.graph = None
        self._graph_key = None

    def substep(self, dt):
        self.plan.substep(dt)

    def run(self, dt, steps, use_graph=True, graph_steps=10):
        """Advance every scene exactly `steps` substeps; with use_graph, graph_steps substeps are replayed per graph
        launch (the substep that warms up a new capture counts as one of them)."""
        done = 0
        if use_graph and steps > graph_steps:
            done += self.capture(dt, graph_steps)
            while steps - done >= graph_steps:
                self.graph.replay()
                done += graph_steps
        while done < steps:
            self.plan.substep(dt)
            done += 1

    def capture(self, dt, k):
        """Record k substeps of the whole batch as one CUDA graph in self.graph (the kernels read the buffer parity on
        the device, so the graph replays correctly however many times it runs).  Building a new graph first runs one
        real substep outside the capture (module loading, kernel attributes); returns how many substeps that
        advanced the batch (1, or 0 when the graph for (dt, k) exists already)."""
        key = (float(dt), int(k))
        if self.graph is not None and self._graph_key == key:
            return 0
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.plan.substep(dt)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            for _ in range(k):
                self.plan.substep(dt)
        self.graph, self._graph_key = g, key
        return 1

    def states(self):
        return [sc.read_state() for sc in self.scenes]

    def snapshot(self):
        """Device copies of what the next substep starts from in every scene: the current T, u, v, w and the pressure
        (the CG warm start).  Air-only scenes carry no other state from one substep to the next."""
        return [dict({nm: sc.current(nm).clone() for nm in ("T", "u", "v", "w")}, p=sc.p.clone()) for sc in self.scenes]

    def restore(self, snap):
        """Put a snapshot back: the substeps that follow compute the same bits as they did after it was taken."""
        for sc, st in zip(self.scenes, snap):
            for nm in ("T", "u", "v", "w"):
                sc.current(nm).copy_(st[nm])
            sc.p.copy_(st["p"])


# ---------------------------------------------------------------------------------------------------- autotuner
_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_cache.json")


def _signature(scenes):
    hist = {}
    for sc in scenes:
        hist[sc.n] = hist.get(sc.n, 0) + 1
    return ",".join(f"{n}x{c}" for n, c in sorted(hist.items()))


def autotune(batch: AirBatch, dt=2e-3, reps=3, candidates=None, cache=True):
    """Time launch-shape candidates (persistent_blocks, group_cells, lanes) of the CG solves on this batch and keep
    the fastest.  Every candidate times the same `reps` substeps from the batch's current state (restored before each
    one, after a warm-up substep), and the batch is left as it was found.  Returns (the chosen triple,
    {"blocks/cells/lanes": ms per substep})."""
    sms = torch.cuda.get_device_properties(batch.device).multi_processor_count
    name = torch.cuda.get_device_name(batch.device)
    key = f"{name}|{_signature(batch.scenes)}"
    plan = batch.plan
    table = {}
    if cache and os.path.exists(_CACHE):
        try:
            table = json.load(open(_CACHE))
        except ValueError:
            table = {}
    if cache and key in table:
        best = tuple(int(v) for v in table[key]["choice"])
        plan.plan.persistent_blocks, plan.plan.group_cells, plan.lanes = best
        return best, table[key]["timings"]
    # group_cells: 0 = the library default (2.4 M cells), 1 = one scene per group, and sizes whose groups, times the
    # lanes solving them side by side, keep the CG vectors (~40 B per cell) inside the 126 MB L2
    candidates = candidates or [(b * sms, g, l) for (g, l) in ((1, 1), (1, 2), (0, 1), (0, 2), (1, 4), (0, 4), (0, 8),
                                                               (600_000, 4), (1_200_000, 2), (800_000, 3))
                                for b in (2, 4, 5)]
    timings = {}
    snap = batch.snapshot()
    for pb, gc, ln in candidates:
        plan.plan.persistent_blocks, plan.plan.group_cells, plan.lanes = pb, gc, ln
        batch.plan.substep(dt)                       # warm-up
        batch.restore(snap)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            batch.plan.substep(dt)
        b.record()
        torch.cuda.synchronize()
        timings[(pb, gc, ln)] = a.elapsed_time(b) / reps
        batch.restore(snap)
    del snap
    best = min(timings, key=timings.get)
    plan.plan.persistent_blocks, plan.plan.group_cells, plan.lanes = best
    out = {"/".join(str(v) for v in k): t for k, t in timings.items()}
    if cache:
        table[key] = {"choice": list(best), "timings": out}
        try:
            json.dump(table, open(_CACHE, "w"), indent=1)
        except OSError:
            pass
    return best, out


def shard_scenarios(scenarios, rank, world):
    """Scenes of this rank when `world` GPUs share a batch: whole scenes, largest first, each to the rank with the
    fewest cells so far (ties to the lowest rank).  Every rank computes the same assignment without communication."""
    load = [0] * world
    mine = []
    order = sorted(range(len(scenarios)), key=lambda i: (-scenarios[i].n, i))
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += scenarios[i].n ** 3
        if r == rank:
            mine.append(i)
    return [scenarios[i] for i in sorted(mine)]


def upload_bytes(sc: AirScenario, setup="device") -> int:
    """Host-to-device bytes of creating the scene: the initial T, plus (statics built on the host) fixed values, cell
    flags, static alpha and face weights."""
    n = sc.n
    N, NF = n ** 3, (n + 1) * n * n
    if setup == "device":
        return 4 * N
    return 4 * N + 4 * N + N + 4 * N + 2 * 3 * 4 * NF


def ensemble(count=64, seed=0, edges=(32, 48, 64, 96, 128), steps=200):
    """The batched-ensemble workload: `count` air-only scenes, edge drawn from `edges` with h = 0.48 m / edge, heater
    power U(100, 800) W, fan U(0, 3) m/s, box heater at x U(0.05, 0.2) m (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.choice(edges))
        out.append(AirScenario(n=n, power=float(rng.uniform(100, 800)), fan=float(rng.uniform(0, 3)),
                               heater_x=float(rng.uniform(0.05, 0.2)), horizon=steps, seed=int(rng.integers(1 << 30)),
                               tag={"index": i}))
    return out

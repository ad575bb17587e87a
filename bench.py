"""Benchmark: 96^3 air substeps/s of Heatflow-MPM's Eulerian air path on B200, plain and batched-served.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload plain|batched|served]

plain (default line) -- the default coupled 96^3 scene: h = 5 mm, trough heater 400 W capped at 120 C, fan 2 m/s, rods
300 C, room 25 C, a seeded ellipsoid of ~16k particles (semi-axes 4/3/5 cm, 2.5 mm jittered lattice) at 20 C, melt
law T_sol 28 / T_liq 34; pressure CG tol 1e-4 (maxiter 400), heat CG tol 1e-6 (maxiter 200); dt = 2 ms.  Newton (the
material solver) is not installed, so the particles keep their positions and velocities (frozen body); the air
substep still scatters them, rebuilds the obstacle fields and updates their temperatures every substep.  Both arms
start from the state after a deterministic spin-up of --spinup substeps, then W warm-up substeps, then K timed
substeps.  `value` = substeps/s with the state resident in HBM (CUDA events on the stream, barrier + synchronize on both
sides, max over ranks); `e2e` = the same through the public API with the particle state copied from pinned host memory
before and the grid temperature copied back after every substep.

batched -- 64 air-only scenes (edge drawn from {32,48,64,96,128}, h = 0.48 m / edge, box heater at x U(0.05,0.2) m,
power U(100,800) W, fan U(0,3) m/s; seeded), one launch per stage per substep for the whole batch, K substeps replayed
from a CUDA graph of --graph-steps substeps.  value = 96^3-equivalent substeps/s (cells x substeps / 96^3 / s).

served -- Poisson arrivals (--rate per s, default 20) of air scenarios (edge from {48,64,96,128}, horizon U(200,2000)
substeps, power U(100,800) W, fan U(0,3) m/s, with probability 1/2 a static solid sphere of radius U(2,6) cm held at
20 C), admitted against an HBM budget and continuously batched, for --serve-seconds of wall clock.  value = 96^3-
equivalent substeps/s while the GPU computes (sum of the batched substeps' CUDA-event times); e2e = the same work over
the wall-clock window (admission, scene upload, plan rebuilds, result download included); p50/p99 of request and
batched-substep latency.

The default line carries compact `batched` and `served` summaries (--no-extras drops them).  The CPU reference arm
(--impl reference) times the CPU port of the reference's algorithm (oracle/) on the host cores, plain workload.
Multi-GPU: plain runs one replica per GPU; batched and served shard whole scenes (requests) across GPUs, no collective
on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "heatflow-mpm_b200"))

import numpy as np  # noqa: E402

DT = 2.0e-3
METRIC = "96^3 air substeps/s (default coupled scene, plain path)"
METRIC_BATCHED = "96^3-equivalent air substeps/s (64-scene batched ensemble)"
METRIC_SERVED = "96^3-equivalent air substeps/s (served Poisson trace, continuous batching)"
PUBLISHED_SUBSTEPS_PER_S = 1000.0 / 7.0   # README.md:46 of the reference: ~7 ms per air substep (RTX 5080)
WORKLOAD = ("default coupled scene 96^3 (h=5 mm, 400 W cap 120 C, fan 2 m/s, ~16k-particle ellipsoid, frozen body), "
            "dt=2 ms, pressure tol 1e-4, heat tol 1e-6")
N96 = 96 ** 3
PARITY_STEPS = 20   # plain line: substeps of the timed region replayed on the CPU port for the parity figures


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed substeps (plain 1000, batched 200)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain", choices=["plain", "batched", "served"])
    ap.add_argument("--spinup", type=int, default=30, help="substeps from the initial scene before warm-up (both arms)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--ref-seconds", type=float, default=60.0, help="budget of the timed CPU reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="plain line without the batched/served summaries")
    ap.add_argument("--resident-tiles", type=int, default=0, help="plain: tiles per group of the resident CG (0: auto)")
    ap.add_argument("--no-graph", action="store_true", help="plain: time eager launches instead of one graph replay")
    ap.add_argument("--streaming", default="none", choices=["none", "heat", "both"],
                    help="plain: CG solves in the streaming kernel instead of the resident one")
    ap.add_argument("--persistent-blocks", type=int, default=0, help="plain: grid of the streaming CG kernel")
    ap.add_argument("--no-tma", action="store_true", help="plain: resident pressure CG without the TMA-staged stencil")
    ap.add_argument("--cg", default="single-reduction", choices=["classic", "single-reduction"],
                    help="plain: pressure solve by the classic Jacobi-PCG or its single-reduction form (one grid "
                         "barrier per iteration)")
    ap.add_argument("--scenes", type=int, default=64, help="batched: scenes in the ensemble")
    ap.add_argument("--graph-steps", type=int, default=10, help="batched: substeps per captured CUDA graph")
    ap.add_argument("--edges", default="32,48,64,96,128", help="batched: grid edges the ensemble draws from")
    ap.add_argument("--no-autotune", action="store_true", help="batched: default launch shape, no tuning")
    ap.add_argument("--launch", default=None, help="batched: fixed CG launch shape 'blocks,group_cells,lanes'")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="served: length of the trace window")
    ap.add_argument("--rate", type=float, default=20.0, help="served: mean arrivals per second")
    ap.add_argument("--hbm-budget", type=float, default=150e9, help="served: HBM admitted for scenes, bytes")
    ap.add_argument("--max-slots", type=int, default=64, help="served: most scenes in one batch")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def _reduce(x, op, dev, world):
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=op)
    return float(t.item())


def reduce_max(x, dev, world):
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX if world > 1 else None, dev, world)


def reduce_sum(x, dev, world):
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM if world > 1 else None, dev, world)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def load_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


# --------------------------------------------------------------------------------------------------- CPU side
def cpu_scene(seed=0):
    """The benchmark scene on the CPU port (oracle) -- no device work."""
    from heatflow_mpm.grid import GridConfig
    from heatflow_mpm.heater import Heater
    from heatflow_mpm.mpm import Material
    from heatflow_mpm.solver import build_spec, KAPPA_AIR
    from heatflow_mpm.synthetic import ellipsoid_particles
    from oracle import oracle as O
    parts = ellipsoid_particles(seed=seed)
    spec, _, _, _ = build_spec(parts, Material(t_sol=28.0, t_liq=34.0), Heater(power=400.0, t_cap=120.0, fan=2.0),
                               GridConfig(L=0.48, h=0.005, t_amb=25.0), 2.5e-3, 20.0, KAPPA_AIR)
    sc = O.scene_from_spec(spec, "f32", mean_mode=0, scatter_mode=0, particles=parts,
                           pvel=np.zeros_like(parts), ptemp=np.full(len(parts), 20.0, np.float32))
    return sc, spec


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def time_cpu_substeps(sc, budget_s, max_steps, min_steps=1):
    t0 = time.perf_counter()
    done = 0
    while done < max_steps and (done < min_steps or time.perf_counter() - t0 < budget_s):
        sc.substep(DT)
        done += 1
    return done, time.perf_counter() - t0


def cpu_scenarios_sample(scenarios, budget_s, per_scene=2):
    """CPU port on air scenarios, per_scene substeps each from their initial state, in order, until budget_s:
    returns (96^3-equivalent substeps/s, substeps done, scenes visited, seconds)."""
    from oracle import oracle as O
    O.set_threads(host_threads())
    cells, done, visited, el = 0, 0, 0, 0.0
    for sc in scenarios:
        if el > budget_s:
            break
        o = O.scene_from_spec(sc.spec(), "f32")
        o.set_state(T=np.where(sc.spec().fixed, sc.spec().tfix, sc.initial_T()).astype(np.float32))
        t0 = time.perf_counter()
        for _ in range(per_scene):
            o.substep(DT)
        el += time.perf_counter() - t0
        cells += per_scene * sc.n ** 3
        done += per_scene
        visited += 1
    return cells / N96 / el, done, visited, el


def plain_config(n, spinup):
    """`config` of the plain line, the same dict in both arms (what the workload is, not what a run measured)."""
    return {"workload": WORKLOAD, "n": n, "cells": n ** 3, "spinup": spinup, "dt": DT,
            "l2": "scene state ~170 MB > 126 MB L2 (inputs larger than L2); the CG working set (~35 MB) stays "
                  "L2-resident within a substep by design"}


def oracle_substeps(sc, steps, budget_s=None):
    """`steps` substeps of the CPU port (fewer once budget_s seconds have passed, at least one): returns (substeps
    done, seconds, pressure CG iterations, heat CG iterations)."""
    t0 = time.perf_counter()
    done, it_p, it_h = 0, 0, 0
    while done < steps and (done == 0 or budget_s is None or time.perf_counter() - t0 < budget_s):
        sc.substep(DT)
        st = sc.stats()
        it_p += int(st["grid_done"])
        it_h += int(st["heat_done"])
        done += 1
    return done, time.perf_counter() - t0, it_p, it_h


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    O.set_threads(host_threads())
    steps = args.steps if args.steps is not None else 1000
    sc, spec = cpu_scene()
    t0 = time.perf_counter()
    for _ in range(args.spinup + args.warmup):
        sc.substep(DT)
    t_setup = time.perf_counter() - t0
    done, el = time_cpu_substeps(sc, budget_s=args.ref_seconds, max_steps=steps, min_steps=min(3, steps))
    v = done / el
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": "substeps/s", "n_gpus": args.gpus,
           "steps": done, "warmup": args.warmup, "ms_per_step": 1000.0 * el / done, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": v / PUBLISHED_SUBSTEPS_PER_S, "dtype": "f32",
           "data": "synthetic (seeded ellipsoid particles, reference heater geometry)",
           "config": plain_config(spec.n, args.spinup),
           "cpu_baseline": {"value": v, "unit": "substeps/s", "cores": O.num_threads(), "kind": "port",
                            "sample": f"{done} substeps (of --steps {steps}, bounded to {args.ref_seconds:.0f} s) of the "
                                      f"workload on the CPU port (oracle/hf_oracle.c, OpenMP), after "
                                      f"{args.spinup}+{args.warmup} untimed substeps ({t_setup:.0f} s)"},
           "e2e": {"value": v, "unit": "substeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "note": "warp-lang is not installable here; the reference's own Warp device='cpu' path is unavailable, "
                   "the CPU port of its algorithm stands in"}
    print(json.dumps(out), flush=True)


# --------------------------------------------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and throttle reasons of GPU `index` during the timed region, read through NVML (nvidia_ml_py) every
    ~2 ms on a thread, so that a region of a few ms still holds samples; nvidia-smi -lms 50 where NVML is unavailable.
    Reads only: no clock or other GPU setting is changed."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASON_BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, index):
        self.index = index
        self.f = None
        self.p = None
        self.thread = None
        self.samples = []

    def _poll(self, nvml, handle, stop):
        reasons_fn = getattr(nvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nvml.nvmlDeviceGetCurrentClocksThrottleReasons
        while not stop.is_set():
            try:
                sm = nvml.nvmlDeviceGetClockInfo(handle, nvml.NVML_CLOCK_SM)
                mx = nvml.nvmlDeviceGetMaxClockInfo(handle, nvml.NVML_CLOCK_SM)
                rs = reasons_fn(handle)
            except Exception:  # noqa: BLE001 - a failed read ends the sampling, it does not end the bench
                break
            self.samples.append((time.perf_counter(), float(sm), float(mx), int(rs)))
            time.sleep(0.002)

    def start(self):
        import threading
        try:
            import pynvml as nvml
            nvml.nvmlInit()
            handle = nvml.nvmlDeviceGetHandleByIndex(self.index)
        except Exception:  # noqa: BLE001 - no NVML: fall back to nvidia-smi
            nvml = None
        if nvml is not None:
            self.stop_evt = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(nvml, handle, self.stop_evt), daemon=True)
            self.thread.start()
            t_wait = time.perf_counter()
            while not self.samples and self.thread.is_alive() and time.perf_counter() - t_wait < 2.0:
                time.sleep(0.001)
            self.t0 = time.perf_counter()
            return
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader",
                                       "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.thread is not None:
            t1 = time.perf_counter()
            self.stop_evt.set()
            self.thread.join(timeout=5)
            inside = [s for s in self.samples if self.t0 <= s[0] <= t1]
            if not inside:
                before = [s for s in self.samples if s[0] <= t1]
                inside = before[-1:]
            if not inside:
                return None
            reasons = sorted(nm for nm, bit in self.REASON_BITS.items() if any(s[3] & bit for s in inside))
            return {"sm_mhz": statistics.median(s[1] for s in inside), "sm_max_mhz": max(s[2] for s in inside),
                    "reasons": reasons, "samples": len(inside), "source": "nvml"}
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().strip().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1].split()[0]))
                mx.append(float(r[2].split()[0]))
            except (ValueError, IndexError):
                continue
            for nm, val in zip(names, r[5:9]):
                if "Active" in val and "Not" not in val:
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvidia-smi"}


# --------------------------------------------------------------------------------------------------- bytes
def pressure_bytes_per_launch(N, iters):
    """Algorithmic bytes of one pressure-solve launch: 52 N per CG iteration (matvec 20 N + vector update 32 N),
    36 N of set-up (read rhs, p, alpha_f x3; write rhs, diag, r, z) and 28 N for the projection (read u,v,w,p;
    write u,v,w), 4-byte words."""
    return (52.0 * iters + 36.0 + 28.0) * N


def substep_bytes(N, it_heat, it_pressure, coupled):
    """Algorithmic bytes of one whole air substep: 158 N + 45 N per heat CG iteration + 52 N per pressure CG iteration
    (air-only; statics counted once per scene), +32 N when particles rebuild the obstacle fields (T pre-stage +8 N,
    heat rhs +12 N, divergence +12 N)."""
    return (158.0 + (32.0 if coupled else 0.0) + 45.0 * it_heat + 52.0 * it_pressure) * N


def roofline(achieved_gbs, peaks, **extra):
    peak = float(peaks.get("hbm_gbs", 6650.0))
    out = {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s", "frac": achieved_gbs / peak,
           "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}
    out.update(extra)
    return out


def stage_breakdown(plan, stages, substeps=20):
    """Mean device time of every stage of a substep, from CUDA events around each stage launch over `substeps`
    substeps run after the timed region (the stages in substep order, warm caches as in the timed run)."""
    import torch
    ev = {nm: [] for nm, _ in stages}
    for _ in range(substeps):
        for nm, fn in stages:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            ev[nm].append((a, b))
    torch.cuda.synchronize()
    return {nm: sum(a.elapsed_time(b) for a, b in v) / len(v) for nm, v in ev.items()}


# --------------------------------------------------------------------------------------------------- plain
def bench_plain(args, dev, rank, world, local):
    import torch
    from heatflow_mpm.synthetic import coupled_default
    steps = args.steps if args.steps is not None else 1000
    sim = coupled_default(device=dev, cg=args.cg)
    sc, plan = sim.scene, sim.plan
    plan.resident_tiles = args.resident_tiles
    plan.plan.persistent_blocks = args.persistent_blocks
    from heatflow_mpm import _lib as L_
    plan.plan.options |= {"none": 0, "heat": L_.HF_PLAN_STREAMING_HEAT, "both": L_.HF_PLAN_STREAMING_CG}[args.streaming]
    if args.no_tma:
        plan.plan.options |= L_.HF_PLAN_NO_TMA
    n = sim.grid.n
    N = n ** 3
    stream = torch.cuda.current_stream()
    for _ in range(args.spinup + args.warmup):
        sim.substep(DT)
    torch.cuda.synchronize()
    st0 = sc.read_state()
    state_at_start = {nm: sc.current(nm).cpu().numpy().copy() for nm in ("T", "u", "v", "w")}
    p_at_start = sc.p.cpu().numpy().copy()
    ptemp_at_start = sc.ptemp.cpu().numpy().copy()
    # ---- timed region: K substeps, stage by stage, events around every pressure-solve launch.  By default the K
    # substeps are captured once as a CUDA graph (external event-record nodes around each pressure launch) and the
    # timed region is that graph's single replay: the same launches without the host in the loop.
    def one_substep(k, stream_):
        plan.obstacle_fields()
        plan.temperature_stage(DT)
        plan.heat_solve(DT)
        plan.particle_update()
        plan.face_stage(DT)
        plan.divergence_stage(DT)
        pe[k][0].record(stream_)
        plan.pressure_cg(DT)
        pe[k][1].record(stream_)

    use_graph = not args.no_graph
    pe = [(torch.cuda.Event(enable_timing=True, external=use_graph), torch.cuda.Event(enable_timing=True, external=use_graph))
          for _ in range(steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    graph = None
    if use_graph:
        cap = torch.cuda.Stream(dev)
        cap.wait_stream(stream)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=cap):
            for k in range(steps):
                one_substep(k, cap)
        torch.cuda.synchronize()
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    t_start.record(stream)
    if graph is not None:
        graph.replay()
    else:
        for k in range(steps):
            one_substep(k, stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    el_ms = reduce_max(t_start.elapsed_time(t_end), dev, world)
    st1 = sc.read_state()
    p_iters = int(st1.total_pressure_iters - st0.total_pressure_iters)
    h_iters = int(st1.total_heat_iters - st0.total_heat_iters)
    cg_ms = sum(a.elapsed_time(b) for a, b in pe)
    value = world * steps / (el_ms / 1000.0)
    # scatter (+ footprint box), obstacle, coeff, prestage, advect_T, heat CG, particle update, face, divergence, pressure CG
    launches_per_step = 10
    stage_ms = stage_breakdown(plan, [("obstacle", plan.obstacle_fields), ("temperature", lambda: plan.temperature_stage(DT)),
                                      ("heat_cg", lambda: plan.heat_solve(DT)), ("particles", plan.particle_update),
                                      ("face", lambda: plan.face_stage(DT)), ("divergence", lambda: plan.divergence_stage(DT)),
                                      ("pressure_cg", lambda: plan.pressure_cg(DT))])
    # ---- end to end through the public API: pinned H2D of the particle state and D2H of grid_T every substep,
    # pipelined two deep (grid_T_async downloads while the next substep runs; step s-2's result is read on the host
    # before step s is launched)
    # the same K substeps as the timed region: restore its start state (the substep is deterministic)
    for nm in ("T", "u", "v", "w"):
        sc.set_current(nm, state_at_start[nm])
    sc.p.copy_(torch.as_tensor(p_at_start, device=dev))
    sc.ptemp.copy_(torch.as_tensor(ptemp_at_start, device=dev))
    pos_h = sim.body.pos_t.cpu().pin_memory()
    vel_h = sim.body.vel_t.cpu().pin_memory()
    out_h = [torch.empty((n, n, n), dtype=torch.float32).pin_memory() for _ in range(2)]
    done = []
    consumed = 0.0
    # one-time set-up of the download path (staging buffers, copy stream) and of the pinned upload, outside the timed
    # loop; neither changes the scene state
    sim.body.set_state(pos_h, vel_h)
    sim.grid_T_async(out_h[1]).synchronize()
    st_e0 = sc.read_state()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in range(steps):
        if s >= 2:
            done[s - 2].synchronize()
            consumed += float(out_h[s % 2][n // 2, n // 2, n // 2])
        sim.body.set_state(pos_h, vel_h)
        sim.substep(DT)
        done.append(sim.grid_T_async(out_h[s % 2]))
    torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t0, dev, world)
    st_e1 = sc.read_state()
    # ---- parity: the first substeps of the timed region again from its start state (the same launches without the
    # graph); the CPU port replays them below and the end states are compared
    par_steps = min(steps, PARITY_STEPS)
    for nm in ("T", "u", "v", "w"):
        sc.set_current(nm, state_at_start[nm])
    sc.p.copy_(torch.as_tensor(p_at_start, device=dev))
    sc.ptemp.copy_(torch.as_tensor(ptemp_at_start, device=dev))
    st_p0 = sc.read_state()
    for _ in range(par_steps):
        plan.substep(DT)
    torch.cuda.synchronize()
    st_p1 = sc.read_state()
    gpu_end = {nm: sc.current(nm).cpu().numpy().copy() for nm in ("T", "u", "v", "w")}
    gpu_end["ptemp"] = sc.ptemp.cpu().numpy().copy()
    gpu_par = (int(st_p1.total_pressure_iters - st_p0.total_pressure_iters),
               int(st_p1.total_heat_iters - st_p0.total_heat_iters), int(st_p1.status))
    e2e = {"value": world * steps / e2e_s, "unit": "substeps/s",
           "h2d_bytes_per_step": int(pos_h.numel() * 4 + vel_h.numel() * 4), "d2h_bytes_per_step": int(out_h[0].numel() * 4),
           "mean_pressure_iters": (st_e1.total_pressure_iters - st_e0.total_pressure_iters) / steps,
           "note": "the timed region's K substeps again from its start state, through HeatflowMPM: body.set_state "
                   "(pinned H2D) + substep + grid_T_async (D2H), two substeps in flight"}
    # ---- roofline of the dominant kernel (pressure CG + projection) and of the whole substep
    peaks = load_peaks()
    cg_bytes = pressure_bytes_per_launch(N, p_iters / steps)
    traffic = None
    single = args.cg == "single-reduction"
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "pressure_cg_one_96.json" if single else "pressure_cg_96.json")))
        traffic = prof["dram_bytes_per_iteration"] * (p_iters / steps) + prof.get("dram_bytes_fixed", 0.0)
    except (OSError, ValueError, KeyError):
        pass
    kernel = ("k_pcg_one<3> (single-reduction pressure Jacobi-PCG + projection: one grid barrier per iteration, one "
              "persistent cooperative launch, TMA-staged register-resident stencil)" if single else
              "k_pcg_tma<2> (pressure Jacobi-PCG + projection, one persistent cooperative launch, TMA-staged "
              "register-resident stencil)")
    roof = roofline(cg_bytes / (cg_ms / steps / 1000.0) / 1e9, peaks, traffic=traffic, kernel=kernel,
                    bytes_per_launch=cg_bytes, ms_per_launch=cg_ms / steps, mean_pressure_iters=p_iters / steps)
    sb = substep_bytes(N, h_iters / steps, p_iters / steps, True)
    sub_gbs = sb / (el_ms / steps / 1000.0) / 1e9
    sub_roof = {"bytes_per_substep": sb, "achieved": sub_gbs, "unit": "GB/s", "frac": sub_gbs / roof["peak"]}
    # ---- CPU baseline: the CPU port from the same state, bounded sample (rank 0, N = 1)
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.set_threads(host_threads())
        osc, _ = cpu_scene()
        osc.set_state(T=state_at_start["T"], u=state_at_start["u"], v=state_at_start["v"], w=state_at_start["w"])
        osc.a["p"][...] = p_at_start
        osc.a["ptemp"][: len(ptemp_at_start)] = ptemp_at_start
        # the sample's first par_steps substeps are the parity replay (not time-bounded); the rest is bounded
        done, el, o_it_p, o_it_h = oracle_substeps(osc, par_steps)
        parity = plain_parity(gpu_end, osc, par_steps, gpu_par, (o_it_p, o_it_h))
        if steps > par_steps and el < args.cpu_seconds:
            d2, e2, _, _ = oracle_substeps(osc, steps - par_steps, args.cpu_seconds - el)
            done, el = done + d2, el + e2
        threads = O.num_threads()
        # the same port on one thread, from the state the sample above reached (bounded to a third of the budget)
        O.set_threads(1)
        done1, el1 = time_cpu_substeps(osc, args.cpu_seconds / 3, max_steps=steps)
        O.set_threads(host_threads())
        cpu = {"value": done / el, "unit": "substeps/s", "cores": threads, "kind": "port",
               "sample": f"{done} substeps of the same workload from the same state on the CPU port "
                         f"(oracle/hf_oracle.c, OpenMP {threads} threads), {el:.1f} s",
               "single_thread": {"value": done1 / el1, "substeps": done1, "seconds": el1}}
    return {"metric": METRIC, "value": value, "unit": "substeps/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": el_ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / PUBLISHED_SUBSTEPS_PER_S, "dtype": "f32",
            "data": "synthetic (seeded ellipsoid particles, reference heater geometry)",
            "config": plain_config(n, args.spinup),
            "details": {"parallelism": f"replicas x{world}",
                        "mean_pressure_iters": p_iters / steps, "mean_heat_iters": h_iters / steps,
                        "cell_updates_per_s": value * N, "substep_status": int(st1.status),
                        "substep_roofline": sub_roof, "stage_ms": stage_ms,
                        "timed_launches": "one CUDA-graph replay of the K substeps" if use_graph else "eager launches",
                        "pressure_cg": args.cg},
            "parity": parity,
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches_per_step * steps, "clocks": ck}


def plain_parity(gpu_end, osc, steps, gpu_iters, oracle_iters):
    """The GPU's end state after the first `steps` timed substeps against the CPU port's replay of the same substeps
    from the same start state (build arithmetic): relative L2 of T, u, v, w and the particle temperatures, max |dT|,
    CG iterations (pressure, heat) and the GPU's status bits."""
    def rel(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
    P = len(gpu_end["ptemp"])
    return {"vs": "oracle/hf_oracle.c (CPU port, build arithmetic), the same substeps from the same start state",
            "substeps": steps, "tolerance_rel_l2": 1e-6,
            "rel_l2_T": rel(gpu_end["T"], osc.T), "rel_l2_u": rel(gpu_end["u"], osc.u),
            "rel_l2_v": rel(gpu_end["v"], osc.v), "rel_l2_w": rel(gpu_end["w"], osc.w),
            "rel_l2_ptemp": rel(gpu_end["ptemp"], osc.a["ptemp"][:P]),
            "max_abs_T": float(np.abs(gpu_end["T"].astype(np.float64) - osc.T).max()),
            "pressure_iters": {"gpu": gpu_iters[0], "oracle": oracle_iters[0]},
            "heat_iters": {"gpu": gpu_iters[1], "oracle": oracle_iters[1]}, "gpu_status": gpu_iters[2]}


# ---------------------------------------------------------------------------------------------------- config 1
CONFIG1 = ("32^3 air-only plume: h=15 mm, box heater (4x4x2 rod cells at x=0.1 m + trough layer), 400 W capped at "
           "120 C, fan 0, walls 25 C, seeded +-0.01 K noise, pressure and heat CG tol 1e-6, dt=2 ms, 100 substeps")


def config1_summary(dev, cpu=True, cpu_seconds=20.0):
    """The CPU-runnable configuration end to end: its 100 substeps on the GPU through HeatflowMPM.substep (CUDA events
    on the stream; the 4 MB state stays in L2; timed after one untimed substep that records the substep graph, from
    the restored initial state) and, with cpu=True, on the CPU port at one thread and at all host threads from the
    same initial state (each bounded to cpu_seconds)."""
    import torch
    from heatflow_mpm.synthetic import plume_box
    sim = plume_box(device=dev)
    sc = sim.scene
    T0 = sc.current("T").cpu().numpy().copy()
    sim.substep(DT)
    torch.cuda.synchronize()
    for nm in ("u", "v", "w"):
        sc.current(nm).zero_()
    sc.set_current("T", T0)
    sc.p.zero_()
    st0 = sc.read_state()
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(100):
        sim.substep(DT)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    st1 = sc.read_state()
    out = {"workload": CONFIG1, "substeps": 100,
           "gpu": {"value": 100 / (ms / 1000.0), "unit": "substeps/s", "ms_per_step": ms / 100,
                   "mean_pressure_iters": (st1.total_pressure_iters - st0.total_pressure_iters) / 100,
                   "mean_heat_iters": (st1.total_heat_iters - st0.total_heat_iters) / 100, "status": int(st1.status)}}
    if cpu:
        from oracle import oracle as O
        res = {}
        for label, threads in (("threads_1", 1), ("threads_all", host_threads())):
            O.set_threads(threads)
            osc = O.scene_from_spec(sc.spec, "f32", mean_mode=0, scatter_mode=0)
            osc.set_state(T=T0)
            done, el = time_cpu_substeps(osc, cpu_seconds, max_steps=100)
            res[label] = {"value": done / el, "unit": "substeps/s", "threads": O.num_threads(), "substeps": done,
                          "seconds": el}
        O.set_threads(host_threads())
        out["cpu_port"] = dict(res, kind="port", sample="the same substeps from the same initial state on the CPU "
                                                          "port (oracle/hf_oracle.c, OpenMP)")
    return out


# --------------------------------------------------------------------------------------------------- batched
def bench_batched(args, dev, rank, world, local, steps, warmup, cpu_sample=True):
    import torch
    from heatflow_mpm.batch import AirBatch, autotune, ensemble, shard_scenarios
    scs_all = ensemble(count=args.scenes, seed=0, edges=tuple(int(e) for e in args.edges.split(",")), steps=steps)
    mine = shard_scenarios(scs_all, rank, world)
    t_build = time.perf_counter()
    batch = AirBatch(mine, device=dev)
    t_build = time.perf_counter() - t_build
    if args.launch:
        pb, gc, lanes = (int(v) for v in args.launch.split(","))
        batch.plan.plan.persistent_blocks, batch.plan.plan.group_cells, batch.plan.lanes = pb, gc, lanes
        tune = None
    elif args.no_autotune:
        (pb, gc, lanes), tune = (0, 0, 0), None
    else:
        (pb, gc, lanes), tune = autotune(batch, dt=DT, reps=2)
    for _ in range(warmup):
        batch.substep(DT)
    G = max(1, min(args.graph_steps, steps))
    batch.capture(DT, G)
    torch.cuda.synchronize()
    st0 = batch.states()
    start = batch.snapshot()   # the end-to-end leg below repeats the timed substeps from here
    stream = torch.cuda.current_stream()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    t_start.record(stream)
    for _ in range(steps // G):
        batch.graph.replay()
    for _ in range(steps % G):
        batch.substep(DT)
    t_end.record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    el_ms = reduce_max(t_start.elapsed_time(t_end), dev, world)
    st1 = batch.states()
    cells_mine = sum(s.n ** 3 for s in mine)
    cells = reduce_sum(cells_mine, dev, world)
    value = cells * steps / N96 / (el_ms / 1000.0)
    it_p = [(b.total_pressure_iters - a.total_pressure_iters) / steps for a, b in zip(st0, st1)]
    it_h = [(b.total_heat_iters - a.total_heat_iters) / steps for a, b in zip(st0, st1)]
    sb_mine = sum(substep_bytes(s.n ** 3, h, p, False) for s, h, p in zip(mine, it_h, it_p))
    sb = reduce_sum(sb_mine, dev, world)
    status = [int(s.status) for s in st1]
    # ---- stage breakdown (eager, outside the timed region): events around the pressure-CG launch of the batch
    B = 10
    pe = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(B)]
    sa = batch.states()
    plan = batch.plan
    for k in range(B):
        plan.temperature_stage(DT)
        plan.heat_solve(DT)
        plan.face_stage(DT)
        plan.divergence_stage(DT)
        pe[k][0].record(stream)
        plan.pressure_cg(DT)
        pe[k][1].record(stream)
    torch.cuda.synchronize()
    sbk = batch.states()
    cg_ms = sum(a.elapsed_time(b) for a, b in pe) / B
    cg_bytes = sum(pressure_bytes_per_launch(s.n ** 3, (b.total_pressure_iters - a.total_pressure_iters) / B)
                   for s, a, b in zip(mine, sa, sbk))
    peaks = load_peaks()
    roof = roofline(cg_bytes / (cg_ms / 1000.0) / 1e9, peaks, traffic=None,
                    kernel="k_pcg<false, true> (streaming persistent pressure Jacobi-PCG + projection over the scene table, TMA-staged double-buffered tile boxes)",
                    bytes_per_launch=cg_bytes, ms_per_launch=cg_ms, measured_on="rank 0 stage breakdown, 10 substeps")
    sub_gbs = sb / (el_ms / steps / 1000.0) / 1e9
    # ---- end to end through the public API: AirBatch.substep per substep, every scene's status block read back
    state_h = torch.empty((len(batch.scenes), batch.scenes[0].state.numel()), dtype=torch.uint8).pin_memory()
    batch.restore(start)
    del start
    e2e_steps = steps
    barrier(world)
    torch.cuda.synchronize()
    se0 = batch.states()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        batch.substep(DT)
        for i, s in enumerate(batch.scenes):
            state_h[i].copy_(s.state, non_blocking=True)
        torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t0, dev, world)
    se1 = batch.states()
    e2e = {"value": cells * e2e_steps / N96 / e2e_s, "unit": "96^3-equivalent substeps/s", "h2d_bytes_per_step": 0,
           "d2h_bytes_per_step": int(state_h.numel()), "steps": e2e_steps,
           "mean_pressure_iters": float(np.mean([(b.total_pressure_iters - a.total_pressure_iters) / e2e_steps
                                                 for a, b in zip(se0, se1)])),
           "note": "the timed substeps again from their start state: AirBatch.substep (eager, no graph) + every "
                   "scene's state block copied to pinned host memory, each substep"}
    cpu = None
    if cpu_sample and rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        v, done, visited, el = cpu_scenarios_sample(scs_all, args.cpu_seconds)
        cpu = {"value": v, "unit": "96^3-equivalent substeps/s", "cores": O.num_threads(), "kind": "port",
               "sample": f"{done} substeps: the ensemble's first {visited} scenes, 2 substeps each from their initial "
                         f"state, on the CPU port (oracle/hf_oracle.c, OpenMP), {el:.1f} s"}
    hist = {}
    for s in scs_all:
        hist[s.n] = hist.get(s.n, 0) + 1
    return {"metric": METRIC_BATCHED, "value": value, "unit": "96^3-equivalent substeps/s", "n_gpus": world,
            "steps": steps, "warmup": warmup, "ms_per_step": el_ms / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded ensemble of air-only box-heater scenes)",
            "config": {"workload": f"batched ensemble: {args.scenes} air-only scenes, edges {dict(sorted(hist.items()))}, "
                                   f"h=0.48 m/edge, box heater x U(0.05,0.2) m, 100-800 W, fan 0-3 m/s, dt=2 ms, "
                                   f"pressure tol 1e-4, heat tol 1e-6",
                       "scenes": args.scenes, "cells": int(cells), "graph_substeps": G, "persistent_blocks": pb,
                       "group_cells": gc, "lanes": lanes,
                       "autotune_ms": tune, "parallelism": f"scene-sharded x{world}",
                       "l2": f"{cells * 4 * 40 / 1e9:.1f} GB of scene state > 126 MB L2 (inputs larger than L2)",
                       "scene_substeps_per_s": len(scs_all) * steps / (el_ms / 1000.0),
                       "cell_updates_per_s": cells * steps / (el_ms / 1000.0),
                       "mean_pressure_iters": float(np.mean(it_p)), "mean_heat_iters": float(np.mean(it_h)),
                       "status_nonzero": int(sum(1 for x in status if x)), "build_s": t_build,
                       "substep_roofline": {"bytes_per_substep": sb, "achieved": sub_gbs, "unit": "GB/s",
                                            "frac": sub_gbs / roof["peak"]}},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": 6 * steps, "clocks": ck}


# --------------------------------------------------------------------------------------------------- served
def bench_served(args, dev, rank, world, local, cpu_sample=True):
    import torch
    from heatflow_mpm.serve import AirServer, poisson_trace
    trace_all = poisson_trace(rate=args.rate, duration=args.serve_seconds, seed=0)
    trace = [r for r in trace_all if r.rid % world == rank]
    srv = AirServer(device=dev, dt=DT, hbm_budget=args.hbm_budget, max_slots=args.max_slots)
    # warm-up: one small request served to completion (module loading, kernel attributes), not counted
    from heatflow_mpm.batch import AirScenario
    from heatflow_mpm.serve import Request
    warm = AirServer(device=dev, dt=DT)
    warm.serve([Request(AirScenario(n=48, horizon=max(3, args.warmup)), 0.0)], time_limit=120.0)
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    out = srv.serve(trace, time_limit=args.serve_seconds)
    torch.cuda.synchronize()
    ck = clocks.stop()
    busy_s = reduce_max(sum(srv.substep_ms) / 1000.0, dev, world)
    wall_s = reduce_max(srv.elapsed, dev, world)
    work = reduce_sum(srv.weighted_substeps, dev, world)
    scene_substeps = reduce_sum(srv.scene_substeps, dev, world)
    steps = max(1, len(srv.substep_ms))
    cpu = None
    if cpu_sample and rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        v, done, visited, el = cpu_scenarios_sample([r.scenario for r in trace_all], args.cpu_seconds)
        cpu = {"value": v, "unit": "96^3-equivalent substeps/s", "cores": O.num_threads(), "kind": "port",
               "sample": f"{done} substeps: the trace's first {visited} requests, 2 substeps each from their initial "
                         f"state, on the CPU port (oracle/hf_oracle.c, OpenMP), {el:.1f} s"}
    return {"metric": METRIC_SERVED, "value": work / busy_s, "unit": "96^3-equivalent substeps/s", "n_gpus": world,
            "steps": len(srv.substep_ms), "warmup": max(3, args.warmup), "ms_per_step": 1000.0 * busy_s / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Poisson trace of air-only trough-heater scenes, half with a static sphere)",
            "config": {"workload": f"served: Poisson arrivals {args.rate}/s for {args.serve_seconds:.0f} s, edges "
                                   f"{{48,64,96,128}}, horizon U(200,2000), 100-800 W, fan 0-3 m/s, sphere r U(2,6) cm "
                                   f"p=0.5, HBM budget {args.hbm_budget / 1e9:.0f} GB, max {args.max_slots} scenes/batch",
                       "requests": len(trace_all), "requests_done": int(reduce_sum(out["requests_done"], dev, world)),
                       "requests_failed": int(reduce_sum(out["requests_failed"], dev, world)),
                       "requests_unfinished": int(reduce_sum(out["requests_unfinished"], dev, world)),
                       "window_s": args.serve_seconds,
                       "completed_fraction": out["completed_fraction"],
                       "request_latency_p50_s": out["request_latency_p50_s"],
                       "request_latency_p99_s": out["request_latency_p99_s"],
                       "unfinished_age_p50_s": out["unfinished_age_p50_s"],
                       "unfinished_age_p99_s": out["unfinished_age_p99_s"],
                       "substep_latency_p50_ms": out["substep_latency_p50_ms"],
                       "substep_latency_p99_ms": out["substep_latency_p99_ms"],
                       "scene_substeps": int(scene_substeps), "plan_builds": out["plan_builds"],
                       "scene_setup": out["setup"], "admit_ms_p50": out["admit_ms_p50"],
                       "admit_ms_p99": out["admit_ms_p99"],
                       "gpu_busy_frac": busy_s / wall_s, "parallelism": f"request-sharded x{world}",
                       "latency_note": "request latency = arrival to result on the host, over the requests completed "
                                       "in the window (rank 0); unfinished ages = window end minus arrival of the "
                                       "requests still queued or running",
                       "l2": "resident scene state of the admitted requests >> 126 MB L2"},
            "roofline": None, "cpu_baseline": cpu,
            "e2e": {"value": work / wall_s, "unit": "96^3-equivalent substeps/s",
                    "h2d_bytes_per_step": int(srv.h2d_bytes / steps), "d2h_bytes_per_step": int(srv.d2h_bytes / steps),
                    "note": "wall clock of the serving window: admission, scene upload, plan rebuilds and result "
                            "download (T of every completed request) included"},
            "gpu_launches": 6 * len(srv.substep_ms), "clocks": ck}


def compact(line):
    keep = ("value", "unit", "ms_per_step", "steps", "e2e", "cpu_baseline", "clocks")
    out = {k: line.get(k) for k in keep}
    out["roofline_frac"] = (line.get("roofline") or {}).get("frac")
    out["config"] = line.get("config")
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.workload == "plain":
        out = bench_plain(args, dev, rank, world, local)
        if not args.no_extras:
            if rank == 0 and world == 1:
                out["config1"] = config1_summary(dev, cpu=not args.no_cpu_baseline, cpu_seconds=args.cpu_seconds)
            b = bench_batched(args, dev, rank, world, local, steps=200, warmup=3, cpu_sample=False)
            out["batched"] = compact(b)
            out["batched"]["plain_ratio"] = b["value"] / out["value"]
            out["served"] = compact(bench_served(args, dev, rank, world, local, cpu_sample=False))
            out["served"]["plain_ratio"] = out["served"]["value"] / out["value"]
    elif args.workload == "batched":
        out = bench_batched(args, dev, rank, world, local, args.steps if args.steps is not None else 200,
                            max(3, args.warmup))
    else:
        out = bench_served(args, dev, rank, world, local)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""bench.py without a GPU: the CPU reference arm prints one JSON line with every key of the output contract (rank 0
alone; other ranks exit 0 silently).  And for bench.py, the package, the entry module and the oracle's front end:
every name a function reads is bound somewhere it can see (a misspelt or stale name in a branch that only a GPU run
takes would otherwise surface only there)."""
import ast
import builtins
import json
import os
import subprocess
import sys

from conftest import ROOT

BENCH = os.path.join(ROOT, "bench.py")


def _run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, BENCH, "--impl", "reference", *args], capture_output=True, text=True,
                          env=env, timeout=600, cwd=ROOT)


def test_reference_arm_contract():
    r = _run({}, "--steps", "2", "--warmup", "3", "--spinup", "2")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True and d["warmup"] == 3
    assert "workload" in d["config"]
    # the same config dict as the GPU arm's plain line (bench.plain_config): what the workload is, nothing measured
    assert set(d["config"]) == {"workload", "n", "cells", "spinup", "dt", "l2"}
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_are_silent():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--steps", "2", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def _bound(nodes, into_functions):
    out, stack = set(), list(nodes)
    while stack:
        n = stack.pop()
        if isinstance(n, ast.Name) and isinstance(n.ctx, (ast.Store, ast.Del)):
            out.add(n.id)
        elif isinstance(n, (ast.FunctionDef, ast.AsyncFunctionDef, ast.ClassDef)):
            out.add(n.name)
            if not into_functions:
                continue
        elif isinstance(n, ast.arg):
            out.add(n.arg)
        elif isinstance(n, (ast.Import, ast.ImportFrom)):
            out.update((a.asname or a.name).split(".")[0] for a in n.names)
        elif isinstance(n, ast.ExceptHandler) and n.name:
            out.add(n.name)
        elif isinstance(n, (ast.Global, ast.Nonlocal)):
            out.update(n.names)
        stack.extend(ast.iter_child_nodes(n))
    return out


def _reads(nodes, visible, where, found):
    """Names read by `nodes` (evaluated in a scope that sees `visible`) that nothing binds."""
    stack = list(nodes)
    while stack:
        n = stack.pop()
        if isinstance(n, (ast.FunctionDef, ast.AsyncFunctionDef, ast.Lambda)):
            _unbound_reads(n, visible, found)      # its decorators and defaults are read here, its body in its own scope
            continue
        if isinstance(n, ast.ClassDef):
            _reads(n.decorator_list + n.bases, visible, where, found)
            inside = visible | _bound(n.body, False)       # class-body names: seen by the body's own statements and by
            for st in n.body:                              # method decorators and defaults, not by method bodies
                if isinstance(st, (ast.FunctionDef, ast.AsyncFunctionDef)):
                    _unbound_reads(st, visible, found, outer=inside)
                else:
                    _reads([st], inside, n.name, found)
            continue
        if isinstance(n, ast.Name) and isinstance(n.ctx, ast.Load) and n.id not in visible:
            found.append(f"{where}:{n.lineno}: {n.id}")
        stack.extend(ast.iter_child_nodes(n))


def _unbound_reads(fn, visible, found, outer=None):
    """fn's decorators and defaults are read in `outer` (default: visible), its body in its own scope over `visible`."""
    args = fn.args
    _reads(getattr(fn, "decorator_list", []) + args.defaults + [d for d in args.kw_defaults if d is not None],
           visible if outer is None else outer, getattr(fn, "name", "lambda"), found)
    params = {a.arg for a in args.posonlyargs + args.args + args.kwonlyargs}
    params |= {a.arg for a in (args.vararg, args.kwarg) if a is not None}
    body = fn.body if isinstance(fn.body, list) else [fn.body]
    local = _bound(body, False) | params | visible
    _reads(body, local, getattr(fn, "name", "lambda"), found)


def _check_file(path):
    tree = ast.parse(open(path).read())
    module = _bound(tree.body, False) | set(dir(builtins)) | {"__file__", "__name__"}
    found = []
    for node in tree.body:
        if isinstance(node, (ast.FunctionDef, ast.AsyncFunctionDef)):
            _unbound_reads(node, module, found)
        elif isinstance(node, ast.ClassDef):
            _reads([node], module, node.name, found)
    return [f"{os.path.basename(path)}:{f}" for f in found]


def test_bench_functions_read_only_bound_names():
    assert not _check_file(BENCH)


def test_package_functions_read_only_bound_names():
    import glob
    files = glob.glob(os.path.join(ROOT, "heatflow-mpm_b200", "heatflow_mpm", "*.py"))
    files += [os.path.join(ROOT, "__graft_entry__.py")] + glob.glob(os.path.join(ROOT, "oracle", "*.py"))
    found = [f for p in sorted(files) for f in _check_file(p)]
    assert not found, found


def test_clock_sampler_with_a_fake_nvml(monkeypatch):
    """bench.ClockSampler reads the SM clock and the clock-event reasons through NVML on a thread during the timed
    region: the samples taken between start() and stop() are summarised (median clock, max clock, the reason names of
    every bit seen).  A fake pynvml stands in for the driver here; it reports sw_power_cap (bit 0x4) and hw_slowdown
    (0x8).  With no NVML at all the sampler falls back to nvidia-smi and, when that is missing too, returns None."""
    import time
    import types
    sys.path.insert(0, ROOT)
    import bench
    class FakeNvml:
        NVML_CLOCK_SM = 1
        reads = 0

        @staticmethod
        def nvmlInit():
            pass

        @staticmethod
        def nvmlDeviceGetHandleByIndex(i):
            return ("gpu", i)

        @classmethod
        def nvmlDeviceGetClockInfo(cls, handle, kind):
            cls.reads += 1
            return 1800

        @staticmethod
        def nvmlDeviceGetMaxClockInfo(handle, kind):
            return 1965

        @staticmethod
        def nvmlDeviceGetCurrentClocksEventReasons(handle):
            return 0x4 | 0x8

    monkeypatch.setitem(sys.modules, "pynvml", FakeNvml)
    cs = bench.ClockSampler(0)
    cs.start()
    time.sleep(0.05)
    out = cs.stop()
    assert out is not None and out["source"] == "nvml"
    assert out["samples"] >= 1 and FakeNvml.reads >= out["samples"]
    assert out["sm_mhz"] == 1800 and out["sm_max_mhz"] == 1965
    assert out["reasons"] == ["hw_slowdown", "sw_power_cap"]

    broken = types.SimpleNamespace(nvmlInit=lambda: (_ for _ in ()).throw(RuntimeError("no driver")))
    monkeypatch.setitem(sys.modules, "pynvml", broken)
    monkeypatch.setenv("PATH", "/nonexistent")
    cs = bench.ClockSampler(0)
    cs.start()
    assert cs.stop() is None

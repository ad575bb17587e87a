"""Frame output of a running simulation without stalling it.

``FrameWriter`` writes the frames of the reference's scene driver (scripts/run_scene.py:31-40:
``frames/frame_NNNN.npz`` with t, pos, vel f32, temp f16, melt f16, grid_T f16 [n^3], air_u f16 [n^3, 3]; the
fields of solver.py:105-110 frame_dict).  A frame is packed on the device by one kernel (``hf_pack_frame``: binary16
conversion with round-to-nearest-even, as numpy's astype(float16)) into a slot of a small ring of device buffers; a
side stream copies the slot and the particle state into pinned host memory while the compute stream runs the next
substeps, and a background thread writes the npz once the copy has landed.  The substep loop only enqueues work.
The files are bit-identical to ``np.savez(path, **sim.frame_dict(t))`` at the same state.
"""
from __future__ import annotations

import ctypes as C
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import _lib


class _Slot:
    def __init__(self, n, P, device):
        N = n ** 3
        self.N, self.P = N, P
        self.dev = torch.empty(4 * N + 2 * max(P, 1), dtype=torch.int16, device=device)
        self.host = torch.empty(self.dev.shape, dtype=torch.int16).pin_memory()
        self.pos = torch.empty((max(P, 1), 3), dtype=torch.float32).pin_memory()
        self.vel = torch.empty((max(P, 1), 3), dtype=torch.float32).pin_memory()
        self.done = torch.cuda.Event()
        self.pending = None      # (path, t, with_air)
        self.future = None


class FrameWriter:
    """Asynchronous frames of one HeatflowMPM (see the module docstring); `depth` frames may be in flight."""

    def __init__(self, sim, out_dir, depth=2):
        self.sim = sim
        self.out = out_dir
        os.makedirs(out_dir, exist_ok=True)
        self.dev = sim.scene.device
        self.slots = [_Slot(sim.grid.n, sim.n, self.dev) for _ in range(depth)]
        self.copy_stream = torch.cuda.Stream(self.dev)
        self.pool = ThreadPoolExecutor(max_workers=1)
        self.k = 0

    def write(self, index: int, t: float, with_air: bool = True) -> str:
        """Enqueue frame `index` at time t; returns the path it will have."""
        slot = self.slots[self.k % len(self.slots)]
        self.k += 1
        self._finish(slot)
        sim, N, P = self.sim, slot.N, slot.P
        base = slot.dev.data_ptr()
        plan = sim.plan
        compute = torch.cuda.current_stream(self.dev)
        _lib.check(plan.L.hf_pack_frame(C.byref(plan.plan), 0, base, base + 2 * N if with_air else None,
                                        base + 8 * N if P else None, base + 8 * N + 2 * P if P else None,
                                        C.c_void_p(compute.cuda_stream)), "hf_pack_frame")
        pos, vel = sim.body.particle_state() if (sim.body is not None and P) else (None, None)
        self.copy_stream.wait_stream(compute)
        with torch.cuda.stream(self.copy_stream):
            slot.host.copy_(slot.dev, non_blocking=True)
            if pos is not None:
                slot.pos[:P].copy_(pos[:P], non_blocking=True)
                slot.vel[:P].copy_(vel[:P], non_blocking=True)
            slot.done.record(self.copy_stream)
        # the slot's device buffer and the particle tensors must outlive the copy
        slot.dev.record_stream(self.copy_stream)
        path = os.path.join(self.out, f"frame_{index:04d}.npz")
        slot.pending = (path, float(t), with_air)
        return path

    def _finish(self, slot):
        if slot.future is not None:
            slot.future.result()
            slot.future = None
        if slot.pending is None:
            return
        path, t, with_air = slot.pending
        slot.pending = None
        slot.done.synchronize()
        N, P = slot.N, slot.P
        h = slot.host.numpy().view(np.float16)
        d = dict(t=np.float32(t), pos=slot.pos[:P].numpy().copy(), vel=slot.vel[:P].numpy().copy(),
                 temp=h[8 * N // 2: 8 * N // 2 + P].copy() if P else np.zeros(0, np.float16),
                 melt=h[8 * N // 2 + P: 8 * N // 2 + 2 * P].copy() if P else np.zeros(0, np.float16),
                 grid_T=h[:N].copy())
        if with_air:
            d["air_u"] = h[N: 4 * N].reshape(N, 3).copy()
        slot.future = self.pool.submit(np.savez, path, **d)

    def flush(self):
        """Wait until every enqueued frame is on disk."""
        for _ in range(2):
            for slot in self.slots:
                self._finish(slot)

    def close(self):
        self.flush()
        self.pool.shutdown()

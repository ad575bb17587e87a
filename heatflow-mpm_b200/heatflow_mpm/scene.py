"""Device-resident air scenes and launch plans over them.

``DeviceScene`` owns every field of one scene as a torch CUDA tensor, in the reference's array shapes (cells (n,n,n);
u (n+1,n,n); v (n,n+1,n); w (n,n,n+1)), and the ``hf_scene`` record that points at them.  ``ScenePlan`` puts one or
more scenes into a launch plan (scene table + 1024-cell work table + workspace, all device tensors) and calls the C
ABI of libheatflow_b200.so on the current torch stream.

Air-only scenes share read-only buffers: their obstacle fields are the static heater fields themselves (kx..mz point at
the static face weights, alpha_s at the static solid fraction) and the particle flux q is one zero face array.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib

F32 = torch.float32


def face_shapes(n):
    return [(n + 1, n, n), (n, n + 1, n), (n, n, n + 1)]


@dataclass
class SceneSpec:
    """Everything that defines one air scene (all defaults are the reference's)."""
    n: int
    h: float
    rho: float = 1.2
    t_amb: float = 25.0
    alpha_f_min: float = 0.05
    g: float = 9.81
    buoyancy: bool = True
    cg_tol: float = 1e-4
    cg_max_iter: int = 400
    heat_tol: float = 1e-6
    heat_maxiter: int = 200
    kappa_air: float = 2.2e-5
    kappa_mat: float = 2.0e-5
    fixed: np.ndarray | None = None          # bool (n,n,n)
    tfix: np.ndarray | None = None           # float (n,n,n)
    source: np.ndarray | None = None         # bool (n,n,n)
    rate: float = 0.0
    t_cap: float = 0.0
    static_alpha: np.ndarray | None = None   # float (n,n,n)
    static_k: list | None = None             # 3 face arrays
    static_m: list | None = None
    n_particles: int = 0
    spacing: float = 2.5e-3
    k_particle: float = 1.0e-3
    t_sol: float = 30.0
    t_liq: float = 36.0
    y_solid: float = 2.0e4
    mu_s: float = 5.0
    mu_l: float = 30.0
    t_max: float = 300.0
    t_init_grid: float | None = None         # initial grid temperature (default t_amb)
    defect_correction: bool = False          # fp64 true-residual check and restart after each CG solve (not in the reference)
    statics: object = None                   # voxelize.SceneStatics built on the device: replaces fixed, tfix, source and
                                             # the static_* arrays
    extra: dict = field(default_factory=dict)


class DeviceScene:
    def __init__(self, spec: SceneSpec, device="cuda:0"):
        _lib.load()
        self.spec = spec
        self.device = torch.device(device)
        n = self.n = spec.n
        dev = self.device
        z = lambda *s, dtype=F32: torch.zeros(s, dtype=dtype, device=dev)
        fs = face_shapes(n)
        t0 = spec.t_amb if spec.t_init_grid is None else spec.t_init_grid
        self.T = [torch.full((n, n, n), t0, dtype=F32, device=dev) for _ in range(2)]
        self.u = [z(*fs[0]) for _ in range(2)]
        self.v = [z(*fs[1]) for _ in range(2)]
        self.w = [z(*fs[2]) for _ in range(2)]
        self.Tw = torch.full((n, n, n), t0, dtype=F32, device=dev)
        for name in ("kap", "hrhs", "hdiag", "tfix", "p", "rhs", "pdiag", "cg_r", "cg_z", "cg_Ap"):
            setattr(self, name, z(n, n, n))
        self.cg_p = [z(n, n, n), z(n, n, n)]
        self.ax, self.ay, self.az = (z(*s) for s in fs)
        self.hk = [z(*s) for s in fs]
        self.ayc, self.azc, self.hkzc = z(n, n, n), z(n, n, n), z(n, n, n)
        self.cell_flags = z(n, n, n, dtype=torch.uint8)
        coupled = spec.n_particles > 0
        dst = spec.statics
        has_static = spec.static_alpha is not None or dst is not None
        if dst is not None:
            self.st_alpha, self.st_k, self.st_m = dst.alpha, list(dst.k), list(dst.m)
        elif has_static:
            up = lambda a: torch.as_tensor(np.require(a, np.float32, ("C", "W")), device=dev)   # host copy if read-only
            self.st_alpha = up(spec.static_alpha)
            self.st_k = [up(a) for a in spec.static_k]
            self.st_m = [up(a) for a in spec.static_m]
        else:
            self.st_alpha, self.st_k, self.st_m = None, [None] * 3, [None] * 3
        if coupled:
            self.alpha_s, self.alpha, self.tsum = z(n, n, n), z(n, n, n), z(n, n, n)
            self.q = [z(*s) for s in fs]
            self.k = [z(*s) for s in fs]
            self.m = [z(*s) for s in fs]
            self.acc = torch.zeros(12 * (n + 1) ** 3, dtype=torch.int64, device=dev)
            P = spec.n_particles
            self.pos, self.pvel = z(P, 3), z(P, 3)
            self.ptemp, self.pmelt, self.pyield, self.pvisc = z(P), z(P), z(P), z(P)
        else:
            zero_face = z((n + 1) * n * n)
            self.zero_cell = z(n, n, n)
            self.q = [zero_face.view(s) for s in fs]
            if has_static:
                self.alpha_s, self.k, self.m = self.st_alpha, list(self.st_k), list(self.st_m)
            else:
                self.alpha_s = self.zero_cell
                self.k = [zero_face.view(s) for s in fs]
                self.m = [zero_face.view(s) for s in fs]
            self.alpha, self.tsum = self.zero_cell, self.zero_cell
            self.acc = None
            self.pos = self.pvel = self.ptemp = self.pmelt = self.pyield = self.pvisc = None
        st0 = _lib.SceneState()
        for i in range(3):
            st0.box[i] = st0.box_prev[i] = 2 ** 31 - 1
            st0.box[3 + i] = st0.box_prev[3 + i] = -2 ** 31
        self.state = torch.frombuffer(bytearray(bytes(st0)), dtype=torch.uint8).to(dev)
        self._parity_host = 0
        self.dirty = False
        if dst is not None:
            self.cell_flags, self.tfix = dst.cell_flags, dst.tfix
        else:
            fixed = np.zeros((n, n, n), bool) if spec.fixed is None else np.asarray(spec.fixed, bool)
            tfix = np.zeros((n, n, n), np.float32) if spec.tfix is None else spec.tfix
            source = np.zeros((n, n, n), bool) if spec.source is None else np.asarray(spec.source, bool)
            self._set_flags(fixed, tfix, source)
        self.rate, self.t_cap = float(spec.rate), float(spec.t_cap)
        self.record = _lib.Scene()
        self.fill_record()
        self.apply_fixed_to_T()

    # --------------------------------------------------------------------------------------------- set-up
    def _set_flags(self, fixed, tfix, source):
        flags = np.asarray(fixed, bool).astype(np.uint8) | (np.asarray(source, bool).astype(np.uint8) << 1)
        self.cell_flags.copy_(torch.as_tensor(flags, device=self.device))
        self.tfix.copy_(torch.as_tensor(np.require(tfix, np.float32, ("C", "W")), device=self.device))

    def set_fixed(self, fixed, values):
        """heat.py:189-192: new Dirichlet mask and values, applied to T at once."""
        src = (self.cell_flags & 2).bool().cpu().numpy()
        self._set_flags(fixed, values, src)
        self.apply_fixed_to_T()

    def set_source(self, mask, rate, t_cap):
        """heat.py:194-196"""
        fixed = (self.cell_flags & 1).bool().cpu().numpy()
        self._set_flags(fixed, self.tfix.cpu().numpy(), mask)
        self.rate, self.t_cap = float(rate), float(t_cap)
        self.fill_record()
        self.dirty = True

    def set_statics(self, alpha, k_faces, m_faces):
        """New static obstacle fields (grid.py:198-200), copied into the scene's static buffers.  A scene built without
        statics gets buffers now (its record changes: the plan is uploaded again before its next launch).  The caller
        rebuilds the obstacle fields (ScenePlan.prepare_statics)."""
        dev = self.device
        up = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device=dev)
        if self.st_alpha is None:
            self.st_alpha, self.st_k, self.st_m = up(alpha), [up(a) for a in k_faces], [up(a) for a in m_faces]
            if self.spec.n_particles == 0:    # air-only scenes use the statics as their obstacle fields
                self.alpha_s, self.k, self.m = self.st_alpha, list(self.st_k), list(self.st_m)
            self.fill_record()
            self.dirty = True
            return
        self.st_alpha.copy_(up(alpha))
        for dst, a in zip(list(self.st_k) + list(self.st_m), list(k_faces) + list(m_faces)):
            dst.copy_(up(a))

    def apply_fixed_to_T(self):
        T = self.T[self.parity()]
        f = (self.cell_flags & 1).bool()
        T[f] = self.tfix[f]

    def fill_record(self):
        s, sp, r = self, self.spec, self.record
        r.n, r.n_particles = s.n, sp.n_particles
        flags = _lib.HF_FLAG_ACTIVE
        if sp.buoyancy:
            flags |= _lib.HF_FLAG_BUOYANCY
        if self.rate > 0:
            flags |= _lib.HF_FLAG_SOURCE
        if sp.n_particles > 0:
            flags |= _lib.HF_FLAG_PARTICLES
        if sp.defect_correction:
            flags |= _lib.HF_FLAG_DEFECT_CORRECTION
        r.flags = flags
        r.cg_max_iter, r.heat_maxiter = sp.cg_max_iter, sp.heat_maxiter
        vals = dict(h=sp.h, rho=sp.rho, t_amb=sp.t_amb, alpha_f_min=sp.alpha_f_min, g=sp.g, cg_tol=sp.cg_tol,
                    heat_tol=sp.heat_tol, kappa_air=sp.kappa_air, kappa_mat=sp.kappa_mat, rate=self.rate, t_cap=self.t_cap,
                    vol=sp.spacing ** 3, k_particle=sp.k_particle, t_sol=sp.t_sol, t_liq=sp.t_liq, y_solid=sp.y_solid,
                    mu_s=sp.mu_s, mu_l=sp.mu_l, t_max=sp.t_max)
        for k, v in vals.items():
            setattr(r, k, float(v))
        P = _lib.ptr
        r.T[0], r.T[1] = P(s.T[0]), P(s.T[1])
        for i in range(2):
            r.u[i], r.v[i], r.w[i] = P(s.u[i]), P(s.v[i]), P(s.w[i])
        for name in ("Tw", "kap", "hrhs", "hdiag", "tfix", "alpha", "tsum", "cell_flags", "p", "rhs", "pdiag", "alpha_s",
                     "ax", "ay", "az", "cg_r", "cg_z", "cg_Ap"):
            setattr(r, name, P(getattr(s, name)))
        r.qx, r.qy, r.qz = (P(a) for a in s.q)
        r.kx, r.ky, r.kz = (P(a) for a in s.k)
        r.mx, r.my, r.mz = (P(a) for a in s.m)
        r.st_alpha = P(s.st_alpha)
        r.st_kx, r.st_ky, r.st_kz = (P(a) for a in s.st_k)
        r.st_mx, r.st_my, r.st_mz = (P(a) for a in s.st_m)
        r.cg_p[0], r.cg_p[1] = P(s.cg_p[0]), P(s.cg_p[1])
        r.pos, r.pvel, r.ptemp, r.pmelt, r.pyield, r.pvisc = (P(a) for a in (s.pos, s.pvel, s.ptemp, s.pmelt, s.pyield, s.pvisc))
        r.hkx, r.hky, r.hkz = (P(a) for a in s.hk)
        r.ayc, r.azc, r.hkzc = P(s.ayc), P(s.azc), P(s.hkzc)
        r.acc = P(s.acc)
        r.state = P(s.state)

    # --------------------------------------------------------------------------------------------- state
    def read_state(self) -> _lib.SceneState:
        buf = self.state.cpu().numpy().tobytes()
        st = _lib.SceneState.from_buffer_copy(buf)
        self._parity_host = int(st.parity)
        return st

    def parity(self) -> int:
        return self.read_state().parity

    def current(self, name):
        """The current buffer of a double-buffered field: T, u, v or w."""
        return getattr(self, name)[self.parity()]

    def set_current(self, name, value):
        self.current(name).copy_(torch.as_tensor(np.asarray(value, np.float32), device=self.device))


class ScenePlan:
    """Scene table + work table + workspace for a list of DeviceScene, and the stage calls over them."""

    def __init__(self, scenes, device="cuda:0", persistent_blocks=0, streaming_cg=False, tma=True, group_cells=0,
                 lanes=0):
        self.L = _lib.load()
        self.scenes = list(scenes)
        self.device = torch.device(device)
        S = len(self.scenes)
        self.host = (_lib.Scene * S)()
        for i, sc in enumerate(self.scenes):
            self.host[i] = sc.record
        C_total = sum(self.L.hf_chunks_for(sc.n) for sc in self.scenes)
        T_total = sum(self.L.hf_tiles_for(sc.n) for sc in self.scenes)
        self.scenes_dev = torch.zeros(C.sizeof(_lib.Scene) * S, dtype=torch.uint8, device=self.device)
        self.work_dev = torch.zeros(2 * max(C_total, 1), dtype=torch.int32, device=self.device)
        self.tiles_dev = torch.zeros(4 * max(T_total, 1), dtype=torch.int32, device=self.device)
        ws_bytes = self.L.hf_workspace_bytes(S, C_total, T_total)
        self.workspace = torch.zeros(ws_bytes, dtype=torch.uint8, device=self.device)
        self.plan = _lib.Plan()
        self.plan.num_scenes = S
        self.plan.scenes_host = C.cast(self.host, C.c_void_p)
        self.plan.scenes_dev = self.scenes_dev.data_ptr()
        self.plan.work_dev = self.work_dev.data_ptr()
        self.plan.tiles_dev = self.tiles_dev.data_ptr()
        self.plan.workspace = self.workspace.data_ptr()
        self.plan.workspace_bytes = ws_bytes
        self.plan.persistent_blocks = persistent_blocks
        self.plan.group_cells = group_cells
        self.plan.options = (_lib.HF_PLAN_STREAMING_CG if streaming_cg else 0) | (0 if tma else _lib.HF_PLAN_NO_TMA)
        self.lanes = lanes
        self.upload()

    @property
    def lanes(self):
        """Lanes of the streaming CG launch: independent scene groups solved side by side (0 or 1: one lane)."""
        return (self.plan.options >> _lib.HF_PLAN_LANES_SHIFT) & 15

    @lanes.setter
    def lanes(self, k):
        if not 0 <= int(k) <= 8:
            raise ValueError("lanes must be 0..8")
        self.plan.options = (self.plan.options & ~(15 << _lib.HF_PLAN_LANES_SHIFT)) | (int(k) << _lib.HF_PLAN_LANES_SHIFT)

    @property
    def resident_tiles(self):
        """Tiles per 256-thread group of the single-scene resident CG variant (0: the fewest that fit)."""
        return (self.plan.options >> _lib.HF_PLAN_RES_TILES_SHIFT) & 3

    @resident_tiles.setter
    def resident_tiles(self, m):
        if not 0 <= int(m) <= 3:
            raise ValueError("resident_tiles must be 0..3")
        self.plan.options = (self.plan.options & ~(3 << _lib.HF_PLAN_RES_TILES_SHIFT)) | (int(m) << _lib.HF_PLAN_RES_TILES_SHIFT)

    @property
    def single_reduction_cg(self):
        """Pressure solve of a single-scene plan (n % 4 == 0) with one grid barrier per CG iteration: the classic
        vector recurrences, beta from the expansion of the next r.z in the iteration's partials, the classic stopping
        test; results within ~1e-6 relative of the classic method.  Off by default."""
        return bool(self.plan.options & _lib.HF_PLAN_SINGLE_REDUCTION_CG)

    @single_reduction_cg.setter
    def single_reduction_cg(self, on):
        if on:
            self.plan.options |= _lib.HF_PLAN_SINGLE_REDUCTION_CG
        else:
            self.plan.options &= ~_lib.HF_PLAN_SINGLE_REDUCTION_CG

    def stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def upload(self):
        for i, sc in enumerate(self.scenes):
            sc.fill_record()
            self.host[i] = sc.record
        _lib.check(self.L.hf_plan_upload(C.byref(self.plan), self.stream()), "hf_plan_upload")

    def _call(self, name, *args):
        if any(sc.dirty for sc in self.scenes):
            self.upload()
            for sc in self.scenes:
                sc.dirty = False
        _lib.check(getattr(self.L, name)(C.byref(self.plan), *args, self.stream()), name)

    def prepare_statics(self):
        """Fill every scene's obstacle fields, face fractions and conductivity once (air-only scenes keep them)."""
        self._call("hf_obstacle_fields", 1)

    def substep(self, dt):
        self._call("hf_substep", float(dt))

    def obstacle_fields(self):
        self._call("hf_obstacle_fields", 0)

    def temperature_stage(self, dt):
        self._call("hf_temperature_stage", float(dt))

    def heat_solve(self, dt):
        self._call("hf_heat_solve", float(dt))

    def particle_update(self):
        self._call("hf_particle_update")

    def face_stage(self, dt):
        self._call("hf_face_stage", float(dt))

    def pressure_solve(self, dt):
        self._call("hf_pressure_solve", float(dt))

    def divergence_stage(self, dt):
        self._call("hf_divergence_stage", float(dt))

    def pressure_cg(self, dt):
        self._call("hf_pressure_cg", float(dt))

    def cell_velocity(self, s=0):
        sc = self.scenes[s]
        out = torch.empty((sc.n ** 3, 3), dtype=F32, device=self.device)
        _lib.check(self.L.hf_cell_velocity(C.byref(self.plan), s, out.data_ptr(), self.stream()), "hf_cell_velocity")
        return out

    def divergence_max(self, s=0):
        out = torch.zeros(1, dtype=F32, device=self.device)
        _lib.check(self.L.hf_divergence_max(C.byref(self.plan), s, out.data_ptr(), self.stream()), "hf_divergence_max")
        return float(out.item()) * self.scenes[s].spec.h

    def speed_max(self, s=0):
        out = torch.zeros(1, dtype=F32, device=self.device)
        _lib.check(self.L.hf_speed_max(C.byref(self.plan), s, out.data_ptr(), self.stream()), "hf_speed_max")
        return float(out.item())

"""ctypes front end of the CPU oracle (hf_oracle.c).  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use this module, as the checker and
the timed CPU baseline; the product never imports it.

``OracleScene`` holds one air scene in the reference layout (cells (n,n,n); u (n+1,n,n); v (n,n+1,n); w (n,n,n+1))
as numpy arrays and advances it with ``or_substep`` (solver.py:63-88 of the reference).  ``precision`` selects the
fp32 mirror (``"f32"``) or the all-FP64 oracle (``"f64"``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
_LIBS = {}


def build(force: bool = False) -> None:
    """Compile liboracle_f32.so / liboracle_f64.so with the Makefile beside this file."""
    libs = [os.path.join(BUILD, f"liboracle_{p}.so") for p in ("f32", "f64")]
    src = os.path.join(HERE, "hf_oracle.c")
    if not force and all(os.path.exists(l) and os.path.getmtime(l) >= os.path.getmtime(src) for l in libs):
        return
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_P = C.c_void_p


class _Scene(C.Structure):
    _fields_ = [("n", C.c_int32), ("n_particles", C.c_int32),
                ("cg_max_iter", C.c_int32), ("buoyancy", C.c_int32), ("heat_maxiter", C.c_int32),
                ("heat_check_every", C.c_int32), ("grid_check_every", C.c_int32), ("mean_mode", C.c_int32),
                ("scatter_mode", C.c_int32), ("pad0", C.c_int32)] + \
               [(f, C.c_double) for f in ("h", "rho", "t_amb", "alpha_f_min", "cg_tol", "kappa_air", "kappa_mat", "rate",
                                          "t_cap", "g", "heat_tol", "vol", "k_particle", "t_sol", "t_liq", "y_solid",
                                          "mu_s", "mu_l", "t_max")] + \
               [(f, _P) for f in ("u", "v", "w", "su", "sv", "sw", "ax", "ay", "az", "qx", "qy", "qz", "kx", "ky", "kz",
                                  "mx", "my", "mz", "p", "rhs", "alpha_s", "diag", "st_alpha", "st_kx", "st_ky", "st_kz",
                                  "st_mx", "st_my", "st_mz", "T", "T2", "Tw", "kap", "alpha", "tsum", "tfix", "hrhs",
                                  "hdiag", "fixed", "src", "pos", "pvel", "ptemp", "pmelt", "pyield", "pvisc", "cg_r",
                                  "cg_z", "cg_p", "cg_Ap", "acc")] + \
               [("heat_iters", C.c_int32), ("grid_iters", C.c_int32), ("heat_done", C.c_int32), ("grid_done", C.c_int32)] + \
               [(f, C.c_double) for f in ("heat_res", "grid_res", "heat_atol", "grid_atol", "mean")]


def lib(precision: str = "f32"):
    if precision not in _LIBS:
        build()
        L = C.CDLL(os.path.join(BUILD, f"liboracle_{precision}.so"))
        L.or_substep.argtypes = [C.POINTER(_Scene), C.c_double]
        L.or_dot.restype = C.c_double
        L.or_dot.argtypes = [_P, _P, C.c_size_t]
        L.or_mean.restype = C.c_double
        L.or_mean.argtypes = [_P, C.c_size_t, C.c_int]
        L.or_num_threads.restype = C.c_int
        L.or_pcg_pressure.restype = C.c_double
        L.or_pcg_pressure.argtypes = [C.POINTER(_Scene), C.c_double, C.c_int, C.c_int, _P]
        _LIBS[precision] = L
    return _LIBS[precision]


def set_threads(t: int) -> None:
    for p in ("f32", "f64"):
        lib(p).or_set_threads(int(t))


def num_threads() -> int:
    return int(lib("f32").or_num_threads())


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def face_shapes(n):
    return [(n + 1, n, n), (n, n + 1, n), (n, n, n + 1)]


class Kernels:
    """One-call wrappers of the per-kernel oracle functions (arrays are numpy, float params are Python floats)."""

    def __init__(self, precision="f32"):
        self.L = lib(precision)
        self.dt = np.float32 if precision == "f32" else np.float64

    def _a(self, a, dtype=None):
        return np.ascontiguousarray(a, dtype=dtype or self.dt)

    def call(self, name, *args):
        conv = []
        for a in args:
            if isinstance(a, np.ndarray):
                conv.append(_ptr(a))
            elif isinstance(a, float):
                conv.append(C.c_double(a))
            else:
                conv.append(C.c_int(int(a)))
        getattr(self.L, name)(*conv)


class OracleScene:
    """One air scene on the CPU (see module docstring)."""

    FIELDS_CELL = ("p", "rhs", "alpha_s", "diag", "T", "T2", "Tw", "kap", "alpha", "tsum", "tfix", "hrhs", "hdiag",
                   "cg_r", "cg_z", "cg_p", "cg_Ap", "st_alpha")

    def __init__(self, n, h, *, precision="f32", rho=1.2, t_amb=25.0, alpha_f_min=0.05, cg_tol=1e-4, cg_max_iter=400,
                 buoyancy=True, kappa_air=2.2e-5, kappa_mat=2.0e-5, g=9.81, heat_tol=1e-6, heat_maxiter=200,
                 heat_check_every=10, grid_check_every=20, mean_mode=0, scatter_mode=0, fixed=None, tfix=None, src=None,
                 rate=0.0, t_cap=0.0, static_alpha=None, static_k=None, static_m=None, particles=None, pvel=None,
                 ptemp=None, spacing=2.5e-3, k_particle=1.0e-3, t_sol=30.0, t_liq=36.0, y_solid=2.0e4, mu_s=5.0,
                 mu_l=30.0, t_max=300.0, t_init_grid=None):
        self.precision = precision
        self.L = lib(precision)
        dt = self.dtype = np.float32 if precision == "f32" else np.float64
        self.n = n
        N = (n, n, n)
        fs = face_shapes(n)
        z = lambda s: np.zeros(s, dt)
        self.a = {}
        for i, nm in enumerate(("u", "v", "w")):
            self.a[nm] = z(fs[i])
            self.a["s" + nm] = z(fs[i])
        for i, ax in enumerate("xyz"):
            for pre in ("a", "q", "k", "m"):
                self.a[pre + ax] = z(fs[i])
            self.a["st_k" + ax] = z(fs[i]) if static_k is None else np.array(static_k[i], dt, order="C")
            self.a["st_m" + ax] = z(fs[i]) if static_m is None else np.array(static_m[i], dt, order="C")
        for nm in self.FIELDS_CELL:
            self.a[nm] = z(N)
        if static_alpha is not None:
            self.a["st_alpha"] = np.array(static_alpha, dt, order="C")
        self.a["fixed"] = np.zeros(N, np.int32) if fixed is None else np.ascontiguousarray(fixed, np.int32)
        self.a["src"] = np.zeros(N, np.int32) if src is None else np.ascontiguousarray(src, np.int32)
        if tfix is not None:
            self.a["tfix"] = np.array(tfix, dt, order="C")
        for nm in ("T", "T2", "Tw"):
            self.a[nm][...] = t_amb if t_init_grid is None else t_init_grid
        P = 0 if particles is None else len(particles)
        self.P = P
        self.a["pos"] = np.ascontiguousarray(np.zeros((max(P, 1), 3)) if particles is None else particles, dt)
        self.a["pvel"] = np.ascontiguousarray(np.zeros((max(P, 1), 3)) if pvel is None else pvel, dt)
        self.a["ptemp"] = np.ascontiguousarray(np.full(max(P, 1), 20.0) if ptemp is None else ptemp, dt)
        for nm in ("pmelt", "pyield", "pvisc"):
            self.a[nm] = z(max(P, 1))
        self.a["acc"] = np.zeros(12 * (n + 1) ** 3, np.int64) if P else None
        s = self.s = _Scene()
        s.n, s.n_particles = n, P
        s.cg_max_iter, s.buoyancy, s.heat_maxiter = cg_max_iter, int(bool(buoyancy)), heat_maxiter
        s.heat_check_every, s.grid_check_every, s.mean_mode, s.scatter_mode = heat_check_every, grid_check_every, mean_mode, scatter_mode
        s.h, s.rho, s.t_amb, s.alpha_f_min, s.cg_tol = h, rho, t_amb, alpha_f_min, cg_tol
        s.kappa_air, s.kappa_mat, s.rate, s.t_cap, s.g, s.heat_tol = kappa_air, kappa_mat, rate, t_cap, g, heat_tol
        s.vol, s.k_particle, s.t_sol, s.t_liq = spacing ** 3, k_particle, t_sol, t_liq
        s.y_solid, s.mu_s, s.mu_l, s.t_max = y_solid, mu_s, mu_l, t_max
        self._bind()
        if static_alpha is None and static_k is None and static_m is None:
            s.st_alpha = None
        # set_fixed applies the fixed values to T immediately (heat.py:189-192)
        f = self.a["fixed"] == 1
        self.a["T"][f] = self.a["tfix"][f]

    def _bind(self):
        for nm, arr in self.a.items():
            setattr(self.s, nm, _ptr(arr) if arr is not None else None)
        self._by_addr = {arr.ctypes.data: arr for arr in self.a.values() if arr is not None}

    def cur(self, name):
        """Current array behind a (possibly swapped) pointer field of the scene struct."""
        return self._by_addr[getattr(self.s, name)]

    @property
    def T(self):
        return self.cur("T")

    @property
    def u(self):
        return self.cur("u")

    @property
    def v(self):
        return self.cur("v")

    @property
    def w(self):
        return self.cur("w")

    @property
    def p(self):
        return self.a["p"]

    def set_state(self, T=None, u=None, v=None, w=None):
        for nm, val in (("T", T), ("u", u), ("v", v), ("w", w)):
            if val is not None:
                self.cur(nm)[...] = val

    def substep(self, dt):
        self.L.or_substep(C.byref(self.s), C.c_double(dt))

    def stats(self):
        s = self.s
        return dict(heat_iters=s.heat_iters, grid_iters=s.grid_iters, heat_done=s.heat_done, grid_done=s.grid_done,
                    heat_res=s.heat_res, grid_res=s.grid_res, heat_atol=s.heat_atol, grid_atol=s.grid_atol, mean=s.mean)

    def cell_velocity(self):
        out = np.zeros((self.n ** 3, 3), self.dtype)
        self.L.or_cell_velocity(C.c_int(self.n), _ptr(self.u), _ptr(self.v), _ptr(self.w), _ptr(out))
        return out

    def divergence_max(self):
        """grid.py:257-260: max |div| * h with scale 1."""
        n = self.n
        rhs = np.zeros((n, n, n), self.dtype)
        A = self.a
        self.L.or_divergence_rhs(C.c_int(n), C.c_double(self.s.h), C.c_double(1.0), _ptr(self.u), _ptr(self.v),
                                 _ptr(self.w), _ptr(A["ax"]), _ptr(A["ay"]), _ptr(A["az"]), _ptr(A["qx"]), _ptr(A["qy"]),
                                 _ptr(A["qz"]), _ptr(rhs))
        return float(np.abs(rhs).max()) * self.s.h

    def speed_max(self):
        return max(float(np.abs(a).max()) for a in (self.u, self.v, self.w))

    def particles(self):
        P = self.P
        return dict(temp=self.a["ptemp"][:P], melt=self.a["pmelt"][:P], yield_stress=self.a["pyield"][:P],
                    viscosity=self.a["pvisc"][:P])


def scene_from_spec(spec, precision="f32", mean_mode=0, scatter_mode=0, particles=None, pvel=None, ptemp=None):
    """OracleScene with the parameters of a heatflow_mpm SceneSpec (any object with the same attribute names)."""
    return OracleScene(spec.n, spec.h, precision=precision, rho=spec.rho, t_amb=spec.t_amb, alpha_f_min=spec.alpha_f_min,
                       cg_tol=spec.cg_tol, cg_max_iter=spec.cg_max_iter, buoyancy=spec.buoyancy, kappa_air=spec.kappa_air,
                       kappa_mat=spec.kappa_mat, g=spec.g, heat_tol=spec.heat_tol, heat_maxiter=spec.heat_maxiter,
                       mean_mode=mean_mode, scatter_mode=scatter_mode, fixed=spec.fixed, tfix=spec.tfix, src=spec.source,
                       rate=spec.rate, t_cap=spec.t_cap, static_alpha=spec.static_alpha, static_k=spec.static_k,
                       static_m=spec.static_m, particles=particles, pvel=pvel, ptemp=ptemp, spacing=spec.spacing,
                       k_particle=spec.k_particle, t_sol=spec.t_sol, t_liq=spec.t_liq, y_solid=spec.y_solid,
                       mu_s=spec.mu_s, mu_l=spec.mu_l, t_max=spec.t_max)


def scene_from_fixture(fx, precision="f32", mean_mode=1, scatter_mode=1):
    """Build an OracleScene from a tests/golden/substep_*.npz fixture (the reference's own inputs)."""
    n = int(fx["n"])
    P = fx["in_pos"].shape[0] if "in_pos" in fx else 0
    sc = OracleScene(n, float(fx["h"]), precision=precision, rho=float(fx["rho"]), t_amb=float(fx["t_amb"]),
                     alpha_f_min=float(fx["alpha_f_min"]), cg_tol=float(fx["cg_tol"]), cg_max_iter=int(fx["cg_max_iter"]),
                     buoyancy=bool(fx["buoyancy"]), kappa_air=float(fx["kappa_air"]), kappa_mat=float(fx["kappa_mat"]),
                     mean_mode=mean_mode, scatter_mode=scatter_mode, fixed=fx["fixed"], tfix=fx["tfix"], src=fx["src"],
                     rate=float(fx["rate"]), t_cap=float(fx["t_cap"]), static_alpha=fx["static_alpha"],
                     static_k=[fx[f"static_k{a}"] for a in range(3)], static_m=[fx[f"static_m{a}"] for a in range(3)],
                     particles=fx["in_pos"] if P else None, pvel=fx["in_pvel"] if P else None,
                     ptemp=fx["in_ptemp"] if P else None, spacing=float(fx["spacing"]), t_sol=float(fx["t_sol"]),
                     t_liq=float(fx["t_liq"]), y_solid=float(fx["yield_solid"]), mu_s=float(fx["mu_s"]),
                     mu_l=float(fx["mu_l"]), t_max=float(fx["t_max"]))
    sc.set_state(T=fx["in_T"], u=fx["in_u"], v=fx["in_v"], w=fx["in_w"])
    return sc

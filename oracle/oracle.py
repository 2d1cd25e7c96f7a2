"""ctypes bindings of the C restatement (`ivp_oracle.c`) -- test infrastructure.

Arrays are NumPy, in the reference's layout and particle order.  The helpers
here mirror the reference's call sequence (`Framework.initialize`,
framework.py:282-290; `IP.solve`, ip.py:331-404; `Framework.forward`,
framework.py:423-544) so tests read like driving the reference.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libivp_oracle.so")
_lib = None

OK, NOT_SPD, NOT_CONVERGED = 0, 1, 2


class Params(ctypes.Structure):
    _fields_ = [
        ("h", ctypes.c_float),
        ("cache_size", ctypes.c_int),
        ("omega", ctypes.c_float),
        ("tol_pcg", ctypes.c_double),
        ("tol_opt", ctypes.c_double),
        ("max_outer", ctypes.c_int),
        ("max_pcg", ctypes.c_int),
        ("fixed_iters", ctypes.c_int),
        ("fast", ctypes.c_int),
    ]


class ViscParams(ctypes.Structure):
    _fields_ = [
        ("visc", ctypes.c_float),
        ("dt", ctypes.c_float),
        ("h", ctypes.c_float),
        ("cache", ctypes.c_int),
        ("max_iter", ctypes.c_int),
        ("tol", ctypes.c_double),
        ("fast", ctypes.c_int),
    ]


class StParams(ctypes.Structure):
    _fields_ = [
        ("sigma", ctypes.c_float),
        ("dt", ctypes.c_float),
        ("d", ctypes.c_float),
        ("h_st", ctypes.c_float),
        ("cache", ctypes.c_int),
        ("max_iter", ctypes.c_int),
        ("tol", ctypes.c_double),
        ("fast", ctypes.c_int),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("outer_iters", ctypes.c_int),
        ("n_err", ctypes.c_int),
        ("final_err", ctypes.c_double),
        ("status", ctypes.c_int),
    ]


def build(force: bool = False) -> str:
    """Compile the restatement with its Makefile (gcc, OpenMP)."""
    src = os.path.join(_HERE, "ivp_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        i, f, d, l = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_long
        L.orc_cubic_kernel.argtypes = [f, f]
        L.orc_cubic_kernel.restype = f
        L.orc_spiky_grad.argtypes = [P, f, P]
        L.orc_build_neighbor_cache.argtypes = [i, P, P, i, f, i, P, P, P, P]
        L.orc_build_neighbor_cache.restype = l
        L.orc_compute_density.argtypes = [i, P, P, P, f, i, P, P, P]
        L.orc_compute_aii.argtypes = [i, P, P, P, i, P, P, P, P]
        L.orc_ip_solve.argtypes = [i, ctypes.POINTER(Params), f, P, P, P, P, P, P, P, P, P, P, P, P, P,
                                   ctypes.POINTER(Stats)]
        L.orc_ip_solve.restype = i
        L.orc_apply_gravity.argtypes = [i, P, P, P, f]
        L.orc_advect_and_clamp.argtypes = [i, P, P, P, f, P, f]
        L.orc_step.argtypes = [i, ctypes.POINTER(Params), f, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P,
                               ctypes.POINTER(Stats), ctypes.POINTER(l), P, f, P, f, P, i]
        L.orc_weiler18_solve.argtypes = [i, ctypes.POINTER(ViscParams), P, P, P, P, P, P, P, P, P, P]
        L.orc_weiler18_solve.restype = i
        L.orc_jeske23_solve.argtypes = [i, ctypes.POINTER(StParams), P, P, P, P, P, P, P, P, P, P, P]
        L.orc_jeske23_solve.restype = i
        L.orc_prj_solve.argtypes = [i, ctypes.POINTER(Params), f, P, P, P, P, P, P, P, P, P, P,
                                    ctypes.POINTER(Stats)]
        L.orc_prj_solve.restype = i
        L.orc_step.restype = i
        L.orc_cg_f64.argtypes = [i, f, i, P, P, P, P, P, P, P, P, d, i, P]
        L.orc_cg_f64.restype = i
        L.orc_ip_system.argtypes = [i, f, i, P, P, P, P, P, P, P, P, P, P, P, P]
        L.orc_apply_A_f64.argtypes = [i, f, i, P, P, P, P, P, P, P, P, P]
        L.orc_num_threads.restype = i
        L.orc_set_num_threads.argtypes = [i]
        _lib = L
    return _lib


def _p(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def num_threads() -> int:
    return int(lib().orc_num_threads())


def set_num_threads(t: int) -> None:
    lib().orc_set_num_threads(int(t))


def cubic_kernel(r: float, h: float) -> float:
    return float(lib().orc_cubic_kernel(float(r), float(h)))


def spiky_grad(r, h: float) -> np.ndarray:
    r = _f32(r)
    out = np.zeros(3, np.float32)
    lib().orc_spiky_grad(_p(r), float(h), _p(out))
    return out


@dataclasses.dataclass
class State:
    """Reference-layout state of one scene (SimulationData + solver buffers)."""

    x: np.ndarray
    v: np.ndarray
    m: np.ndarray
    m_inv: np.ndarray
    is_dynamic: np.ndarray
    density0: np.ndarray
    h: float
    cache_size: int
    domain_size: np.ndarray
    gravity: np.ndarray
    dt: float
    omega: float = 10.0
    tol_pcg: float = 1e-6
    tol_opt: float = 1e-3
    max_outer: int = 1000
    max_pcg: int = 1000
    fixed_iters: bool = False
    material: Optional[np.ndarray] = None
    viscosity: float = 0.0        # Weiler18 kinematic viscosity (0 = off)
    visc_iters: int = 0
    surface_tension: float = 0.0  # Jeske23 sigma (0 = off)
    st_iters: int = 0
    pressure_method: int = 1      # pressureMethod: 1 IP, 0 PRJ
    count: Optional[np.ndarray] = None
    ids: Optional[np.ndarray] = None
    gradW: Optional[np.ndarray] = None
    density: Optional[np.ndarray] = None
    k: Optional[np.ndarray] = None
    overflow: int = 0
    # stats of the last solve (names follow pressure_base.py:331-339)
    stats_density_errors: list = dataclasses.field(default_factory=list)
    stats_pcg_iters: list = dataclasses.field(default_factory=list)
    stats_outer_iters: int = 0
    stats_final_density_error: float = 0.0
    status: int = OK

    @classmethod
    def from_scene(cls, sc, **over) -> "State":
        m, m_inv = sc.masses()
        kw = dict(x=_f32(sc.x).copy(), v=_f32(sc.v).copy(), m=m, m_inv=m_inv,
                  is_dynamic=_i32(sc.is_dynamic), density0=_f32(sc.density0), h=sc.support_radius,
                  cache_size=sc.cache_size, domain_size=_f32(sc.domain_size),
                  gravity=_f32(sc.gravity), dt=sc.dt, omega=sc.omega, tol_pcg=sc.tol_pcg,
                  tol_opt=sc.density_error_tol, max_outer=sc.max_outer_iters,
                  max_pcg=sc.max_iteration_pcg, fixed_iters=sc.fixed_outer_iters,
                  material=_i32(sc.material),
                  viscosity=float(sc.viscosity_coeff) if int(sc.viscosity_method) == 1 else 0.0,
                  surface_tension=float(sc.surface_tension_coeff) if int(sc.surface_tension_method) == 1 else 0.0,
                  pressure_method=int(getattr(sc, "pressure_method", 1)))
        kw.update(over)
        return cls(**kw)

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    def params(self, fast: bool) -> Params:
        return Params(h=self.h, cache_size=self.cache_size, omega=self.omega, tol_pcg=self.tol_pcg,
                      tol_opt=self.tol_opt, max_outer=self.max_outer, max_pcg=self.max_pcg,
                      fixed_iters=int(self.fixed_iters), fast=int(fast))

    # --- Framework._rebuild_neighbors_and_density (framework.py:282-290)
    def rebuild(self, only_dynamic: bool = True) -> None:
        n, c = self.n, self.cache_size
        self.count = np.zeros(n, np.int32)
        self.ids = np.zeros(n * c, np.int32)
        self.gradW = np.zeros((n * c, 3), np.float32)
        if self.density is None:
            self.density = self.density0.copy()
        if self.k is None:
            self.k = np.zeros(n, np.float32)
        L = lib()
        self.overflow = int(L.orc_build_neighbor_cache(n, _p(self.x), _p(self.is_dynamic), int(only_dynamic),
                                                       self.h, c, _p(_f32(self.domain_size)), _p(self.count),
                                                       _p(self.ids), _p(self.gradW)))
        L.orc_compute_density(n, _p(self.x), _p(self.m), _p(self.is_dynamic), self.h, c, _p(self.count),
                              _p(self.ids), _p(self.density))
        L.orc_compute_aii(n, _p(self.m), _p(self.m_inv), _p(self.is_dynamic), c, _p(self.count), _p(self.ids),
                          _p(self.gradW), _p(self.k))

    def neighbour_sets(self, i: int) -> set:
        cnt = min(int(self.count[i]), self.cache_size)
        return set(int(j) for j in self.ids[i * self.cache_size: i * self.cache_size + cnt])

    # --- IP.solve (ip.py:331-404)
    def solve(self, fast: bool = True, divergence: bool = False, return_d: bool = False):
        n = self.n
        P = self.params(fast)
        err = np.zeros(self.max_outer + 1, np.float64)
        pcg = np.zeros(max(self.max_outer, 1), np.int32)
        div = np.zeros(n, np.float32) if divergence else None
        d = np.zeros((n, 3), np.float32) if return_d else None
        st = Stats()
        status = lib().orc_ip_solve(n, ctypes.byref(P), float(self.dt), _p(self.density), _p(self.density0),
                                    _p(self.m), _p(self.is_dynamic), _p(self.count), _p(self.ids), _p(self.gradW),
                                    _p(self.k), _p(self.v), _p(err), _p(pcg), _p(div), _p(d), ctypes.byref(st))
        self._record(st, err, pcg)
        self.status = int(status)
        return d if return_d else div

    def _record(self, st: Stats, err, pcg):
        ne = min(st.n_err, self.max_outer + 1)
        self.stats_density_errors = [float(e) for e in err[:ne]]
        self.stats_pcg_iters = [int(q) for q in pcg[:min(st.outer_iters, len(pcg))]]
        self.stats_outer_iters = int(st.outer_iters)
        self.stats_final_density_error = float(st.final_err)

    # --- Framework.forward with IP only (framework.py:423-544)
    def step(self, fast: bool = True) -> int:
        n = self.n
        P = self.params(fast)
        err = np.zeros(self.max_outer + 1, np.float64)
        pcg = np.zeros(max(self.max_outer, 1), np.int32)
        st = Stats()
        ov = ctypes.c_long(0)
        vit = ctypes.c_int(0)
        sit = ctypes.c_int(0)
        status = lib().orc_step(n, ctypes.byref(P), float(self.dt), _p(self.gravity), _p(self.domain_size),
                                _p(self.x), _p(self.v), _p(self.density0), _p(self.m), _p(self.m_inv),
                                _p(self.is_dynamic), _p(self.count), _p(self.ids), _p(self.gradW),
                                _p(self.density), _p(self.k), _p(err), _p(pcg), ctypes.byref(st), ctypes.byref(ov),
                                _p(self.material), float(self.viscosity), ctypes.byref(vit),
                                float(self.surface_tension), ctypes.byref(sit), int(self.pressure_method == 0))
        self.visc_iters = int(vit.value)
        self.st_iters = int(sit.value)
        self._record(st, err, pcg)
        self.overflow = int(ov.value)
        self.status = int(status)
        return int(status)

    # --- PRJ.solve (prj.py:296-340) on the current lists
    def prj_solve(self, fast: bool = True, omega: float = 0.5) -> int:
        n = self.n
        P = self.params(fast)
        P.omega = float(omega)
        err = np.zeros(self.max_outer + 2, np.float64)
        st = Stats()
        status = lib().orc_prj_solve(n, ctypes.byref(P), float(self.dt), _p(self.density), _p(self.density0),
                                     _p(self.m), _p(self.is_dynamic), _p(self.count), _p(self.ids), _p(self.gradW),
                                     _p(self.k), _p(self.v), _p(err), ctypes.byref(st))
        self._record(st, err, np.zeros(1, np.int32))
        self.stats_pcg_iters = []
        self.status = int(status)
        return int(status)

    # --- Weiler18.solve (weiler18.py:371-401) on the current lists
    def viscosity_solve(self, coeff: float, fast: bool = True) -> int:
        V = ViscParams(visc=float(coeff), dt=float(self.dt), h=self.h, cache=self.cache_size, max_iter=1000,
                       tol=1e-5, fast=int(fast))
        return int(lib().orc_weiler18_solve(self.n, ctypes.byref(V), _p(self.x), _p(self.v), _p(self.m),
                                            _p(self.density), _p(self.density0), _p(self.material),
                                            _p(self.is_dynamic), _p(self.count), _p(self.ids), _p(self.gradW)))

    # --- Jeske23.solve (jeske23.py:585-655) on the current lists
    def surface_tension_solve(self, sigma: float, fast: bool = True, particle_radius: Optional[float] = None):
        """Returns (CG iterations, div, b) of one Jeske23 solve (v updated)."""
        d = np.float32(2.0 * particle_radius) if particle_radius is not None else np.float32(0.5 * self.h)
        S = StParams(sigma=float(sigma), dt=float(self.dt), d=float(d), h_st=float(np.float32(2.0) * d),
                     cache=self.cache_size, max_iter=100, tol=1e-5, fast=int(fast))
        div = np.zeros(self.n, np.float32)
        b = np.zeros((self.n, 3), np.float32)
        it = lib().orc_jeske23_solve(self.n, ctypes.byref(S), _p(self.x), _p(self.v), _p(self.m), _p(self.density),
                                     _p(self.material), _p(self.is_dynamic), _p(self.count), _p(self.ids),
                                     _p(self.gradW), _p(div), _p(b))
        return int(it), div, b

    # --- one outer-iteration linear system and its FP64 solution
    def system(self, d: np.ndarray):
        n = self.n
        c = np.where(self.is_dynamic == 1, self.density - self.density0, 0).astype(np.float32)
        t = np.zeros(n, np.float32)
        f = np.zeros(n, np.float32)
        dfdt = np.zeros(n, np.float32)
        rhs = np.zeros((n, 3), np.float32)
        lib().orc_ip_system(n, self.omega, self.cache_size, _p(_f32(d)), _p(c), _p(self.m), _p(self.is_dynamic),
                            _p(self.count), _p(self.ids), _p(self.gradW), _p(self.k), _p(t), _p(f), _p(dfdt),
                            _p(rhs))
        return t, f, dfdt, rhs

    def cg_f64(self, dfdt, rhs, rel_tol=1e-13, max_iter=20000):
        x = np.zeros((self.n, 3), np.float64)
        it = lib().orc_cg_f64(self.n, self.omega, self.cache_size, _p(self.m), _p(_f32(dfdt)), _p(self.k),
                              _p(self.is_dynamic), _p(self.count), _p(self.ids), _p(self.gradW), _p(_f32(rhs)),
                              float(rel_tol), int(max_iter), _p(x))
        return x, int(it)

    def apply_A_f64(self, dfdt, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        out = np.zeros_like(p)
        lib().orc_apply_A_f64(self.n, self.omega, self.cache_size, _p(self.m), _p(_f32(dfdt)), _p(self.k),
                              _p(self.is_dynamic), _p(self.count), _p(self.ids), _p(self.gradW), _p(p), _p(out))
        return out


def advect_and_clamp(x, v, is_dynamic, dt, domain, padding):
    x = _f32(x).copy()
    v = _f32(v).copy()
    lib().orc_advect_and_clamp(x.shape[0], _p(x), _p(v), _p(_i32(is_dynamic)), float(dt), _p(_f32(domain)),
                               float(padding))
    return x, v

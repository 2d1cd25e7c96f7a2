"""Engine: the CUDA IP pressure step over one or more independent scenes.

PyTorch owns every device buffer (particle arrays and one workspace tensor);
`libivp.so` receives their pointers through the C ABI.  Scenes are
concatenated in the particle arrays (scene s owns a contiguous range), which
is how the batched and served forms run many scenes in one set of launches.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check


def _stream_ptr(stream: Optional[torch.cuda.Stream] = None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


@dataclasses.dataclass
class EngineOptions:
    lanes_per_particle: int = 0   # 0: chosen from the scenes (ivp_resolve_options)
    particles_per_block: int = 0  # 0: follows the lane count (256 threads per CTA)
    list_stride: int = 64
    max_hist: int = 128
    use_graphs: bool = True
    persistent: bool = True
    row_format: int = 0  # 0 default (full), 1 full {J, j}, 2 compact {j, w}, 3 bf16 gradients
    build_kernel: int = 0  # 1 thread per particle, 2 warp per cell; 0: chosen from the scenes

    def to_c(self) -> _lib.Options:
        o = _lib.Options()
        o.lanes_per_particle = self.lanes_per_particle
        o.particles_per_block = self.particles_per_block
        o.list_stride = self.list_stride
        o.max_hist = self.max_hist
        o.use_graphs = int(self.use_graphs)
        o.persistent = int(self.persistent)
        o.row_format = int(self.row_format)
        o.build_kernel = int(self.build_kernel)
        return o


def scene_desc(sc, offset: int) -> _lib.SceneDesc:
    """C descriptor of a `scenes.Scene` occupying particles [offset, offset+n)."""
    d = _lib.SceneDesc()
    d.particle_offset = offset
    d.n_particles = sc.n
    d.n_dynamic = sc.n_dynamic
    d.particle_radius = sc.particle_radius
    for a in range(3):
        d.domain_size[a] = float(sc.domain_size[a])
        d.gravity[a] = float(sc.gravity[a])
    d.dt = sc.dt
    d.omega = sc.omega
    d.tol_pcg = sc.tol_pcg
    d.density_error_tol = sc.density_error_tol
    d.max_outer_iters = sc.max_outer_iters
    d.max_iteration_pcg = sc.max_iteration_pcg
    d.fixed_outer_iters = int(sc.fixed_outer_iters)
    d.cache_size = sc.cache_size
    d.viscosity_coeff = sc.viscosity_coeff
    d.viscosity_method = sc.viscosity_method
    d.surface_tension_method = int(getattr(sc, "surface_tension_method", 0))
    d.surface_tension_coeff = float(getattr(sc, "surface_tension_coeff", 0.0))
    # pressureMethod (framework.py:168-174): 1 IP, 0 PRJ
    d.pressure_solver = 1 if int(getattr(sc, "pressure_method", 1)) == 0 else 0
    return d


def workspace_bytes(scenes: Sequence, options: Optional["EngineOptions"] = None) -> int:
    """Device workspace an Engine over `scenes` allocates (ivp_workspace_bytes)."""
    L = _lib.load()
    descs = (_lib.SceneDesc * len(scenes))()
    off = 0
    for i, sc in enumerate(scenes):
        descs[i] = scene_desc(sc, off)
        off += sc.n
    opt = (options or EngineOptions()).to_c()
    nbytes = ctypes.c_size_t(0)
    check(L.ivp_workspace_bytes(descs, len(scenes), ctypes.byref(opt), ctypes.byref(nbytes)), "ivp_workspace_bytes")
    return int(nbytes.value)


@dataclasses.dataclass
class Stats:
    """Per-scene result of the last IP solve (names of pressure_base.py:331-339)."""

    status: int
    stats_outer_iters: int
    stats_final_density_error: float
    stats_density_errors: list
    stats_pcg_iters: list
    overflow_particles: int
    total_pcg_iters: int
    last_pap: float = 0.0        # p^T A p of the last CG iteration (reported with NOT_SPD)
    last_cg_iter: int = 0        # CG iterations completed in the last PCG call


class Engine:
    """IP pressure-step engine over `scenes` (list of `scenes.Scene`).

    Particle arrays are allocated here in the reference's layout and scene
    order; pass `arrays=` to bind existing tensors instead (dict with x, v, m,
    density0, is_dynamic, material, density, k[, divergence]).
    """

    def __init__(self, scenes: Sequence, device: str = "cuda", options: Optional[EngineOptions] = None,
                 arrays: Optional[dict] = None, stream: Optional[torch.cuda.Stream] = None,
                 divergence: bool = False):
        self.L = _lib.load()
        self.scenes = list(scenes)
        self.device = torch.device(device)
        self.options = options or EngineOptions()
        self.offsets = np.zeros(len(self.scenes) + 1, np.int64)
        for i, sc in enumerate(self.scenes):
            self.offsets[i + 1] = self.offsets[i] + sc.n
        self.n_total = int(self.offsets[-1])
        descs = (_lib.SceneDesc * len(self.scenes))()
        for i, sc in enumerate(self.scenes):
            descs[i] = scene_desc(sc, int(self.offsets[i]))
        self._descs = descs
        opt = self.options.to_c()
        self._opt = opt
        res = _lib.Options()
        check(self.L.ivp_resolve_options(descs, len(self.scenes), ctypes.byref(opt), ctypes.byref(res)),
              "ivp_resolve_options")
        # the lane count and tile size the engine runs with
        self.lanes_per_particle = int(res.lanes_per_particle)
        self.particles_per_block = int(res.particles_per_block)
        self.build_kernel = int(res.build_kernel)
        nbytes = ctypes.c_size_t(0)
        check(self.L.ivp_workspace_bytes(descs, len(self.scenes), ctypes.byref(opt), ctypes.byref(nbytes)),
              "ivp_workspace_bytes")
        self.workspace_bytes = int(nbytes.value)
        # 256-byte aligned workspace carved from one uint8 tensor
        self._ws_raw = torch.empty(self.workspace_bytes + 256, dtype=torch.uint8, device=self.device)
        base = self._ws_raw.data_ptr()
        self._ws_ptr = (base + 255) & ~255
        if arrays is None:
            arrays = self._alloc_arrays(divergence)
        self.arrays = arrays
        self._handle = ctypes.c_void_p()
        st = _stream_ptr(stream)
        check(self.L.ivp_engine_create(descs, len(self.scenes), ctypes.byref(opt), ctypes.c_void_p(self._ws_ptr),
                                       ctypes.c_size_t(self.workspace_bytes), ctypes.c_void_p(st),
                                       ctypes.byref(self._handle)), "ivp_engine_create")
        self._bind()

    # ------------------------------------------------------------ arrays
    def _alloc_arrays(self, divergence: bool) -> dict:
        dev = self.device
        x = np.ascontiguousarray(np.concatenate([sc.x for sc in self.scenes]), dtype=np.float32)
        v = np.ascontiguousarray(np.concatenate([sc.v for sc in self.scenes]), dtype=np.float32)
        ms = [sc.masses() for sc in self.scenes]
        m = np.concatenate([a for a, _ in ms]).astype(np.float32)
        a = {
            "x": torch.from_numpy(x).to(dev),
            "v": torch.from_numpy(v).to(dev),
            "m": torch.from_numpy(m).to(dev),
            "density0": torch.from_numpy(np.concatenate([sc.density0 for sc in self.scenes])).to(dev),
            "is_dynamic": torch.from_numpy(np.concatenate([sc.is_dynamic for sc in self.scenes]).astype(np.int32)).to(dev),
            "material": torch.from_numpy(np.concatenate([sc.material for sc in self.scenes]).astype(np.int32)).to(dev),
        }
        a["density"] = a["density0"].clone()
        a["k"] = torch.zeros(self.n_total, dtype=torch.float32, device=dev)
        if divergence:
            a["divergence"] = torch.zeros(self.n_total, dtype=torch.float32, device=dev)
        return a

    def _bind(self):
        a = self.arrays
        for k in ("x", "v"):
            assert a[k].is_contiguous() and a[k].dtype == torch.float32 and a[k].shape[-1] == 3
        p = _lib.Particles()
        p.x = a["x"].data_ptr()
        p.v = a["v"].data_ptr()
        p.m = a["m"].data_ptr()
        p.density0 = a["density0"].data_ptr()
        p.is_dynamic = a["is_dynamic"].data_ptr()
        p.material = a["material"].data_ptr()
        p.density = a["density"].data_ptr()
        p.kdiag = a["k"].data_ptr()
        p.divergence = a["divergence"].data_ptr() if a.get("divergence") is not None else None
        p.n_total = self.n_total
        check(self.L.ivp_engine_bind(self._handle, ctypes.byref(p)), "ivp_engine_bind")

    def rebind(self, arrays: dict):
        self.arrays = arrays
        self._bind()

    def close(self):
        if getattr(self, "_handle", None) and self._handle.value:
            self.L.ivp_engine_destroy(self._handle)
            self._handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ calls
    def update_scene(self, i: int, sc, stream=None):
        d = scene_desc(sc, int(self.offsets[i]))
        check(self.L.ivp_update_scene(self._handle, i, ctypes.byref(d), ctypes.c_void_p(_stream_ptr(stream))),
              "ivp_update_scene")
        self._descs[i] = d

    def build(self, stream=None):
        """NeighbourSearch.build + build_cache + compute_density + compute_Aii."""
        check(self.L.ivp_neighbour_build(self._handle, ctypes.c_void_p(_stream_ptr(stream))), "ivp_neighbour_build")

    def compute_density(self, stream=None):
        check(self.L.ivp_compute_density(self._handle, ctypes.c_void_p(_stream_ptr(stream))), "ivp_compute_density")

    def compute_aii(self, stream=None):
        check(self.L.ivp_compute_aii(self._handle, ctypes.c_void_p(_stream_ptr(stream))), "ivp_compute_aii")

    def solve(self, stream=None):
        """IP.solve(dt) of every scene (asynchronous)."""
        check(self.L.ivp_ip_solve(self._handle, ctypes.c_void_p(_stream_ptr(stream))), "ivp_ip_solve")

    def viscosity_solve(self, stream=None):
        """Weiler18.solve(coeff, dt) of every scene with implicit viscosity."""
        check(self.L.ivp_viscosity_solve(self._handle, ctypes.c_void_p(_stream_ptr(stream))), "ivp_viscosity_solve")

    def prj_solve(self, stream=None):
        """PRJ.solve(dt) of every scene whose pressure method is PRJ (0)."""
        check(self.L.ivp_prj_solve(self._handle, ctypes.c_void_p(_stream_ptr(stream))), "ivp_prj_solve")

    def surface_tension_solve(self, stream=None):
        """Jeske23.solve(sigma, sigma, dt) of every scene with implicit surface tension."""
        check(self.L.ivp_surface_tension_solve(self._handle, ctypes.c_void_p(_stream_ptr(stream))),
              "ivp_surface_tension_solve")

    def apply_gravity(self, stream=None):
        check(self.L.ivp_apply_gravity(self._handle, ctypes.c_void_p(_stream_ptr(stream))), "ivp_apply_gravity")

    def advect(self, stream=None):
        check(self.L.ivp_advect(self._handle, ctypes.c_void_p(_stream_ptr(stream))), "ivp_advect")

    def step(self, n: int = 1, stream=None):
        """n Framework.forward() steps of every scene (asynchronous)."""
        check(self.L.ivp_step(self._handle, int(n), ctypes.c_void_p(_stream_ptr(stream))), "ivp_step")

    def step_io(self, x_in=None, v_in=None, x_out=None, v_out=None, first: int = 0, count=None, stream=None):
        """One step whose x and v of particles [first, first + count) come
        from and go back to page-locked host tensors (float32, (count, 3)),
        the copies overlapped with the step's kernels (ivp_step_io).  Inputs
        and outputs may be the same tensors.  Asynchronous: the outputs are
        complete once the stream has passed the step."""
        import torch
        n = self.n_total - first if count is None else int(count)

        def ptr(t):
            if t is None:
                return None
            if t.device.type != "cpu" or not t.is_pinned() or t.dtype != torch.float32 or not t.is_contiguous():
                raise ValueError("step_io needs contiguous, page-locked float32 host tensors")
            if t.numel() != 3 * n:
                raise ValueError(f"step_io: expected {n} x 3 values, got {t.numel()}")
            return ctypes.c_void_p(t.data_ptr())

        check(self.L.ivp_step_io(self._handle, ptr(x_in), ptr(v_in), ptr(x_out), ptr(v_out), int(first), n,
                                 ctypes.c_void_p(_stream_ptr(stream))), "ivp_step_io")

    def set_wait_limit(self, ns: int):
        """Test hook: longest wait on a grid barrier of the persistent kernels
        (ns <= 0 restores the default of 2 s)."""
        check(self.L.ivp_set_wait_limit(self._handle, int(ns)), "ivp_set_wait_limit")

    def reset_counters(self, stream=None):
        check(self.L.ivp_reset_counters(self._handle, ctypes.c_void_p(_stream_ptr(stream))), "ivp_reset_counters")

    def profile_step(self, n: int = 1, stream=None) -> dict:
        """n steps with host-driven launches and CUDA events around each
        kernel: {kernel name: (total ms, launches)}."""
        ms = np.zeros(_lib.K_COUNT, np.float64)
        cnt = np.zeros(_lib.K_COUNT, np.int32)
        check(self.L.ivp_profile_step(self._handle, int(n), ctypes.c_void_p(_stream_ptr(stream)),
                                      ms.ctypes.data_as(ctypes.c_void_p), cnt.ctypes.data_as(ctypes.c_void_p)),
              "ivp_profile_step")
        return {name: (float(ms[i]), int(cnt[i])) for i, name in enumerate(_lib.KERNEL_NAMES) if cnt[i] > 0}

    def prepare(self):
        """Instantiates the build and step graphs without launching them
        (host work only), so the first build() and step() launch at once."""
        check(self.L.ivp_prepare(self._handle), "ivp_prepare")

    def raw_stats_all(self, stream=None) -> list:
        """ivp_read_stats of every scene, one stream synchronisation."""
        out = (_lib.SolveStats * len(self.scenes))()
        check(self.L.ivp_read_stats_all(self._handle, ctypes.c_void_p(_stream_ptr(stream)), out),
              "ivp_read_stats_all")
        return list(out)

    def step_chunk(self, n: int, stream=None) -> "Chunk":
        """Launches n steps, each between two CUDA events, and returns at once
        (the per-step device times are read from the returned Chunk)."""
        return Chunk(self, n, stream)

    def raw_stats(self, scene: int = 0, stream=None) -> _lib.SolveStats:
        s = _lib.SolveStats()
        check(self.L.ivp_read_stats(self._handle, scene, ctypes.c_void_p(_stream_ptr(stream)), ctypes.byref(s)),
              "ivp_read_stats")
        return s

    def stats(self, scene: int = 0, stream=None) -> Stats:
        """The last solve's statistics and per-outer-iteration history of a
        scene (one stream synchronisation)."""
        if getattr(self, "_hist", None) is None:
            cap = self.options.max_hist
            self._hist = (np.zeros(cap, np.float64), np.zeros(cap, np.int32), ctypes.c_int32(0), ctypes.c_int32(0))
        err, pcg, ne, npc = self._hist
        s = _lib.SolveStats()
        check(self.L.ivp_read_solve(self._handle, scene, ctypes.c_void_p(_stream_ptr(stream)), ctypes.byref(s),
                                    err.ctypes.data_as(ctypes.c_void_p), pcg.ctypes.data_as(ctypes.c_void_p),
                                    len(err), ctypes.byref(ne), ctypes.byref(npc)), "ivp_read_solve")
        return Stats(status=int(s.status), stats_outer_iters=int(s.outer_iters),
                     stats_final_density_error=float(s.final_density_error),
                     stats_density_errors=[float(e) for e in err[:ne.value]],
                     stats_pcg_iters=[int(q) for q in pcg[:npc.value]],
                     overflow_particles=int(s.overflow_particles), total_pcg_iters=int(s.total_pcg_iters),
                     last_pap=float(s.last_pap), last_cg_iter=int(s.last_cg_iter))

    def neighbours(self, scene: int = 0, cache: Optional[int] = None, stream=None):
        """(count[n], ids[n, cache]) of a scene in the reference layout, local
        particle indices; rows of static particles are zero."""
        sc = self.scenes[scene]
        cache = cache or sc.cache_size
        n = sc.n
        count = torch.zeros(n, dtype=torch.int32, device=self.device)
        ids = torch.full((n, cache), -1, dtype=torch.int32, device=self.device)
        check(self.L.ivp_export_neighbours(self._handle, scene, ctypes.c_void_p(count.data_ptr()),
                                           ctypes.c_void_p(ids.data_ptr()), cache,
                                           ctypes.c_void_p(_stream_ptr(stream))), "ivp_export_neighbours")
        return count.cpu().numpy(), ids.cpu().numpy()

    # ------------------------------------------------------------ views
    def scene_slice(self, i: int) -> slice:
        return slice(int(self.offsets[i]), int(self.offsets[i + 1]))

    def get(self, name: str, scene: int = 0) -> np.ndarray:
        return self.arrays[name][self.scene_slice(scene)].cpu().numpy()


class Chunk:
    """n steps of an engine in flight on a stream, with a CUDA event pair
    around each step: `done()` polls, `wait()` blocks, `step_ms()` gives the
    device time of every step once done."""

    def __init__(self, eng: Engine, n: int, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream()
        self.n = int(n)
        self.starts = [torch.cuda.Event(enable_timing=True) for _ in range(self.n)]
        self.ends = [torch.cuda.Event(enable_timing=True) for _ in range(self.n)]
        for k in range(self.n):
            self.starts[k].record(s)
            eng.step(1, stream=s)
            self.ends[k].record(s)

    def done(self) -> bool:
        return self.n == 0 or self.ends[-1].query()

    def wait(self):
        if self.n:
            self.ends[-1].synchronize()

    def step_ms(self) -> list:
        return [a.elapsed_time(b) for a, b in zip(self.starts, self.ends)]

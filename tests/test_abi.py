"""The C-ABI library loads and exports every symbol include/ivp.h declares
(no GPU needed: nothing is called that touches a device)."""
import ctypes
import os
import re

import torch

from implicitvelocityprojection_b200 import _lib, build

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(REPO, "include", "ivp.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(ivp_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_and_binding_agree():
    declared = _declared()
    assert "ivp_engine_create" in declared and "ivp_ip_solve" in declared
    assert sorted(_lib.SIGNATURES) == declared


def test_library_exports_every_symbol():
    path = build.build()
    L = ctypes.CDLL(path)
    for name in _declared():
        assert hasattr(L, name), name


def test_status_strings_and_defaults():
    L = _lib.load()
    assert L.ivp_status_string(0) == b"ok"
    assert b"non-positive" in L.ivp_status_string(1)
    o = _lib.Options()
    L.ivp_default_options(o)
    assert o.lanes_per_particle == 0 and o.particles_per_block == 0  # chosen from the scenes
    assert o.list_stride >= 60 and o.use_graphs == 1


def test_resolve_options_picks_lanes_from_the_tile_count():
    """Lane count 0 becomes 4 lanes x 64 particles for few tiles per SM and 2
    lanes x 128 for many (the SM count of a B200 where no device is
    visible); explicit settings are kept, a particles-per-block of 0 follows
    the lane count."""
    from implicitvelocityprojection_b200 import scenes as S
    from implicitvelocityprojection_b200.engine import scene_desc
    L = _lib.load()
    sc = S.small_column()
    d = (_lib.SceneDesc * 1)()
    d[0] = scene_desc(sc, 0)
    o = _lib.Options()
    L.ivp_default_options(o)
    r = _lib.Options()
    assert L.ivp_resolve_options(d, 1, ctypes.byref(o), ctypes.byref(r)) == 0
    assert (r.lanes_per_particle, r.particles_per_block) == (4, 64)
    assert r.list_stride == o.list_stride and r.use_graphs == o.use_graphs
    sms = 148
    if torch.cuda.is_available():
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    big = (_lib.SceneDesc * 2)()
    for i in range(2):
        big[i] = scene_desc(sc, 0)
        big[i].n_dynamic = 16 * sms * 64 // 2 + 64 * i  # one tile above 16 per SM in total
        big[i].n_particles = big[i].n_dynamic
    big[1].particle_offset = big[0].n_particles
    assert L.ivp_resolve_options(big, 2, ctypes.byref(o), ctypes.byref(r)) == 0
    assert (r.lanes_per_particle, r.particles_per_block) == (2, 128)
    big[1].n_dynamic -= 64
    big[1].n_particles = big[1].n_dynamic
    assert L.ivp_resolve_options(big, 2, ctypes.byref(o), ctypes.byref(r)) == 0
    assert (r.lanes_per_particle, r.particles_per_block) == (4, 64)
    o.lanes_per_particle = 8
    assert L.ivp_resolve_options(big, 2, ctypes.byref(o), ctypes.byref(r)) == 0
    assert (r.lanes_per_particle, r.particles_per_block) == (8, 32)


def test_workspace_query_without_device():
    """Sizing is pure host arithmetic and validates arguments."""
    from implicitvelocityprojection_b200 import scenes as S
    from implicitvelocityprojection_b200.engine import scene_desc
    L = _lib.load()
    sc = S.small_column()
    d = (_lib.SceneDesc * 1)()
    d[0] = scene_desc(sc, 0)
    o = _lib.Options()
    L.ivp_default_options(o)
    n = ctypes.c_size_t(0)
    assert L.ivp_workspace_bytes(d, 1, ctypes.byref(o), ctypes.byref(n)) == 0
    assert n.value > sc.n * 100
    bad = _lib.Options()
    L.ivp_default_options(bad)
    bad.lanes_per_particle = 3
    assert L.ivp_workspace_bytes(d, 1, ctypes.byref(bad), ctypes.byref(n)) == _lib.BAD_ARG
    d[0].cache_size = 1000
    assert L.ivp_workspace_bytes(d, 1, ctypes.byref(o), ctypes.byref(n)) == _lib.BAD_ARG

"""The C-ABI library loads and exports every symbol include/ivp.h declares
(no GPU needed: nothing is called that touches a device)."""
import ctypes
import os
import re

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
    assert o.lanes_per_particle * o.particles_per_block == 256
    assert o.list_stride >= 60 and o.use_graphs == 1


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

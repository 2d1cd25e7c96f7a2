"""The allocation-free entry point ivp_density_aii_noalloc, called through the
C ABI, against the regular neighbour build (ivp_neighbour_build).

It serves callers that cannot allocate device memory (code inside another
runtime's memory arena, whose GPU memory another allocator owns, and loops
that cannot take cudaMalloc's synchronisation).  Two calls in a row must both
reproduce the engine's density and k, which also shows that what one call
leaves in the shared scratch array does not leak into the next.  This file
sorts last so that a run stopping at the first failure has run everything
else first.
"""
import ctypes

import numpy as np
import pytest
import torch

from implicitvelocityprojection_b200 import _lib
from implicitvelocityprojection_b200 import scenes as S

pytestmark = pytest.mark.gpu

RTOL = 1e-4


def _call(L, sc, x, m, dyn, density, k, stream):
    dom = (ctypes.c_float * 3)(*[float(a) for a in sc.domain_size])
    return L.ivp_density_aii_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(m.data_ptr()),
                                     ctypes.c_void_p(dyn.data_ptr()), sc.n, ctypes.c_float(sc.particle_radius),
                                     ctypes.cast(dom, ctypes.c_void_p), sc.cache_size,
                                     ctypes.c_void_p(density.data_ptr()), ctypes.c_void_p(k.data_ptr()),
                                     ctypes.c_void_p(stream))


def test_noalloc_matches_engine_twice():
    from implicitvelocityprojection_b200.engine import Engine
    L = _lib.load()
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for sc in (S.small_column(seed=4), S.random_column(5000, 2.0, seed=9)):
        eng = Engine([sc])
        eng.build()
        ref_density, ref_k = eng.get("density"), eng.get("k")
        m = eng.arrays["m"]
        x = eng.arrays["x"]
        dyn = eng.arrays["is_dynamic"]
        dmask = sc.is_dynamic == 1
        for _ in range(2):
            density = torch.full((sc.n,), -1.0, dtype=torch.float32, device=dev)
            k = torch.full((sc.n,), -1.0, dtype=torch.float32, device=dev)
            assert _call(L, sc, x, m, dyn, density, k, stream) == _lib.OK
            torch.cuda.synchronize()
            d, kk = density.cpu().numpy(), k.cpu().numpy()
            np.testing.assert_allclose(d[dmask], ref_density[dmask], rtol=RTOL)
            np.testing.assert_allclose(kk[dmask], ref_k[dmask], rtol=RTOL)
            assert np.all(kk[~dmask] == 0.0)
            assert np.all(d[~dmask] == -1.0)  # static densities are left untouched


def test_noalloc_matches_reference_fixture(golden_dir):
    """Density and k against the reference's own neighbour build, density and
    Aii (tests/golden/block_solve.npz), on two calls in a row."""
    import os
    g = np.load(os.path.join(golden_dir, "block_solve.npz"))
    L = _lib.load()
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream().cuda_stream
    n = g["x"].shape[0]
    sc = S.Scene(x=np.array(g["x"], np.float32), v=np.array(g["v0"], np.float32), is_dynamic=g["is_dynamic"],
                 material=g["material"], density0=g["density0"], particle_radius=float(g["particle_radius"]),
                 domain_size=g["domain_size"], dt=float(g["dt"]))
    x = torch.from_numpy(sc.x).to(dev)
    m = torch.from_numpy(np.array(g["m"], np.float32)).to(dev)
    dyn = torch.from_numpy(np.array(g["is_dynamic"], np.int32)).to(dev)
    dmask = g["is_dynamic"] == 1
    for _ in range(2):
        density = torch.full((n,), -1.0, dtype=torch.float32, device=dev)
        k = torch.full((n,), -1.0, dtype=torch.float32, device=dev)
        assert _call(L, sc, x, m, dyn, density, k, stream) == _lib.OK
        torch.cuda.synchronize()
        np.testing.assert_allclose(density.cpu().numpy()[dmask], g["density"][dmask], rtol=RTOL)
        np.testing.assert_allclose(k.cpu().numpy()[dmask], g["k"][dmask], rtol=RTOL)


def test_noalloc_rejects_oversized_inputs():
    L = _lib.load()
    dev = torch.device("cuda")
    big = S.lattice_block([0.1, 0.1, 0.1], (41, 41, 41), 0.02)  # 68,921 > 65,536 particles
    sc = S.assemble([big], [], particle_radius=0.01, domain_size=[1.0, 1.0, 1.0])
    x = torch.from_numpy(sc.x).to(dev)
    m = torch.from_numpy(sc.masses()[0]).to(dev)
    dyn = torch.from_numpy(sc.is_dynamic).to(dev)
    out = torch.zeros(sc.n, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    assert _call(L, sc, x, m, dyn, out, out.clone(), stream) == _lib.BAD_ARG
    # too many grid cells: 1,000,000 > 262,144
    small = S.assemble([S.lattice_block([0.1, 0.1, 0.1], (4, 4, 4), 0.02)], [], particle_radius=0.01,
                       domain_size=[4.0, 4.0, 4.0])
    xs = torch.from_numpy(small.x).to(dev)
    ms = torch.from_numpy(small.masses()[0]).to(dev)
    ds = torch.from_numpy(small.is_dynamic).to(dev)
    o = torch.zeros(small.n, dtype=torch.float32, device=dev)
    assert _call(L, small, xs, ms, ds, o, o.clone(), stream) == _lib.BAD_ARG
    assert "IVP_NOALLOC_MAX_CELLS" in L.ivp_last_error().decode()  # the reason, for the caller

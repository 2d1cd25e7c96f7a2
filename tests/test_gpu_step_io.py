"""Steps with host input and output (ivp_step_io): the copies run inside the
step, overlapped with its kernels, and the results are those of a plain step
with the same copies made around it, bit for bit."""
import ctypes

import numpy as np
import pytest
import torch

import _gpu_helpers as H
from implicitvelocityprojection_b200 import _lib
from implicitvelocityprojection_b200 import scenes as S

pytestmark = pytest.mark.gpu


def _pinned(a):
    t = torch.empty(tuple(a.shape), dtype=torch.float32).pin_memory()
    t.copy_(torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32)))
    return t


def _scenes():
    return [S.column_in_box((10, 16, 10), 0.02, (0.3, 0.5, 0.3), seed=21, viscosity_method=1, viscosity_coeff=1e-3),
            S.random_column(3000, 2.0, seed=22)]


@pytest.mark.parametrize("use_graphs,persistent", [(True, True), (True, False), (False, True)])
def test_step_io_equals_step_with_copies(use_graphs, persistent):
    """The fluid state of both scenes, held on the host, stepped 4 times:
    step_io (inputs and outputs aliased) against ivp_step with the copies made
    around it by the caller."""
    scs = _scenes()
    a = H.engine(scs, use_graphs=use_graphs, persistent=persistent)
    b = H.engine(scs, use_graphs=use_graphs, persistent=persistent)
    for e in (a, b):
        e.build()
    n = a.n_total
    xa, va = _pinned(a.arrays["x"].cpu().numpy()), _pinned(a.arrays["v"].cpu().numpy())
    xb, vb = xa.clone().pin_memory(), va.clone().pin_memory()
    for _ in range(4):
        a.step_io(xa, va, xa, va)
        b.arrays["x"].copy_(xb, non_blocking=True)
        b.arrays["v"].copy_(vb, non_blocking=True)
        b.step(1)
        xb.copy_(b.arrays["x"], non_blocking=True)
        vb.copy_(b.arrays["v"], non_blocking=True)
        torch.cuda.synchronize()
        assert torch.equal(xa, xb) and torch.equal(va, vb)
        assert torch.equal(xa, a.arrays["x"].cpu()) and torch.equal(va, a.arrays["v"].cpu())
    for i in range(len(scs)):
        assert a.stats(i).status == 0 and a.stats(i).stats_outer_iters == b.stats(i).stats_outer_iters
    assert xa.shape[0] == n


def test_step_io_range_and_null_pointers():
    """Only a range of particles, outputs only, and inputs only."""
    sc = S.column_in_box((10, 16, 10), 0.02, (0.3, 0.5, 0.3), seed=23)
    nd = sc.n_dynamic
    a = H.engine([sc])
    b = H.engine([sc])
    for e in (a, b):
        e.build()
    # outputs only: a plain step, then the fluid x, v appear in the host tensors
    xo = torch.zeros((nd, 3), dtype=torch.float32).pin_memory()
    vo = torch.zeros((nd, 3), dtype=torch.float32).pin_memory()
    a.step_io(None, None, xo, vo, first=0, count=nd)
    b.step(1)
    torch.cuda.synchronize()
    assert torch.equal(xo, b.arrays["x"][:nd].cpu()) and torch.equal(vo, b.arrays["v"][:nd].cpu())
    # inputs only, over the fluid range: a changed velocity is used by the step
    vi = vo.clone().pin_memory()
    vi[:, 0] += 0.05
    a.step_io(None, vi, None, None, first=0, count=nd)
    b.arrays["v"][:nd].copy_(vi)
    b.step(1)
    torch.cuda.synchronize()
    assert torch.equal(a.arrays["x"], b.arrays["x"]) and torch.equal(a.arrays["v"], b.arrays["v"])


def test_step_io_rejects_pageable_and_bad_ranges():
    """Host buffers must be page-locked; the range must lie in the particle
    arrays.  Nothing is launched on a rejected call."""
    sc = S.column_in_box((6, 8, 6), 0.02, (0.2, 0.3, 0.2), seed=24)
    e = H.engine([sc])
    e.build()
    L = _lib.load()
    pageable = np.zeros((sc.n, 3), np.float32)
    p = ctypes.c_void_p(pageable.ctypes.data)
    st = L.ivp_step_io(e._handle, p, None, None, None, 0, sc.n, None)
    assert st == _lib.BAD_ARG
    pinned = torch.zeros((sc.n, 3), dtype=torch.float32).pin_memory()
    q = ctypes.c_void_p(pinned.data_ptr())
    assert L.ivp_step_io(e._handle, None, None, q, None, 1, sc.n, None) == _lib.BAD_ARG
    assert L.ivp_step_io(e._handle, None, None, q, None, -1, 10, None) == _lib.BAD_ARG
    with pytest.raises(ValueError):
        e.step_io(torch.zeros((sc.n, 3)), None, None, None)
    # the engine still steps normally
    e.step(1)
    assert e.stats(0).status == 0


def test_framework_forward_host_equals_forward():
    """Framework.forward_host(x, v) against forward() with the caller's own
    copies: same statistics and the same host state, bit for bit."""
    from implicitvelocityprojection_b200.config import SimConfig
    from implicitvelocityprojection_b200.framework import Framework
    from implicitvelocityprojection_b200.neighbour_search import NeighbourSearch
    from implicitvelocityprojection_b200.simulation_data import SimulationData
    sc = S.column_in_box((10, 16, 10), 0.02, (0.3, 0.5, 0.3), seed=25, viscosity_method=1, viscosity_coeff=1e-3)
    fws = []
    for _ in range(2):
        cfg = SimConfig.from_scene(sc)
        ps = SimulationData.from_scene(sc, cfg, device="cuda")
        fw = Framework(ps, NeighbourSearch(cfg.domain_size, cfg.support_radius, ps), cfg)
        fw.initialize()
        fws.append((fw, ps))
    nd = sc.n_dynamic
    (fa, pa), (fb, pb) = fws
    xa, va = _pinned(pa.x[:nd].cpu().numpy()), _pinned(pa.v[:nd].cpu().numpy())
    xb, vb = xa.clone().pin_memory(), va.clone().pin_memory()
    for _ in range(3):
        fa.forward_host(xa, va)
        pb.x[:nd].copy_(xb)
        pb.v[:nd].copy_(vb)
        fb.forward()
        xb.copy_(pb.x[:nd])
        vb.copy_(pb.v[:nd])
        torch.cuda.synchronize()
        assert torch.equal(xa, xb) and torch.equal(va, vb)
        assert fa.pressure.stats_outer_iters == fb.pressure.stats_outer_iters
        assert fa.pressure.stats_density_errors == fb.pressure.stats_density_errors

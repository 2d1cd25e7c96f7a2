"""Scene ingestion from the reference's JSON format, pinned to the reference
loader's own output (tests/golden/scene_ingest.npz, made by running
scene_loader.py on tests/golden/scene_blocks.json)."""
import copy
import json
import os

import numpy as np
import pytest

from implicitvelocityprojection_b200.scene_io import load_scene

HERE = os.path.dirname(os.path.abspath(__file__))
SCENE = os.path.join(HERE, "golden", "scene_blocks.json")


def test_blocks_shell_walls_bit_identical_to_reference_loader(golden_dir):
    g = np.load(os.path.join(golden_dir, "scene_ingest.npz"))
    sc = load_scene(SCENE)
    assert sc.n == g["x"].shape[0]
    assert np.array_equal(sc.x, g["x"])
    assert np.array_equal(sc.v, g["v"])
    assert np.array_equal(sc.is_dynamic, g["is_dynamic"])
    assert np.array_equal(sc.material, g["material"])
    assert np.array_equal(sc.density0, g["density0"])
    m, _ = sc.masses()
    assert np.array_equal(m, g["m"])
    assert np.allclose(sc.domain_size, g["domain_size"])
    assert sc.viscosity_method == 1 and sc.surface_tension_method == 1 and sc.surface_tension_coeff == 0.05
    assert sc.dt == 0.001 and sc.gravity == (0.0, -9.81, 0.0)


def test_mesh_bodies_need_voxelised_points():
    with open(SCENE) as f:
        data = json.load(f)
    d = copy.deepcopy(data)
    d["RigidBodies"] = [{"objectId": 5, "geometryFile": "./data/models/box.obj", "isDynamic": False}]
    with pytest.raises(NotImplementedError):
        load_scene(d)
    pts = np.array([[0.5, 0.05, 0.25], [0.52, 0.05, 0.25]], np.float32)
    d["RigidBodies"][0]["voxelizedPoints"] = pts.tolist()
    sc = load_scene(d)
    base = load_scene(SCENE)
    assert sc.n == base.n + 2
    nf = int(base.is_dynamic.sum())
    assert np.array_equal(sc.x[nf:nf + 2], pts)  # rigid bodies come before generated bodies and walls
    assert np.all(sc.material[nf:nf + 2] == 0) and np.all(sc.is_dynamic[nf:nf + 2] == 0)
    d2 = copy.deepcopy(data)
    d2["ScheduledSpawns"] = [{"objectId": 9}]
    with pytest.raises(NotImplementedError):
        load_scene(d2)


@pytest.mark.gpu
def test_ingested_scene_steps_like_the_oracle():
    from oracle import oracle as O
    from implicitvelocityprojection_b200.engine import Engine
    sc = load_scene(SCENE)
    eng = Engine([sc])
    eng.build()
    st = O.State.from_scene(sc)
    st.rebuild()
    dyn = sc.is_dynamic == 1
    for _ in range(3):
        eng.step(1)
        st.step(fast=True)
        assert eng.stats(0).status == 0 and st.status == 0
    assert np.abs(eng.get("x")[dyn] - st.x[dyn]).max() < 1e-5


def test_loader_interface_populates_simulation_data():
    from implicitvelocityprojection_b200.config import SimConfig
    from implicitvelocityprojection_b200.scene_io import SceneLoader
    from implicitvelocityprojection_b200.simulation_data import SimulationData
    cfg = SimConfig.from_json(SCENE)
    loader = SceneLoader(cfg)
    data = loader.prepare_scene()
    ps = SimulationData(cfg, device="cpu")
    loader.populate_scene(ps, data)
    sc = data["scene"]
    n = ps.particle_num
    assert n == sc.n
    assert np.array_equal(ps.x[:n].numpy(), sc.x)
    m, _ = sc.masses()
    assert np.array_equal(ps.m[:n].numpy(), m)

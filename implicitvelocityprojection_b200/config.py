"""SimConfig: the reference's scene configuration object
(`scripts/io/config_builder.py:10-157`), same field names, same JSON keys and
the same lazy `get_cfg(name, default)` lookup of solver keys."""
from __future__ import annotations

import dataclasses
import json
from typing import Optional


@dataclasses.dataclass
class SimConfig:
    domain_size: tuple = (1.0, 1.0, 1.0)
    domain_start: tuple = (0.0, 0.0, 0.0)
    particle_radius: float = 0.01
    support_radius: float = 0.04
    particle_diameter: float = 0.02
    density0: float = 1000.0
    dt: float = 0.0016
    gravity: tuple = (0.0, -9.8, 0.0)
    viscosity_method: int = 0
    surface_tension_method: int = 0
    viscosity_coeff: float = 0.01
    surface_tension_coeff: float = 0.01
    scene_data: Optional[dict] = dataclasses.field(default=None)

    def __post_init__(self):
        # config_builder.py:46-52
        self.particle_diameter = 2.0 * self.particle_radius
        self.support_radius = 4.0 * self.particle_radius

    @classmethod
    def from_json(cls, scene_file_path: str) -> "SimConfig":
        with open(scene_file_path, "r") as f:
            scene_data = json.load(f)
        return cls.from_dict(scene_data)

    @classmethod
    def from_dict(cls, scene_data: dict) -> "SimConfig":
        cfg = scene_data.get("Configuration", {})
        start = tuple(cfg.get("domainStart", [0.0, 0.0, 0.0]))
        end = tuple(cfg.get("domainEnd", [1.0, 1.0, 1.0]))
        return cls(domain_size=tuple(e - s for s, e in zip(start, end)), domain_start=start,
                   particle_radius=float(cfg.get("particleRadius", 0.01)),
                   dt=float(cfg.get("timeStepSize", 0.0016)), density0=float(cfg.get("density0", 1000.0)),
                   gravity=tuple(cfg.get("gravitation", [0.0, -9.8, 0.0])),
                   viscosity_method=int(cfg.get("viscosityMethod", 0)),
                   surface_tension_method=int(cfg.get("surfaceTensionMethod", 0)),
                   viscosity_coeff=float(cfg.get("viscosityCoeff", 0.01)),
                   surface_tension_coeff=float(cfg.get("surfaceTensionCoeff", 0.01)),
                   scene_data=scene_data)

    @classmethod
    def from_scene(cls, sc) -> "SimConfig":
        """Config of a synthetic `scenes.Scene`."""
        return cls.from_dict({"Configuration": sc.config()})

    def get_cfg(self, name: str, default=None):
        if self.scene_data is None:
            return default
        return self.scene_data.get("Configuration", {}).get(name, default)

    def _list(self, key):
        return [] if self.scene_data is None else self.scene_data.get(key, [])

    def get_rigid_bodies(self):
        return self._list("RigidBodies")

    def get_solid_bodies(self):
        return self._list("SolidBodies")

    def get_fluid_blocks(self):
        return self._list("FluidBlocks")

    def get_fluid_bodies(self):
        return self._list("FluidBodies")

    def get_scheduled_spawns(self):
        return self._list("ScheduledSpawns")

    def get_generated_bodies(self):
        return self._list("GeneratedBodies")

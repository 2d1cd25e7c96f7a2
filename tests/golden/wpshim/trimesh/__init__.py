"""Import stand-in for trimesh: the reference's scene loader imports it at
module level but only uses it to voxelise OBJ meshes, which the fixture
scenes do not contain.  Any use raises."""


def __getattr__(name):
    raise ImportError(f"trimesh.{name} is not available: OBJ voxelisation is outside the fixture scenes")

"""PyAurora/geometry.py: meshes of a scene file's "objects"."""
from .core import Named, _Transformable

__all__ = ["Mesh", "ObjMesh", "TriangleMesh"]


class Mesh(_Transformable, Named):
    def __init__(self, name, serialize):
        s = list(serialize) + ["name", "transforms", "material", "type"]
        Named.__init__(self, name, s)
        self._s["type"] = "geometry"

    def setMaterial(self, m):
        self._s["material"] = m


class ObjMesh(Mesh):
    """An OBJ file with `subdlevels` levels of Loop subdivision."""

    def __init__(self, name, subdlevels, path):
        Mesh.__init__(self, name, ["path", "subdlevels"])
        self._s["path"] = path
        self._s["subdlevels"] = subdlevels


class TriangleMesh(Mesh):
    """Inline points and indices (serialised as PyAurora does; the reference's scene-file
    parser reads OBJ meshes only, and so does this loader)."""

    def __init__(self, name, points, pointIndices):
        Mesh.__init__(self, name, ["points", "pointIndices"])
        self._s["points"] = points
        self._s["pointIndices"] = pointIndices

"""PyAurora/lights.py: square and environment lights."""
from .core import Named, _Transformable

__all__ = ["Light", "SquareLight", "EnvLight"]


class Light(_Transformable, Named):
    def __init__(self, name, serialize):
        s = list(serialize) + ["transforms", "type", "name"]
        Named.__init__(self, name, s)
        self._s["type"] = "light"


class SquareLight(Light):
    """A [-scaleX, scaleX] x [-scaleY, scaleY] quad emitting color * 2^exposure."""

    def __init__(self, name, scaleX, scaleY, color, exposure):
        Light.__init__(self, name, ["scaleX", "scaleY", "color", "exposure"])
        self._s["color"] = [float(c) for c in color]
        self._s["exposure"] = float(exposure)
        self._s["scaleX"] = float(scaleX)
        self._s["scaleY"] = float(scaleY)


class EnvLight(Light):
    """An environment: color * 2^exposure, times the lat-long `envmap` image if one is named."""

    def __init__(self, name, color, exposure, envmap):
        Light.__init__(self, name, ["color", "exposure", "envmap"])
        self._s["color"] = [float(c) for c in color]
        self._s["exposure"] = float(exposure)
        self._s["type"] = "envlight"
        self._s["envmap"] = envmap

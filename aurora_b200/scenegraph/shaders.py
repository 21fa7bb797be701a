"""PyAurora/shaders.py: texture shaders and materials. A colour or float argument may be a
value or the name of a shader (a string)."""
from .core import Named

__all__ = ["Texture2DShader", "TriplanarTextureShader", "Material", "MatteMaterial", "MetalMaterial",
           "TransmitMaterial", "GlassMaterial", "CarMaterial", "KelemenMaterial"]


def _color(c):
    return c if isinstance(c, str) else [float(c[0]), float(c[1]), float(c[2])]


class Texture2DShader(Named):
    def __init__(self, name, attributetype, texturename):
        Named.__init__(self, name, ["texturename", "type", "attributetype"])
        self._s["texturename"] = texturename
        self._s["type"] = "texture2DShader"
        self._s["attributetype"] = attributetype


class TriplanarTextureShader(Named):
    def __init__(self, name, attributetype, texturename, scale):
        Named.__init__(self, name, ["texturename", "scale", "type", "attributetype"])
        self._s["texturename"] = texturename
        self._s["type"] = "triplanarTextureShader"
        self._s["scale"] = scale
        self._s["attributetype"] = attributetype


class Material(Named):
    def setNormalMap(self, normalmap):
        self._s["normalmap"] = normalmap
        if "normalmap" not in self._serialize:
            self._serialize.append("normalmap")


class MatteMaterial(Material):
    def __init__(self, name, color=(1, 1, 1)):
        Named.__init__(self, name, ["color", "type"])
        self._s["color"] = _color(color)
        self._s["type"] = "matteMaterial"


class MetalMaterial(Material):
    def __init__(self, name, reflectance, roughnessA, roughnessB, mix, gain):
        Named.__init__(self, name, ["reflectance", "roughnessA", "roughnessB", "mix", "gain", "type"])
        self._s["reflectance"] = _color(reflectance)
        self._s["roughnessA"] = roughnessA
        self._s["roughnessB"] = roughnessB
        self._s["mix"] = mix
        self._s["gain"] = gain
        self._s["type"] = "metalMaterial"


class TransmitMaterial(Material):
    """Serialised as PyAurora does; the reference's parser has no transmitMaterial."""

    def __init__(self, name, color=(1, 1, 1), ior=1.333):
        Named.__init__(self, name, ["color", "ior", "type"])
        self._s["color"] = _color(color)
        self._s["ior"] = float(ior)
        self._s["type"] = "transmitMaterial"


class GlassMaterial(Material):
    def __init__(self, name, specCol=(1, 1, 1), transmitCol=(1, 1, 1), reflectance=1.0, ior=1.333):
        Named.__init__(self, name, ["specColor", "transmitColor", "reflectance", "ior", "type"])
        self._s["specColor"] = _color(specCol)
        self._s["transmitColor"] = _color(transmitCol)
        self._s["reflectance"] = float(reflectance)
        self._s["ior"] = float(ior)
        self._s["type"] = "glassMaterial"


class CarMaterial(Material):
    """Serialised as PyAurora does; its construction is disabled in the reference's parser."""

    def __init__(self, name, diffcolor=(1, 1, 1), clearcoatreflectance=0.1, clearcoatroughness=0.1,
                 toppaintcolor=(1, 1, 1), basespectopreflectance=0.2, basespectoproughness=0.2,
                 bottompaintcolor=(1, 1, 1), basespecbottomreflectance=0.3, basespecbottomroughness=0.3):
        Named.__init__(self, name, ["diffusecolor", "clearcoatreflectance", "clearcoatroughness", "toppaintcolor",
                                    "basespectopreflectance", "basespectoproughness", "bottompaintcolor",
                                    "basespecbottomreflectance", "basespecbottomroughness", "type"])
        self._s.update(diffusecolor=_color(diffcolor), clearcoatreflectance=float(clearcoatreflectance),
                       clearcoatroughness=float(clearcoatroughness), toppaintcolor=_color(toppaintcolor),
                       basespectopreflectance=float(basespectopreflectance),
                       basespectoproughness=float(basespectoproughness), bottompaintcolor=_color(bottompaintcolor),
                       basespecbottomreflectance=float(basespecbottomreflectance),
                       basespecbottomroughness=float(basespecbottomroughness), type="carMaterial")


class KelemenMaterial(Material):
    def __init__(self, name, diffcolor=(1, 1, 1), speccolor=(1, 1, 1), roughness=50, reflectance=0.1):
        Named.__init__(self, name, ["diffusecolor", "speccolor", "roughness", "reflectance", "type"])
        self._s["diffusecolor"] = _color(diffcolor)
        self._s["speccolor"] = _color(speccolor)
        self._s["roughness"] = roughness
        self._s["reflectance"] = reflectance
        self._s["type"] = "kelemenMaterial"

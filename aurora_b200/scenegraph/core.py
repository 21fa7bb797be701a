"""PyAurora/core.py: the Serializable framework, Scene, Camera and render()."""
import json
import math
import os
import time

__all__ = ["Serializable", "Scene", "Camera", "render", "scene_json"]


class Serializable(object):
    """Objects that write themselves into a JSON dictionary (PyAurora/core.py:15-53).

    Each key named in `serialize` starts as an empty list in self._s. On serialisation a
    list of plain dicts (transforms) is written as that list, a list of Serializable
    objects as a dict filled by each item's serialize(), an empty list as an empty dict,
    and any other value as itself."""

    def __init__(self, name, serialize):
        self._s = {key: [] for key in serialize}
        self._s["name"] = str(name)
        self._serialize = list(serialize)

    def getName(self):
        return self._s["name"]

    def _value(self, value):
        if isinstance(value, Serializable):
            out = {}
            value.serialize(out)
            return out
        if isinstance(value, list):
            out = {}
            for item in value:
                if isinstance(item, dict):
                    return value
                item.serialize(out)
            return out
        return value

    def serialize(self, root):
        for key in self._serialize:
            root[key] = self._value(self._s[key])


class _Transformable(object):
    """translate / scale / rotateX / rotateY / rotateZ, appended in call order."""

    def translate(self, x, y, z):
        self._s["transforms"].append({"translate": [float(x), float(y), float(z)]})

    def scale(self, x, y, z):
        self._s["transforms"].append({"scale": [float(x), float(y), float(z)]})

    def rotateX(self, x):
        self._s["transforms"].append({"rotateX": float(x)})

    def rotateY(self, x):
        self._s["transforms"].append({"rotateY": float(x)})

    def rotateZ(self, x):
        self._s["transforms"].append({"rotateZ": float(x)})


class Named(Serializable):
    """An object written as root[name] = {its keys} (meshes, lights, materials, shaders):
    values as they are (lists included), a Serializable value as its own dictionary."""

    def serialize(self, root):
        obj = {}
        for key in self._serialize:
            v = self._s[key]
            if isinstance(v, Serializable):
                obj[key] = {}
                v.serialize(obj[key])
            else:
                obj[key] = v
        root[self.getName()] = obj


class Scene(Serializable):
    def __init__(self):
        Serializable.__init__(self, "scene", ["options", "renderCam", "objects", "materials", "shaders"])
        self._s["options"] = {}

    def setOptions(self, options):
        self._s["options"] = options

    def setCamera(self, camera):
        self._s["renderCam"] = [camera]

    def append(self, obj):
        self._s["objects"].append(obj)

    def appendShader(self, shader):
        self._s["shaders"].append(shader)

    def appendMaterial(self, material):
        self._s["materials"].append(material)


class Camera(_Transformable, Serializable):
    def __init__(self, fov=math.pi / 4):
        Serializable.__init__(self, "camera", ["transforms", "fov"])
        self._s["fov"] = float(fov)


def scene_json(scene):
    """The scene as the JSON dictionary PyAurora's render() writes."""
    root = {}
    scene.serialize(root)
    return root


def render(scene, path=None, ctx=None, mode="wavefront", write_image=True, pass_spp=None, interval=1.0):
    """Writes the scene file (to `path`, default ./aurora_scene.json), loads it with the
    library's scene-file loader and renders it with the file's options on the GPU. The
    film is written, as OpenexrDisplay writes it (half RGBA), to the options' `filename`
    (relative to the scene file's folder) when there is one. With `pass_spp` the samples
    are rendered in passes of that many and the image is also rewritten after a pass
    whenever `interval` seconds have passed since the last write (the reference's
    progressive display, renderer.cpp:240-262). Returns the (H, W, 4) film."""
    import numpy as np
    import aurora_b200 as ab
    from aurora_b200 import _abi
    path = path or os.path.join(os.getcwd(), "aurora_scene.json")
    text = "// AURORA SCENE FILE\n// generated %s\n" % time.strftime("%Y-%m-%d %H:%M:%S", time.localtime())
    root = scene_json(scene)
    with open(path, "w") as f:
        f.write(text + json.dumps(root, indent=4))
    own = ctx is None
    ctx = ctx or ab.Context(0)
    try:
        sc = ab.Scene(ctx, json_path=path)
        try:
            o = sc.file_opts
            o.mode = _abi.RENDER_WAVEFRONT if mode == "wavefront" else _abi.RENDER_PLAIN
            film = np.zeros((sc.height, sc.width, 4), np.float32)
            out = root.get("options", {}).get("filename")
            out = os.path.join(os.path.dirname(os.path.abspath(path)), out) if write_image and out else None
            if pass_spp:
                last = [time.monotonic()]

                def on_pass(img, done):
                    if out and time.monotonic() - last[0] >= interval:
                        ab.write_film(out, img)
                        last[0] = time.monotonic()
                    return False
                sc.render_progressive(o, pass_spp, on_pass, out=film)
            else:
                sc.render(o, out=film)
        finally:
            sc.close()
        if out:
            ab.write_film(out, film)
        return film
    finally:
        if own:
            ctx.close()

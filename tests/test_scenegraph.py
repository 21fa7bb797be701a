"""aurora_b200.scenegraph: PyAurora's scene-building classes (PyAurora/core.py, geometry.py,
lights.py, shaders.py) writing the JSON scene file that the library's loader reads."""
import json
import os

import numpy as np
import pytest

from aurora_b200 import _abi, scenes
from aurora_b200.scenegraph import core, geometry, lights, shaders
from test_scene_file import BOXES, METAL, WALLS, flat_obj, write_box_scene


def box_scene_graph(d, width=64, height=64, spp=4):
    """The box workload of write_box_scene, built with the PyAurora classes."""
    s = core.Scene()
    s.setOptions({"resolution": [width, height], "pixelsamples": spp, "lightsamples": 1, "mindepth": 5,
                  "maxdepth": 5, "filename": "box.exr"})
    cam = core.Camera(fov=scenes.FOV40)
    cam.translate(0, 0, 3.5)
    s.setCamera(cam)
    for name, corners, mat in WALLS:
        v, f = scenes.quad(*corners)
        flat_obj(os.path.join(d, name + ".obj"), v, f)
        m = geometry.ObjMesh(name, 0, name + ".obj")
        m.setMaterial(mat)
        s.append(m)
    bv, bf, _ = scenes.box_mesh()
    flat_obj(os.path.join(d, "box.obj"), bv, bf)
    for k, (x, y, z, sx, sy, sz, ry) in enumerate(BOXES):
        m = geometry.ObjMesh(f"o{5 + k}_box{k}", 0, "box.obj")
        m.translate(x, y, z)
        m.rotateY(ry)
        m.scale(sx, sy, sz)
        m.setMaterial("m3_box")
        s.append(m)
    light = lights.SquareLight("o7_light", 0.25, 0.25, [17.0, 12.0, 4.0], 0.0)
    light.translate(0, 0.999, 0)
    light.rotateX(-90)
    s.append(light)
    s.appendMaterial(shaders.MatteMaterial("m0_wall", [0.73, 0.73, 0.73]))
    s.appendMaterial(shaders.MatteMaterial("m1_red", [0.65, 0.05, 0.05]))
    s.appendMaterial(shaders.MatteMaterial("m2_green", [0.12, 0.45, 0.15]))
    s.appendMaterial(shaders.MetalMaterial("m3_box", list(METAL["specular"]), 0.3, 0.6, 0.4, list(METAL["gain"])))
    return s


def test_serialised_layout():
    s = core.Scene()
    s.setOptions({"resolution": [16, 16]})
    cam = core.Camera(0.5)
    cam.rotateY(10)
    s.setCamera(cam)
    g = geometry.ObjMesh("g", 2, "m.obj")
    g.setMaterial("k")
    s.append(g)
    s.append(lights.EnvLight("sky", [1, 1, 1], 0.5, "sky.exr"))
    k = shaders.KelemenMaterial("k", "tex", [1, 1, 1], 0.2, 0.5)
    k.setNormalMap([0.1, 0.2, 0.9])
    s.appendMaterial(k)
    s.appendShader(shaders.TriplanarTextureShader("tex", "color", "t.exr", 0.25))
    root = core.scene_json(s)
    assert root["options"] == {"resolution": [16, 16]}
    assert root["renderCam"] == {"transforms": [{"rotateY": 10.0}], "fov": 0.5}
    assert root["objects"]["g"] == {"path": "m.obj", "subdlevels": 2, "name": "g", "transforms": [],
                                    "material": "k", "type": "geometry"}
    assert root["objects"]["sky"] == {"color": [1.0, 1.0, 1.0], "exposure": 0.5, "envmap": "sky.exr",
                                      "transforms": [], "type": "envlight", "name": "sky"}
    assert root["materials"]["k"] == {"diffusecolor": "tex", "speccolor": [1.0, 1.0, 1.0], "roughness": 0.2,
                                      "reflectance": 0.5, "type": "kelemenMaterial", "normalmap": [0.1, 0.2, 0.9]}
    assert root["shaders"]["tex"] == {"texturename": "t.exr", "scale": 0.25, "type": "triplanarTextureShader",
                                      "attributetype": "color"}
    empty = core.scene_json(core.Scene())
    assert empty["objects"] == {} and empty["renderCam"] == {}


def test_graph_scene_loads_like_the_hand_written_file(tmp_path):
    d = str(tmp_path)
    ref, ref_opts, _ = scenes.load_scene_file(write_box_scene(d))
    path = os.path.join(d, "graph.json")
    root = core.scene_json(box_scene_graph(d))
    with open(path, "w") as f:
        f.write("// AURORA SCENE FILE\n" + json.dumps(root, indent=4))
    got, opts, info = scenes.load_scene_file(path)
    assert (opts.spp, opts.min_depth, opts.max_depth) == (ref_opts.spp, ref_opts.min_depth, ref_opts.max_depth)
    assert info["output"] == "box.exr"
    for field in ("verts", "tri_vidx", "tri_attr", "corner_normals", "attr_material", "attr_emission"):
        np.testing.assert_array_equal(getattr(got, field), getattr(ref, field), err_msg=field)
    assert [bytes(m) for m in got.materials] == [bytes(m) for m in ref.materials]


def test_parser_refusals(tmp_path):
    d = str(tmp_path)
    s = box_scene_graph(d)
    s.appendMaterial(shaders.CarMaterial("car"))
    path = os.path.join(d, "car.json")
    with open(path, "w") as f:
        json.dump(core.scene_json(s), f)
    with pytest.raises(_abi.AuroraError) as e:
        scenes.load_scene_file(path)
    assert e.value.status == _abi.ERR_UNSUPPORTED

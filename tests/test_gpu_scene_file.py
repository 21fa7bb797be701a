"""Scenes loaded from the reference's file format (aur_scene_load_json) render on the
device like the oracle's CPU render of the same flattened arrays."""
import json
import os

import numpy as np
import pytest

from test_scene_file import icosahedron, write_box_scene, write_obj

pytestmark = pytest.mark.gpu


def _render_both(ctx, kelemen_tables, oracle_lib, path, spp):
    import aurora_b200 as ab
    from aurora_b200 import _abi, scenes
    data, opts, _ = scenes.load_scene_file(path)
    scene = ab.Scene(ctx, json_path=path)
    assert scene.ntri == data.ntri and scene.file_opts.spp == opts.spp
    o = ab.render_opts(spp, opts.max_depth, opts.min_depth, 1, mode=_abi.RENDER_WAVEFRONT)
    gpu = scene.render(o).film
    scene.close()
    cpu, m2, _ = oracle_lib.OracleScene(data, kelemen_tables).render(spp, opts.max_depth, opts.min_depth, 1)
    return gpu, cpu, m2


def _check(gpu, cpu, m2, spp):
    sigma = np.sqrt(m2 / max(spp - 1, 1) / spp)
    diff = np.abs(gpu[..., :3].astype(np.float64) - cpu[..., :3])
    assert np.mean(diff <= 3 * sigma + 1e-4) > 0.99
    np.testing.assert_allclose(gpu[..., 3], cpu[..., 3], atol=1e-6)


def test_box_scene_file_renders_like_oracle(ctx, kelemen_tables, oracle_lib, tmp_path):
    path = write_box_scene(str(tmp_path), 64, 64, spp=8)
    gpu, cpu, m2 = _render_both(ctx, kelemen_tables, oracle_lib, path, 8)
    _check(gpu, cpu, m2, 8)


def test_loop_subdivided_kelemen_sphere_file(ctx, kelemen_tables, oracle_lib, tmp_path):
    """The sphere workload as the reference builds it: an icosahedron OBJ with 4 levels of
    Loop subdivision (limit surface), a Kelemen material, a ground quad and a square light."""
    d = str(tmp_path)
    v, f = icosahedron()
    write_obj(os.path.join(d, "ico.obj"), v, f, normals=v)
    g = np.array([[-5, -1, 5], [5, -1, 5], [5, -1, -5], [-5, -1, -5]], np.float64)
    write_obj(os.path.join(d, "ground.obj"), g, [[0, 1, 2], [0, 2, 3]], normals=np.tile([0, 1.0, 0], (4, 1)))
    scene = {"options": {"resolution": [64, 64], "pixelsamples": 8, "lightsamples": 1, "mindepth": 6,
                         "maxdepth": 6, "filename": "sphere.exr"},
             "renderCam": {"fov": 0.36397, "transforms": [{"translate": [0, 0.6, 5]}, {"rotateX": -8}]},
             "materials": {"ground": {"type": "matteMaterial", "color": [0.5, 0.5, 0.5]},
                           "sphere": {"type": "kelemenMaterial", "diffusecolor": [0.6, 0.6, 0.6],
                                      "speccolor": [1, 1, 1], "reflectance": 0.5, "roughness": 0.2}},
             "objects": {"a_ground": {"type": "geometry", "path": "ground.obj", "name": "g", "material": "ground",
                                      "transforms": [], "subdlevels": 0},
                         "b_sphere": {"type": "geometry", "path": "ico.obj", "name": "s", "material": "sphere",
                                      "transforms": [], "subdlevels": 4},
                         "c_light": {"type": "light", "name": "l", "scaleX": 0.5, "scaleY": 0.5, "exposure": 1.0,
                                     "color": [8, 8, 8],
                                     "transforms": [{"translate": [-2, 3, 1]}, {"rotateX": -90}]}}}
    path = os.path.join(d, "sphere.json")
    json.dump(scene, open(path, "w"))
    gpu, cpu, m2 = _render_both(ctx, kelemen_tables, oracle_lib, path, 8)
    _check(gpu, cpu, m2, 8)
    assert gpu[..., 3].mean() > 0.3   # the sphere and the ground fill the frame


def test_scenegraph_render_writes_the_film(ctx, kelemen_tables, oracle_lib, tmp_path):
    """PyAurora's render(scene) in-process: the scene file it writes renders like the oracle's
    CPU render of the loaded arrays, and the film goes to the options' filename as half EXR."""
    from aurora_b200 import scenes
    from aurora_b200.scenegraph import core
    from test_film_io import read_exr
    from test_scenegraph import box_scene_graph
    d = str(tmp_path)
    path = os.path.join(d, "graph.json")
    film = core.render(box_scene_graph(d, 48, 48, spp=8), path=path, ctx=ctx)
    data, opts, _ = scenes.load_scene_file(path)
    cpu, m2, _ = oracle_lib.OracleScene(data, kelemen_tables).render(8, opts.max_depth, opts.min_depth, opts.seed)
    _check(film, cpu, m2, 8)
    img, _ = read_exr(os.path.join(d, "box.exr"))
    np.testing.assert_array_equal(img, film.astype(np.float16).astype(np.float32))

"""The scene-file loader (aur_scene_file_read: the reference's JSON schema, OBJ meshes,
Loop subdivision, square lights) on the host, against the Python scene builder, an
independent numpy statement of Loop's rules, and the oracle's renders."""
import json
import math
import os

import numpy as np
import pytest

from aurora_b200 import _abi, scenes


def write_obj(path, verts, faces, normals=None, uvs=None):
    """faces index verts (and per-vertex normals / uvs) 0-based; writes 1-based v/vt/vn."""
    with open(path, "w") as f:
        for v in verts:
            f.write("v %.9g %.9g %.9g\n" % tuple(v))
        if uvs is not None:
            for t in uvs:
                f.write("vt %.9g %.9g\n" % tuple(t))
        if normals is not None:
            for n in normals:
                f.write("vn %.9g %.9g %.9g\n" % tuple(n))
        for tri in faces:
            if normals is not None and uvs is not None:
                f.write("f " + " ".join(f"{i + 1}/{i + 1}/{i + 1}" for i in tri) + "\n")
            elif normals is not None:
                f.write("f " + " ".join(f"{i + 1}//{i + 1}" for i in tri) + "\n")
            else:
                f.write("f " + " ".join(f"{i + 1}" for i in tri) + "\n")


def flat_obj(path, verts, faces):
    """Per-face flat normals, corners unshared (what the builder's normals=None gives)."""
    verts = np.asarray(verts, np.float64)
    v, n, fs = [], [], []
    for tri in faces:
        a, b, c = verts[tri[0]], verts[tri[1]], verts[tri[2]]
        fn = np.cross(b - a, c - a)
        fn /= np.linalg.norm(fn)
        for k in range(3):
            v.append(verts[tri[k]])
            n.append(fn)
        fs.append([len(v) - 3, len(v) - 2, len(v) - 1])
    write_obj(path, v, fs, normals=n)


METAL = dict(type_=_abi.MAT_METAL, specular=(0.9, 0.6, 0.3), roughness=0.3, roughness_b=0.6, mix=0.4,
             gain=(1.0, 0.9, 0.8))

WALLS = [("o0_floor", [(-1, -1, 1), (1, -1, 1), (1, -1, -1), (-1, -1, -1)], "m0_wall"),
         ("o1_ceiling", [(-1, 1, 1), (-1, 1, -1), (1, 1, -1), (1, 1, 1)], "m0_wall"),
         ("o2_back", [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)], "m0_wall"),
         ("o3_left", [(-1, -1, 1), (-1, -1, -1), (-1, 1, -1), (-1, 1, 1)], "m1_red"),
         ("o4_right", [(1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1)], "m2_green")]
BOXES = [(-0.35, -0.4, -0.3, 0.6, 1.2, 0.6, 15.0), (0.4, -0.7, 0.35, 0.6, 0.6, 0.6, -18.0)]


def write_box_scene(d, width=64, height=64, spp=4):
    """The box workload (with a metal material on the boxes) as a scene file."""
    objects = {}
    for name, corners, mat in WALLS:
        v, f = scenes.quad(*corners)
        flat_obj(os.path.join(d, name + ".obj"), v, f)
        objects[name] = {"type": "geometry", "path": name + ".obj", "name": name, "material": mat,
                         "transforms": [], "subdlevels": 0}
    bv, bf, _ = scenes.box_mesh()
    flat_obj(os.path.join(d, "box.obj"), bv, bf)
    for k, (x, y, z, sx, sy, sz, ry) in enumerate(BOXES):
        name = f"o{5 + k}_box{k}"
        objects[name] = {"type": "geometry", "path": "box.obj", "name": name, "material": "m3_box",
                         "transforms": [{"translate": [x, y, z]}, {"rotateY": ry}, {"scale": [sx, sy, sz]}],
                         "subdlevels": 0}
    objects["o7_light"] = {"type": "light", "name": "light", "scaleX": 0.25, "scaleY": 0.25, "exposure": 0.0,
                           "color": [17.0, 12.0, 4.0], "transforms": [{"translate": [0, 0.999, 0]}, {"rotateX": -90}]}
    scene = {
        "options": {"resolution": [width, height], "pixelsamples": spp, "lightsamples": 1, "mindepth": 5,
                    "maxdepth": 5, "filename": "box.exr"},
        "renderCam": {"fov": scenes.FOV40, "transforms": [{"translate": [0, 0, 3.5]}]},
        "materials": {
            "m0_wall": {"type": "matteMaterial", "color": [0.73, 0.73, 0.73]},
            "m1_red": {"type": "matteMaterial", "color": [0.65, 0.05, 0.05]},
            "m2_green": {"type": "matteMaterial", "color": [0.12, 0.45, 0.15]},
            "m3_box": {"type": "metalMaterial", "reflectance": list(METAL["specular"]), "roughnessA": 0.3,
                       "roughnessB": 0.6, "mix": 0.4, "gain": list(METAL["gain"])}},
        "objects": objects,
    }
    path = os.path.join(d, "box.json")
    with open(path, "w") as f:
        json.dump(scene, f, indent=1)
    return path


def corners(data):
    return data.verts[data.tri_vidx.astype(np.int64)]   # (ntri, 3, 3)


def test_box_scene_file_matches_builder(tmp_path, oracle_lib):
    path = write_box_scene(str(tmp_path))
    got, opts, info = scenes.load_scene_file(path)
    ref = scenes.box_scene(64, 64, spp=4, box_mat=METAL)
    assert (opts.spp, opts.min_depth, opts.max_depth) == (4, 5, 5)
    assert info == {"output": "box.exr", "light_samples": 1}
    assert got.ntri == ref.ntri == 36 and (got.width, got.height) == (64, 64)
    assert got.fov == np.float32(ref.fov)
    np.testing.assert_array_equal(got.tri_attr, ref.tri_attr)
    np.testing.assert_array_equal(got.attr_material, ref.attr_material)
    np.testing.assert_allclose(got.attr_emission, ref.attr_emission, rtol=1e-7)
    np.testing.assert_allclose(corners(got), corners(ref), atol=2e-6)
    np.testing.assert_allclose(got.corner_normals, ref.corner_normals, atol=2e-6)
    assert len(got.materials) == len(ref.materials)
    for a, b in zip(got.materials, ref.materials):
        assert bytes(a) == bytes(b)
    assert len(got.lights) == 1
    np.testing.assert_allclose(np.array(got.lights[0].object_to_camera), np.array(ref.lights[0].object_to_camera),
                               atol=1e-6)
    # the same image from the oracle's CPU renders of both flattenings
    tables = np.zeros((21, 64, 32), np.float32)
    a, _, _ = oracle_lib.OracleScene(got, tables).render(4, 5, 5, 1, want_m2=False)
    b, _, _ = oracle_lib.OracleScene(ref, tables).render(4, 5, 5, 1, want_m2=False)
    assert abs(a[..., :3].mean() - b[..., :3].mean()) < 1e-3 * b[..., :3].mean()
    assert np.mean(np.abs(a - b) > 1e-4) < 0.02


def icosahedron():
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                  (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    _, f = scenes.icosphere(0)
    return v, f


def loop_once_and_limit(v, f):
    """Independent float64 statement of one Loop level on a closed mesh, then the limit
    positions: even (1 - n b) P + b sum, odd 3/8 + 1/8, limit gamma = 1/(n + 3/(8 b))."""
    nv = len(v)
    nbr = [set() for _ in range(nv)]
    opp = {}
    for tri in f:
        for k in range(3):
            a, b, c = tri[k], tri[(k + 1) % 3], tri[(k + 2) % 3]
            nbr[a].add(b); nbr[b].add(a)
            opp.setdefault((min(a, b), max(a, b)), []).append(c)
    beta = lambda n: 3 / 16 if n == 3 else 3 / (8 * n)
    even = np.array([(1 - len(nbr[i]) * beta(len(nbr[i]))) * v[i] + beta(len(nbr[i])) * v[list(nbr[i])].sum(0)
                     for i in range(nv)])
    edges = sorted(opp)
    eid = {e: nv + j for j, e in enumerate(edges)}
    odd = np.array([3 / 8 * (v[a] + v[b]) + 1 / 8 * (v[opp[(a, b)][0]] + v[opp[(a, b)][1]]) for a, b in edges])
    P = np.concatenate([even, odd])
    faces = []
    for tri in f:
        a, b, c = tri
        ab, bc, ca = eid[(min(a, b), max(a, b))], eid[(min(b, c), max(b, c))], eid[(min(c, a), max(c, a))]
        faces += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
    nbr2 = [set() for _ in range(len(P))]
    for tri in faces:
        for k in range(3):
            nbr2[tri[k]].add(tri[(k + 1) % 3]); nbr2[tri[(k + 1) % 3]].add(tri[k])
    gamma = lambda n: 1 / (n + 3 / (8 * beta(n)))
    lim = np.array([(1 - len(nbr2[i]) * gamma(len(nbr2[i]))) * P[i] + gamma(len(nbr2[i])) * P[list(nbr2[i])].sum(0)
                    for i in range(len(P))])
    return lim


def write_single(d, obj_name, levels, extra_objects=None, materials=None, shaders=None):
    scene = {"options": {"resolution": [16, 16], "pixelsamples": 1, "lightsamples": 1, "mindepth": 3,
                         "maxdepth": 3, "filename": "x.exr"},
             "renderCam": {"fov": 0.5, "transforms": [{"translate": [0, 0, 5]}]},
             "materials": materials or {"m": {"type": "matteMaterial", "color": [0.5, 0.5, 0.5]}},
             "objects": {"g": {"type": "geometry", "path": obj_name, "name": "g", "material": "m",
                               "transforms": [], "subdlevels": levels}}}
    if shaders:
        scene["shaders"] = shaders
    if extra_objects:
        scene["objects"].update(extra_objects)
    p = os.path.join(d, "s.json")
    with open(p, "w") as f:
        json.dump(scene, f)
    return p


def test_loop_subdivision_of_icosahedron(tmp_path):
    v, f = icosahedron()
    write_obj(str(tmp_path / "ico.obj"), v, f, normals=v)
    for levels in (1, 2, 3):
        data, _, _ = scenes.load_scene_file(write_single(str(tmp_path), "ico.obj", levels))
        assert data.ntri == 20 * 4 ** levels
        P = corners(data).reshape(-1, 3).astype(np.float64) - np.array([0, 0, -5.0])   # undo the camera
        r = np.linalg.norm(P, axis=1)
        # the limit surface of the unit icosahedron: an original vertex lands at
        # 1/2 P + 1/10 (sum of its 5 neighbours) = 0.7236 P; the rest within 3%
        assert 0.70 < r.min() and r.max() < 0.724 and r.max() - r.min() < 0.03 * r.mean()
        n = data.corner_normals.reshape(-1, 3)
        assert np.min(np.sum(n * P, 1) / (np.linalg.norm(n, axis=1) * r)) > 0.99   # limit normals point outward
        # closed: every edge of the welded mesh is shared by exactly two triangles
        e = np.sort(np.concatenate([data.tri_vidx[:, [0, 1]], data.tri_vidx[:, [1, 2]], data.tri_vidx[:, [2, 0]]]), 1)
        _, cnt = np.unique(e, axis=0, return_counts=True)
        assert np.all(cnt == 2)
    # one level against the independent numpy statement (same positions as a set)
    data, _, _ = scenes.load_scene_file(write_single(str(tmp_path), "ico.obj", 1))
    got = np.unique(np.round(data.verts.astype(np.float64) - np.array([0, 0, -5.0]), 5), axis=0)
    want = np.unique(np.round(loop_once_and_limit(v, f), 5), axis=0)
    assert got.shape == want.shape
    np.testing.assert_allclose(got, want, atol=2e-5)


def test_loop_subdivision_keeps_planar_boundary_meshes_planar(tmp_path):
    v = np.array([(-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0), (0, 0, 0)], np.float64)
    f = np.array([[0, 1, 4], [1, 2, 4], [2, 3, 4], [3, 0, 4]])
    uv = (v[:, :2] + 1) / 2
    write_obj(str(tmp_path / "sq.obj"), v, f, normals=np.tile([0, 0, 1.0], (5, 1)), uvs=uv)
    data, _, _ = scenes.load_scene_file(write_single(str(tmp_path), "sq.obj", 2))
    assert data.ntri == 4 * 16
    P = corners(data).reshape(-1, 3)
    assert np.all(np.abs(P[:, 2] + 5.0) < 1e-6)
    assert np.all(np.abs(P[:, :2]) <= 1.0 + 1e-6)
    n = data.corner_normals.reshape(-1, 3)
    n = n / np.linalg.norm(n, axis=1, keepdims=True)
    assert np.all(np.abs(np.abs(n[:, 2]) - 1) < 1e-5)
    uvs = data.corner_uvs.reshape(-1, 2)
    assert uvs.min() >= -1e-6 and uvs.max() <= 1 + 1e-6 and uvs.std() > 0.1


def write_pfm(path, rgb):
    h, w, _ = rgb.shape
    with open(path, "wb") as f:
        f.write(b"PF\n%d %d\n-1.0\n" % (w, h))
        f.write(np.ascontiguousarray(rgb[::-1], "<f4").tobytes())   # rows bottom to top


def test_texture_shader_and_kelemen_material(tmp_path):
    v, f = scenes.quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0))
    write_obj(str(tmp_path / "q.obj"), v, f, normals=np.tile([0, 0, 1.0], (4, 1)), uvs=(v[:, :2] + 1) / 2)
    tex = np.random.default_rng(3).uniform(0, 1, size=(8, 16, 3)).astype(np.float32)
    write_pfm(str(tmp_path / "t.pfm"), tex)
    mats = {"m": {"type": "kelemenMaterial", "diffusecolor": "tex", "speccolor": [1, 1, 1], "reflectance": 0.5,
                  "roughness": 0.2}}
    shaders = {"tex": {"attributetype": "color", "type": "texture2DShader", "texturename": "t.pfm"}}
    data, _, _ = scenes.load_scene_file(write_single(str(tmp_path), "q.obj", 0, materials=mats, shaders=shaders))
    assert len(data.textures) == 1
    np.testing.assert_array_equal(data.textures[0], tex)           # top row first, as Texture2D reads it
    m = data.materials[0]
    assert m.type == _abi.MAT_KELEMEN and m.diffuse_tex == 0 and m.specular_tex == -1 and m.roughness_tex == -1
    assert m.reflectance == np.float32(0.5) and m.roughness == np.float32(0.2)


def test_triplanar_shader_normal_map_and_object_transform(tmp_path):
    """triplanarTextureShader (scale), a normal map from a shader and a constant one, and
    each attribute's cameraToObject (the inverse of its camera-space transform)."""
    v, f = scenes.quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0))
    write_obj(str(tmp_path / "q.obj"), v, f, normals=np.tile([0, 0, 1.0], (4, 1)))
    tex = np.random.default_rng(4).uniform(0, 1, size=(4, 8, 3)).astype(np.float32)
    write_pfm(str(tmp_path / "t.pfm"), tex)
    shaders = {"tri": {"attributetype": "color", "type": "triplanarTextureShader", "texturename": "t.pfm",
                       "scale": 0.25},
               "rough": {"attributetype": "float", "type": "triplanarTextureShader", "texturename": "t.pfm",
                         "scale": 2.0},
               "nrm": {"attributetype": "color", "type": "texture2DShader", "texturename": "t.pfm"}}
    mats = {"m": {"type": "kelemenMaterial", "diffusecolor": "tri", "speccolor": [1, 1, 1], "reflectance": 0.5,
                  "roughness": "rough", "normalmap": "nrm"},
            "n": {"type": "matteMaterial", "color": [0.5, 0.5, 0.5], "normalmap": [0.1, 0.2, 0.9]}}
    p = write_single(str(tmp_path), "q.obj", 0, materials=mats, shaders=shaders)
    s = json.load(open(p))
    s["objects"]["g"]["transforms"] = [{"translate": [0.5, -1, 2]}, {"rotateY": 30}, {"scale": [2, 2, 2]}]
    s["objects"]["h"] = {"type": "geometry", "path": "q.obj", "name": "h", "material": "n", "transforms": [],
                         "subdlevels": 0}
    json.dump(s, open(p, "w"))
    data, _, _ = scenes.load_scene_file(p)
    names = sorted(shaders)                                        # shaders are visited in key order
    np.testing.assert_array_equal(data.tex_triplanar_scale,
                                  np.array([shaders[k].get("scale", 0.0) for k in names], np.float32))
    m, n = data.materials[0], data.materials[1]
    assert m.diffuse_tex == names.index("tri") and m.roughness_tex == names.index("rough")
    assert m.normal_kind == _abi.NORMAL_TEXTURE and m.normal_tex == names.index("nrm")
    assert n.normal_kind == _abi.NORMAL_CONSTANT and n.normal_tex == -1
    np.testing.assert_array_equal(np.array(n.normal), np.array([0.1, 0.2, 0.9], np.float32))
    # cameraToObject maps the camera-space corners back to the object's quad
    assert data.attr_c2o.shape == (2, 16)
    c2o = data.attr_c2o[0].reshape(4, 4).astype(np.float64)
    P = corners(data)[data.tri_attr == 0].reshape(-1, 3).astype(np.float64)
    obj = P @ c2o[:3, :3].T + c2o[:3, 3]
    np.testing.assert_allclose(np.abs(obj[:, :2]), 1.0, atol=1e-5)
    np.testing.assert_allclose(obj[:, 2], 0.0, atol=1e-5)


@pytest.mark.parametrize("mutate,status", [
    (lambda s: s.pop("options"), _abi.ERR_PARSE),
    (lambda s: s["materials"].update({"m": {"type": "glassMaterial"}}), _abi.ERR_PARSE),
    (lambda s: s["materials"].update({"m": {"type": "matteMaterial", "color": [1, 1, 1], "normalmap": "n"}}),
     _abi.ERR_PARSE),
    (lambda s: s.update({"shaders": {"t": {"attributetype": "color", "type": "triplanarTextureShader",
                                           "texturename": "t.pfm", "scale": 0}}}), _abi.ERR_PARSE),
    (lambda s: s.update({"shaders": {"t": {"attributetype": "color", "type": "noiseShader",
                                           "texturename": "t.pfm"}}}), _abi.ERR_PARSE),
    (lambda s: s["objects"].update({"e": {"type": "envlight"}}), _abi.ERR_PARSE),
    (lambda s: s["objects"].update({"e": {"type": "envlight", "transforms": [], "exposure": 0, "color": [1, 1, 1],
                                          "envmap": "sky.exr"}}), _abi.ERR_IO),
    (lambda s: s["objects"].update({"e": {"type": "envlight", "transforms": [], "exposure": 0, "color": [1, 1, 1],
                                          "envmap": "sky.hdr"}}), _abi.ERR_UNSUPPORTED),
    (lambda s: s["objects"]["g"].update({"material": "nope"}), _abi.ERR_PARSE),
    (lambda s: s["objects"]["g"].update({"path": "missing.obj"}), _abi.ERR_IO),
    (lambda s: s["materials"]["m"].update({"color": "noshader"}), _abi.ERR_PARSE),
    (lambda s: s["options"].update({"resolution": [16]}), _abi.ERR_PARSE),
])
def test_scene_file_errors(tmp_path, mutate, status):
    v, f = scenes.quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0))
    write_obj(str(tmp_path / "q.obj"), v, f, normals=np.tile([0, 0, 1.0], (4, 1)))
    p = write_single(str(tmp_path), "q.obj", 0)
    s = json.load(open(p))
    mutate(s)
    json.dump(s, open(p, "w"))
    with pytest.raises(_abi.AuroraError) as e:
        scenes.load_scene_file(p)
    assert e.value.status == status


def test_json_syntax_error_names_the_line(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text('{\n "options": {\n  "resolution": [16, 16],\n  oops\n }\n}\n')
    with pytest.raises(_abi.AuroraError) as e:
        scenes.load_scene_file(str(p))
    assert e.value.status == _abi.ERR_PARSE and "line 4" in str(e.value)


def test_light_samples_option(tmp_path):
    """The file's lightsamples reach the render options; the (wavefront) renderer the file
    selects takes any number of paths per camera sample."""
    v, f = scenes.quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0))
    write_obj(str(tmp_path / "q.obj"), v, f, normals=np.tile([0, 0, 1.0], (4, 1)))
    p = write_single(str(tmp_path), "q.obj", 0)
    s = json.load(open(p))
    s["options"]["lightsamples"] = 8
    json.dump(s, open(p, "w"))
    _, opts, info = scenes.load_scene_file(p)
    assert opts.light_samples == 8 and opts.mode == _abi.RENDER_WAVEFRONT and info["light_samples"] == 8
    s["options"]["lightsamples"] = 1
    json.dump(s, open(p, "w"))
    _, opts, _ = scenes.load_scene_file(p)
    assert opts.light_samples == 1 and opts.mode == _abi.RENDER_WAVEFRONT


def test_other_image_formats_are_refused(tmp_path):
    v, f = scenes.quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0))
    write_obj(str(tmp_path / "q.obj"), v, f, normals=np.tile([0, 0, 1.0], (4, 1)))
    (tmp_path / "t.png").write_bytes(b"\x89PNG")
    shaders = {"tex": {"attributetype": "color", "type": "texture2DShader", "texturename": "t.png"}}
    mats = {"m": {"type": "matteMaterial", "color": "tex"}}
    with pytest.raises(_abi.AuroraError) as e:
        scenes.load_scene_file(write_single(str(tmp_path), "q.obj", 0, materials=mats, shaders=shaders))
    assert e.value.status == _abi.ERR_UNSUPPORTED and "OpenEXR" in str(e.value)


def test_glass_material(tmp_path):
    v, f = scenes.quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0))
    write_obj(str(tmp_path / "q.obj"), v, f, normals=np.tile([0, 0, 1.0], (4, 1)))
    mats = {"m": {"type": "glassMaterial", "specColor": [1, 1, 1], "transmitColor": [0.9, 0.8, 0.7],
                  "reflectance": 0.04, "ior": 1.5}}
    data, _, _ = scenes.load_scene_file(write_single(str(tmp_path), "q.obj", 0, materials=mats))
    m = data.materials[0]
    assert m.type == _abi.MAT_GLASS and m.ior == np.float32(1.5) and m.reflectance == np.float32(0.04)
    assert tuple(m.specular) == (1, 1, 1) and np.allclose(tuple(m.diffuse), (0.9, 0.8, 0.7))


def test_environment_light_file(tmp_path):
    v, f = scenes.quad((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0))
    write_obj(str(tmp_path / "q.obj"), v, f, normals=np.tile([0, 0, 1.0], (4, 1)))
    env = np.random.default_rng(4).uniform(0, 2, (8, 16, 3)).astype(np.float32)
    write_pfm(str(tmp_path / "sky.pfm"), env)
    p = write_single(str(tmp_path), "q.obj", 0, extra_objects={
        "sky": {"type": "envlight", "name": "sky", "transforms": [], "exposure": 1.0, "color": [1, 1, 1],
                "envmap": "sky.pfm"}})
    data, _, _ = scenes.load_scene_file(p)
    assert len(data.lights) == 1 and data.lights[0].type == _abi.LIGHT_ENV and data.lights[0].tex == 0
    np.testing.assert_array_equal(data.textures[0], env)
    # the camera-to-world matrix of the render camera (translate 0 0 5)
    m = np.array(data.lights[0].object_to_camera).reshape(4, 4)
    np.testing.assert_allclose(m, [[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 5], [0, 0, 0, 1]])
    assert data.attr_material[-1] == len(data.materials) - 1 and data.ntri == 2

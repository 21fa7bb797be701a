"""Scene assembly and the synthetic workloads the renderer is measured on.

``SceneBuilder`` flattens objects and lights into the camera-space soup that
Renderer::buildRenderEnvironment produces (Aurora/src/frontend/renderer.cpp:99-145):
objects first (attribute i = object i), then the light shapes (attribute
nobj + j, a constant black material and emission colour * 2^exposure),
per-corner normals and uvs (TriangleMesh::makeEmbree, triangleMesh.cpp:57-81)
and the square lights' quads (SquareLight::shape, squareLight.cpp:78-93).

The five workloads (box scene, Kelemen icosphere, large terrain, 64-scene
batch, differentiable texture scene) are generated in code from their seeds;
no external data is read. Camera space: eye at the origin looking down -z,
+y up; the ``fov`` value is the reference's slope factor (camera.cpp:51-52),
so a field of view of F degrees is fov = tan(F/2).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import _abi

F32 = np.float32


# ----------------------------------------------------------------------------- geometry helpers
def look_at(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """World-to-camera matrix (float64) for a camera at `eye` looking at `target` (-z forward)."""
    eye, target, up = (np.asarray(v, np.float64) for v in (eye, target, up))
    f = target - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, up)
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3] = r, u, -f
    m[:3, 3] = -m[:3, :3] @ eye
    return m


def translate(x, y, z) -> np.ndarray:
    m = np.eye(4)
    m[:3, 3] = (x, y, z)
    return m


def rot_x(deg) -> np.ndarray:
    c, s = math.cos(math.radians(deg)), math.sin(math.radians(deg))
    m = np.eye(4)
    m[1, 1], m[1, 2], m[2, 1], m[2, 2] = c, -s, s, c
    return m


def rot_y(deg) -> np.ndarray:
    c, s = math.cos(math.radians(deg)), math.sin(math.radians(deg))
    m = np.eye(4)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = c, s, -s, c
    return m


def scale(x, y, z) -> np.ndarray:
    return np.diag([x, y, z, 1.0])


def quad(p0, p1, p2, p3):
    """Two triangles (p0,p1,p2), (p0,p2,p3)."""
    v = np.array([p0, p1, p2, p3], np.float64)
    return v, np.array([[0, 1, 2], [0, 2, 3]], np.int64)


def box_mesh():
    """Unit cube [-0.5,0.5]^3 as 12 triangles with flat (per-face) vertices."""
    faces = [((-1, 0, 0), [(0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0)]),
             ((1, 0, 0), [(1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1)]),
             ((0, -1, 0), [(0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1)]),
             ((0, 1, 0), [(0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0)]),
             ((0, 0, -1), [(0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0)]),
             ((0, 0, 1), [(0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)])]
    verts, idx, nrm = [], [], []
    for n, corners in faces:
        b = len(verts)
        for c in corners:
            verts.append(np.array(c, np.float64) - 0.5)
            nrm.append(n)
        idx += [[b, b + 1, b + 2], [b, b + 2, b + 3]]
    return np.array(verts), np.array(idx, np.int64), np.array(nrm, np.float64)


def icosphere(level: int):
    """Icosahedron with `level` midpoint subdivisions projected to the unit sphere (20*4^level triangles)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = np.array(v, np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    faces = np.array(f, np.int64)
    for _ in range(level):
        # unique edge midpoints
        e = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        mids = verts[uniq[:, 0]] + verts[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = len(verts)
        verts = np.concatenate([verts, mids])
        m = inv.reshape(3, -1).T + base           # midpoints of edges (01, 12, 20) per face
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        faces = np.concatenate([np.stack([a, m01, m20], 1), np.stack([b, m12, m01], 1),
                                np.stack([c, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return verts, faces


def value_noise_fbm(x, z, octaves, amplitude, seed, base_freq=0.5):
    """Fractional Brownian motion of smooth value noise (lattice values in [-1,1])."""
    rng = np.random.default_rng(seed)
    h = np.zeros_like(x)
    amp, freq = amplitude, base_freq
    for _ in range(octaves):
        lat = rng.uniform(-1.0, 1.0, size=(257, 257))
        fx, fz = (x * freq) % 256.0, (z * freq) % 256.0
        ix, iz = np.floor(fx).astype(np.int64), np.floor(fz).astype(np.int64)
        tx, tz = fx - ix, fz - iz
        sx, sz = tx * tx * (3 - 2 * tx), tz * tz * (3 - 2 * tz)
        a = lat[ix, iz] * (1 - sx) + lat[ix + 1, iz] * sx
        b = lat[ix, iz + 1] * (1 - sx) + lat[ix + 1, iz + 1] * sx
        h += amp * (a * (1 - sz) + b * sz)
        amp *= 0.5
        freq *= 2.0
    return h


# ----------------------------------------------------------------------------- scene data
@dataclass
class SceneData:
    """Flattened camera-space scene (the inputs of aur_scene_create)."""
    verts: np.ndarray
    tri_vidx: np.ndarray
    tri_attr: np.ndarray
    corner_normals: np.ndarray
    corner_uvs: np.ndarray
    attr_material: np.ndarray
    attr_emission: np.ndarray
    materials: list
    lights: list
    textures: list
    fov: float
    width: int
    height: int
    name: str = ""
    render: dict = field(default_factory=dict)   # spp, max_depth, min_depth, seed of the workload
    tex_triplanar_scale: object = None   # (ntex,) float32: 0 = uv shader, > 0 = triplanar scale; None = all uv
    attr_c2o: object = None              # (nattr, 16) float32 camera-to-object per attribute; None = identity
    _keep: list = field(default_factory=list, repr=False)

    @property
    def ntri(self) -> int:
        return int(self.tri_vidx.shape[0])

    def texels(self) -> np.ndarray:
        if not self.textures:
            return np.zeros(0, np.float32)
        return np.concatenate([np.ascontiguousarray(t, np.float32).ravel() for t in self.textures])

    def desc(self) -> _abi.SceneDesc:
        mats = (_abi.MaterialDesc * len(self.materials))(*self.materials)
        lights = (_abi.LightDesc * max(1, len(self.lights)))(*self.lights)
        tex = self.texels()
        dims = np.array([[t.shape[1], t.shape[0]] for t in self.textures], np.int32).reshape(-1, 2)
        arrs = [np.ascontiguousarray(a) for a in (self.verts, self.tri_vidx, self.tri_attr, self.corner_normals,
                                                  self.corner_uvs, self.attr_material, self.attr_emission)]
        self._keep = [mats, lights, tex, dims] + arrs
        tscale = None if self.tex_triplanar_scale is None else np.ascontiguousarray(self.tex_triplanar_scale, F32)
        c2o = None if self.attr_c2o is None else np.ascontiguousarray(self.attr_c2o, F32).reshape(-1, 16)
        if tscale is not None:
            assert tscale.shape == (len(self.textures),)
            self._keep.append(tscale)
        if c2o is not None:
            assert c2o.shape[0] == len(self.attr_material)
            self._keep.append(c2o)
        d = _abi.SceneDesc()
        d.verts, d.nvert = arrs[0].ctypes.data, arrs[0].shape[0]
        d.tri_vidx, d.tri_attr = arrs[1].ctypes.data, arrs[2].ctypes.data
        d.corner_normals, d.corner_uvs, d.ntri = arrs[3].ctypes.data, arrs[4].ctypes.data, arrs[1].shape[0]
        d.attr_material, d.attr_emission, d.nattr = arrs[5].ctypes.data, arrs[6].ctypes.data, arrs[5].shape[0]
        d.materials, d.nmat = C.addressof(mats), len(self.materials)
        d.lights, d.nlight = C.addressof(lights), len(self.lights)
        d.texels = tex.ctypes.data if tex.size else None
        d.tex_dims = dims.ctypes.data if dims.size else None
        d.ntex = len(self.textures)
        d.fov, d.width, d.height = self.fov, self.width, self.height
        d.tex_triplanar_scale = tscale.ctypes.data if tscale is not None and tscale.size else None
        d.attr_camera_to_object = c2o.ctypes.data if c2o is not None else None
        return d

    def material_params(self) -> np.ndarray:
        """(nmat, 4): diffuse rgb + roughness, the differentiable per-material block."""
        return np.array([[m.diffuse[0], m.diffuse[1], m.diffuse[2], m.roughness] for m in self.materials],
                        np.float32)


def _mat(type_, diffuse=(0, 0, 0), specular=(0, 0, 0), gain=(1, 1, 1), roughness=0.0, roughness_b=0.0,
         reflectance=0.0, mix=0.0, diffuse_tex=-1, specular_tex=-1, roughness_tex=-1, ior=1.0, normal_tex=None,
         normal=None) -> _abi.MaterialDesc:
    """normal_tex: a texture index used as the normal map; normal: a constant normal-map colour."""
    kind = (_abi.NORMAL_TEXTURE if normal_tex is not None else
            _abi.NORMAL_CONSTANT if normal is not None else _abi.NORMAL_NONE)
    return _abi.MaterialDesc(type_, _abi.f3(*diffuse), _abi.f3(*specular), _abi.f3(*gain), roughness, roughness_b,
                             reflectance, mix, diffuse_tex, specular_tex, roughness_tex, ior, kind,
                             -1 if normal_tex is None else normal_tex, _abi.f3(*(normal or (0, 0, 0))))


def _xform_f32(m: np.ndarray, p: np.ndarray) -> np.ndarray:
    """Transform::operator()(Point) in float32 operation order (transform.cpp:196-204)."""
    m = m.astype(F32)
    x, y, z = (p[:, k].astype(F32) for k in range(3))
    out = []
    for r in range(3):
        out.append(((m[r, 0] * x + m[r, 1] * y) + m[r, 2] * z) + m[r, 3])
    return np.stack(out, 1).astype(F32)


class SceneBuilder:
    """Collects objects (world space) and lights and flattens them into camera space."""

    def __init__(self, width, height, fov, world_to_camera=None, name=""):
        self.width, self.height, self.fov, self.name = width, height, float(fov), name
        self.w2c = np.eye(4) if world_to_camera is None else np.asarray(world_to_camera, np.float64)
        self.materials: list = []
        self.textures: list = []
        self.tex_scales: list = []  # triplanar scale per texture (0: uv lookup)
        self.objects: list = []     # (verts_cam f32, faces, corner normals f32, corner uvs f32, material, c2o)
        self.lights: list = []      # (LightDesc, shape verts cam f32, faces, corner normals, emission)

    def material(self, type_, **kw) -> int:
        self.materials.append(_mat(type_, **kw))
        return len(self.materials) - 1

    def texture(self, rgb: np.ndarray, triplanar_scale: float = 0.0) -> int:
        """An image (H, W, 3) as a texture shader: the uv lookup, or with triplanar_scale > 0 the
        triplanar projection in the object space of the mesh that uses it."""
        self.textures.append(np.ascontiguousarray(rgb, np.float32))
        self.tex_scales.append(float(triplanar_scale))
        return len(self.textures) - 1

    def mesh(self, verts, faces, material, normals=None, uvs=None, object_to_world=None):
        """verts (n,3) object space; normals per vertex (None: flat face normals); uvs (n,2)."""
        o2w = np.eye(4) if object_to_world is None else object_to_world
        o2c = self.w2c @ o2w
        verts = np.asarray(verts, np.float64)
        faces = np.asarray(faces, np.int64)
        used = np.unique(faces)
        if used.size < verts.shape[0]:          # keep only the referenced vertices
            remap = np.zeros(verts.shape[0], np.int64)
            remap[used] = np.arange(used.size)
            verts = verts[used]
            normals = None if normals is None else np.asarray(normals, np.float64)[used]
            uvs = None if uvs is None else np.asarray(uvs, np.float64)[used]
            faces = remap[faces]
        vc = (verts @ o2c[:3, :3].T + o2c[:3, 3]).astype(F32)
        if normals is None:
            a, b, c = (verts[faces[:, k]] for k in range(3))
            fn = np.cross(b - a, c - a)
            fn /= np.maximum(np.linalg.norm(fn, axis=1, keepdims=True), 1e-30)
            cn = np.repeat(fn[:, None, :], 3, axis=1)
        else:
            cn = np.asarray(normals, np.float64)[faces]
        cn = (cn @ o2c[:3, :3].T).astype(F32).reshape(-1, 9)
        if uvs is None:
            cu = np.zeros((faces.shape[0], 6), F32)
        else:
            cu = np.asarray(uvs, np.float64)[faces].astype(F32).reshape(-1, 6)
        c2o = np.linalg.inv(o2c).astype(F32).ravel()            # AttributeState::cameraToObject
        self.objects.append((vc, faces, cn, cu, material, c2o))
        return len(self.objects) - 1

    def square_light(self, object_to_world, size_x, size_y, color, exposure=0.0):
        """SquareLight: quad [-sx,sx]x[-sy,sy] at z=0 emitting toward the object's -z."""
        o2c = self.w2c @ object_to_world
        ld = _abi.LightDesc()
        ld.type = _abi.LIGHT_SQUARE
        ld.tex = -1
        for k, v in enumerate(o2c.astype(F32).ravel()):
            ld.object_to_camera[k] = v
        ld.size_x, ld.size_y = size_x, size_y
        ld.color = _abi.f3(*color)
        ld.exposure = exposure
        p = np.array([[-size_x, -size_y, 0], [-size_x, size_y, 0], [size_x, size_y, 0], [size_x, -size_y, 0]], F32)
        pc = _xform_f32(o2c, p)
        faces = np.array([[0, 1, 3], [2, 1, 3]], np.int64)         # SquareLight::shape index order
        ln = np.cross((pc[0] - pc[1]).astype(np.float64), (pc[1] - pc[2]).astype(np.float64))
        ln /= np.linalg.norm(ln)
        n_shape = (o2c[:3, :3] @ ln).astype(F32)                  # makeEmbree transforms the normal again
        cn = np.tile(n_shape, (2, 3)).astype(F32)
        em = (np.array(color, F32) * F32(2.0 ** exposure)).astype(F32)
        self.lights.append((ld, pc, faces, cn, em))

    def sphere_light(self, center_world, radius, color, exposure=0.0, tessellation=2):
        """Sphere light (no reference counterpart): sampled analytically, visible as an icosphere."""
        c = (self.w2c @ np.append(np.asarray(center_world, np.float64), 1.0))[:3]
        ld = _abi.LightDesc()
        ld.type = _abi.LIGHT_SPHERE
        ld.tex = -1
        ld.center = _abi.f3(*c.astype(F32))
        ld.radius = radius
        ld.color = _abi.f3(*color)
        ld.exposure = exposure
        v, f = icosphere(tessellation)
        vc = (v * radius + c).astype(F32)
        cn = v[f].astype(F32).reshape(-1, 9)
        em = (np.array(color, F32) * F32(2.0 ** exposure)).astype(F32)
        self.lights.append((ld, vc, f, cn, em))

    def env_light(self, color=(1.0, 1.0, 1.0), exposure=0.0, texture=None):
        """InfiniteAreaLight: a constant colour, or a latitude-longitude env map (H, W, 3; row 0 is
        up) looked up in world directions. No geometry."""
        ld = _abi.LightDesc()
        ld.type = _abi.LIGHT_ENV
        c2w = np.linalg.inv(self.w2c).astype(F32)
        for k, v in enumerate(c2w.ravel()):
            ld.object_to_camera[k] = v
        ld.color = _abi.f3(*color)
        ld.exposure = exposure
        ld.tex = -1 if texture is None else self.texture(texture)
        self.lights.append((ld, None, None, None, np.ones(3, F32)))   # emission() = 1, unused

    def build(self, render=None) -> SceneData:
        const = len(self.materials)
        materials = list(self.materials) + [_mat(_abi.MAT_CONSTANT)]
        verts, faces, attr, cn, cu = [], [], [], [], []
        base = 0
        nobj = len(self.objects)
        for i, (vc, f, n, u, _, _) in enumerate(self.objects):
            verts.append(vc); faces.append(f + base); attr.append(np.full(len(f), i, np.int32))
            cn.append(n); cu.append(u); base += len(vc)
        for j, (ld, vc, f, n, em) in enumerate(self.lights):
            if vc is None:      # environment light: an attribute but no shape
                continue
            verts.append(vc); faces.append(f + base); attr.append(np.full(len(f), nobj + j, np.int32))
            cn.append(n); cu.append(np.zeros((len(f), 6), F32)); base += len(vc)
        attr_mat = np.array([o[4] for o in self.objects] + [const] * len(self.lights), np.int32)
        attr_em = np.array([[0, 0, 0]] * nobj + [l[4] for l in self.lights], F32).reshape(-1, 3)
        c2o = np.array([o[5] for o in self.objects] + [np.eye(4, dtype=F32).ravel()] * len(self.lights),
                       F32).reshape(-1, 16)
        scales = np.array(self.tex_scales, F32) if any(s != 0.0 for s in self.tex_scales) else None
        return SceneData(np.concatenate(verts).astype(F32), np.concatenate(faces).astype(np.uint32),
                         np.concatenate(attr), np.concatenate(cn).astype(F32), np.concatenate(cu).astype(F32),
                         attr_mat, attr_em, materials, [l[0] for l in self.lights], list(self.textures),
                         self.fov, self.width, self.height, self.name, dict(render or {}), scales, c2o)


def load_scene_file(path: str):
    """Reads a scene file of the reference's JSON schema (options, renderCam, shaders,
    materials, objects with OBJ meshes and square lights) with the library's host-side
    loader (aur_scene_file_read; no device work). Returns (SceneData, RenderOpts, info)
    where info holds the file's output name and light-sample count."""
    h = C.c_void_p()
    _abi.check(_abi.lib().aur_scene_file_read(path.encode(), C.byref(h)), "aur_scene_file_read")
    try:
        d = _abi.SceneDesc()
        o = _abi.RenderOpts()
        _abi.check(_abi.lib().aur_scene_file_desc(h, C.byref(d), C.byref(o)), "aur_scene_file_desc")

        def arr(ptr, n, dtype, shape):
            if n == 0 or not ptr:
                return np.zeros([0 if x == -1 else x for x in shape], dtype)
            ct = {np.float32: C.c_float, np.uint32: C.c_uint32, np.int32: C.c_int32}[dtype]
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(n,)).copy().reshape(shape)
        verts = arr(d.verts, 3 * d.nvert, np.float32, (d.nvert, 3))
        vidx = arr(d.tri_vidx, 3 * d.ntri, np.uint32, (d.ntri, 3))
        tattr = arr(d.tri_attr, d.ntri, np.int32, (d.ntri,))
        cn = arr(d.corner_normals, 9 * d.ntri, np.float32, (d.ntri, 9))
        cu = arr(d.corner_uvs, 6 * d.ntri, np.float32, (d.ntri, 6))
        amat = arr(d.attr_material, d.nattr, np.int32, (d.nattr,))
        aem = arr(d.attr_emission, 3 * d.nattr, np.float32, (d.nattr, 3))
        mats = [_abi.MaterialDesc.from_buffer_copy(C.cast(d.materials, C.POINTER(_abi.MaterialDesc))[i])
                for i in range(d.nmat)]
        lights = [_abi.LightDesc.from_buffer_copy(C.cast(d.lights, C.POINTER(_abi.LightDesc))[i])
                  for i in range(d.nlight)]
        dims = arr(d.tex_dims, 2 * d.ntex, np.int32, (d.ntex, 2))
        texels = arr(d.texels, int(3 * (dims[:, 0] * dims[:, 1]).sum()) if d.ntex else 0, np.float32, (-1,))
        textures, off = [], 0
        for w_, h_ in dims:
            n = 3 * int(w_) * int(h_)
            textures.append(texels[off:off + n].reshape(int(h_), int(w_), 3))
            off += n
        tscale = arr(d.tex_triplanar_scale, d.ntex, np.float32, (d.ntex,)) if d.tex_triplanar_scale else None
        c2o = arr(d.attr_camera_to_object, 16 * d.nattr, np.float32, (d.nattr, 16)) if d.attr_camera_to_object \
            else None
        info = {"output": _abi.lib().aur_scene_file_output(h).decode(),
                "light_samples": int(_abi.lib().aur_scene_file_light_samples(h))}
        data = SceneData(verts, vidx, tattr, cn, cu, amat, aem, mats, lights, textures, float(d.fov), int(d.width),
                         int(d.height), os.path.basename(path),
                         dict(spp=o.spp, max_depth=o.max_depth, min_depth=o.min_depth, seed=0), tscale, c2o)
        return data, o, info
    finally:
        _abi.lib().aur_scene_file_destroy(h)


FOV40 = math.tan(math.radians(20.0))


# ----------------------------------------------------------------------------- workloads
def box_scene(width=256, height=256, spp=16, max_depth=5, seed=1, rng_seed=None, wall=(0.73, 0.73, 0.73),
              red=(0.65, 0.05, 0.05), green=(0.12, 0.45, 0.15), box_mat=None, lift=0.0) -> SceneData:
    """Closed box: 5 wall quads of side 2 (10 tris), two rotated boxes (24 tris), a 0.5x0.5 ceiling
    light of radiance (17,12,4); Lambert walls, Cook-Torrance boxes (roughness 0.3, F0 0.04);
    40 degree pinhole; roulette off (min_depth = max_depth). With `rng_seed` the box poses and
    materials are drawn from that seed (the 64-scene batch). `lift` raises the boxes off the floor
    (their bottom faces otherwise lie in the floor's plane, where rays inside a transparent box
    hit both at exactly the same distance)."""
    b = SceneBuilder(width, height, FOV40, world_to_camera=translate(0, 0, -3.5), name="box")
    r = np.random.default_rng(rng_seed) if rng_seed is not None else None
    if r is not None:
        wall = tuple(r.uniform(0.5, 0.8, 3))
        red = (r.uniform(0.5, 0.8), r.uniform(0.02, 0.1), r.uniform(0.02, 0.1))
        green = (r.uniform(0.05, 0.2), r.uniform(0.3, 0.6), r.uniform(0.05, 0.2))
    m_wall = b.material(_abi.MAT_MATTE, diffuse=wall)
    m_red = b.material(_abi.MAT_MATTE, diffuse=red)
    m_green = b.material(_abi.MAT_MATTE, diffuse=green)
    if box_mat is None:
        rough = 0.3 if r is None else float(r.uniform(0.1, 0.6))
        col = (0.8, 0.8, 0.8) if r is None else tuple(r.uniform(0.4, 0.9, 3))
        m_box = b.material(_abi.MAT_COOKTORRANCE, specular=col, roughness=rough, reflectance=0.04)
    else:
        m_box = b.material(**box_mat)
    for v, mat in (([(-1, -1, 1), (1, -1, 1), (1, -1, -1), (-1, -1, -1)], m_wall),     # floor
                   ([(-1, 1, 1), (-1, 1, -1), (1, 1, -1), (1, 1, 1)], m_wall),         # ceiling
                   ([(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)], m_wall),     # back
                   ([(-1, -1, 1), (-1, -1, -1), (-1, 1, -1), (-1, 1, 1)], m_red),      # left
                   ([(1, -1, -1), (1, -1, 1), (1, 1, 1), (1, 1, -1)], m_green)):       # right
        verts, faces = quad(*v)
        b.mesh(verts, faces, mat)
    bv, bf, bn = box_mesh()
    if r is None:
        poses = [(-0.35, -0.4, -0.3, 0.6, 1.2, 0.6, 15.0), (0.4, -0.7, 0.35, 0.6, 0.6, 0.6, -18.0)]
    else:
        poses = []
        for k in range(2):
            h = float(r.uniform(0.4, 1.3))
            x = (0.4 if k else -0.35) + float(r.uniform(-0.15, 0.15))
            poses.append((x, -1 + h / 2, float(r.uniform(-0.5, 0.4)), 0.55, h, 0.55, float(r.uniform(-40, 40))))
    for (x, y, z, sx, sy, sz, ry) in poses:
        o2w = translate(x, y + lift, z) @ rot_y(ry) @ scale(sx, sy, sz)
        b.mesh(bv, bf, m_box, normals=None, object_to_world=o2w)
    b.square_light(translate(0, 0.999, 0) @ rot_x(-90.0), 0.25, 0.25, (17.0, 12.0, 4.0), 0.0)
    return b.build(render=dict(spp=spp, max_depth=max_depth, min_depth=max_depth, seed=seed))


def sphere_scene(width=512, height=512, spp=64, max_depth=6, seed=2, ground_texture=None, env=None,
                 sphere_mat=None) -> SceneData:
    """Icosphere (5 subdivisions, 20480 tris, radius 1) with a Kelemen material (roughness 0.2,
    reflectance 0.5, diffuse 0.6) on a 10x10 Lambert 0.5 ground, lit by one quad light and one
    sphere light. Roulette off. `env` adds an environment light (SceneBuilder.env_light
    arguments); `sphere_mat` replaces the sphere's material (_mat arguments)."""
    b = SceneBuilder(width, height, FOV40, world_to_camera=look_at((0, 1.2, 5.0), (0, 0, 0)), name="sphere")
    tex = -1
    if ground_texture is not None:
        tex = b.texture(ground_texture)
    m_ground = b.material(_abi.MAT_MATTE, diffuse=(0.5, 0.5, 0.5), diffuse_tex=tex)
    if sphere_mat is None:
        m_sphere = b.material(_abi.MAT_KELEMEN, diffuse=(0.6, 0.6, 0.6), specular=(1.0, 1.0, 1.0), roughness=0.2,
                              reflectance=0.5)
    else:
        m_sphere = b.material(**sphere_mat)
    gv = np.array([[-5, -1, 5], [5, -1, 5], [5, -1, -5], [-5, -1, -5]], np.float64)
    guv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float64)
    b.mesh(gv, np.array([[0, 1, 2], [0, 2, 3]]), m_ground, normals=np.tile([0, 1, 0], (4, 1)), uvs=guv)
    v, f = icosphere(5)
    b.mesh(v, f, m_sphere, normals=v)
    b.square_light(translate(-2.0, 3.0, 1.0) @ rot_x(-90.0), 0.5, 0.5, (8.0, 8.0, 8.0), 0.0)
    b.sphere_light((2.2, 1.2, 1.5), 0.3, (30.0, 24.0, 18.0), 0.0)
    if env is not None:
        b.env_light(**env)
    return b.build(render=dict(spp=spp, max_depth=max_depth, min_depth=max_depth, seed=seed))


def mirror_quad_scene(width=16, height=16, spp=4, max_depth=1, seed=9, spec=(0.8, 0.6, 0.4),
                      env=(0.5, 1.0, 2.0), exposure=0.0) -> SceneData:
    """A 4x4 mirror quad (glassMaterial with reflectance 1: always SpecMirror) facing the camera at
    distance 3, filling the view, under a constant environment light and nothing else. Every
    camera ray hits the mirror and its reflection escapes, so every pixel is env * 2^exposure *
    spec, at any max_depth (the last escape happens after the last shaded vertex at max_depth 1)."""
    b = SceneBuilder(width, height, 0.4, name="mirror")
    m = b.material(_abi.MAT_GLASS, specular=spec, diffuse=(1.0, 1.0, 1.0), reflectance=1.0, ior=1.5)
    verts, faces = quad((-2, -2, -3), (2, -2, -3), (2, 2, -3), (-2, 2, -3))
    b.mesh(verts, faces, m)
    b.env_light(color=env, exposure=exposure)
    return b.build(render=dict(spp=spp, max_depth=max_depth, min_depth=max_depth, seed=seed))


def shader_scene(width=128, height=128, spp=16, max_depth=6, seed=3, tex_seed=11, sphere_level=4) -> SceneData:
    """Texture-shader workload: triplanar colour and roughness shaders, a normal-map texture and a
    constant normal map. A Kelemen sphere (triplanar diffuse, scale 0.5; triplanar roughness,
    scale 0.8; constant normal map (0.1, 0.05, 1)) and a rotated Lambert box (triplanar colour,
    scale 0.3, projected in the box's object space) on a 10x10 Lambert ground (triplanar
    colour, scale 0.7; a normal-map texture over its uvs), one quad light and one sphere light.
    Textures uniform random (seed `tex_seed`). Roulette off."""
    r = np.random.default_rng(tex_seed)
    b = SceneBuilder(width, height, FOV40, world_to_camera=look_at((0, 1.2, 5.0), (0, 0, 0)), name="shaders")
    t_ground = b.texture(r.uniform(0.2, 0.8, (32, 32, 3)), triplanar_scale=0.7)
    nrm = np.concatenate([r.uniform(0.0, 0.3, (16, 16, 2)), r.uniform(0.8, 1.0, (16, 16, 1))], -1)
    t_nrm = b.texture(nrm)
    t_sphere = b.texture(r.uniform(0.2, 0.8, (16, 16, 3)), triplanar_scale=0.5)
    t_rough = b.texture(r.uniform(0.1, 0.6, (8, 8, 3)), triplanar_scale=0.8)
    t_box = b.texture(r.uniform(0.2, 0.8, (8, 8, 3)), triplanar_scale=0.3)
    m_ground = b.material(_abi.MAT_MATTE, diffuse=(0.5, 0.5, 0.5), diffuse_tex=t_ground, normal_tex=t_nrm)
    m_sphere = b.material(_abi.MAT_KELEMEN, diffuse=(0.6, 0.6, 0.6), specular=(1.0, 1.0, 1.0), roughness=0.2,
                          reflectance=0.5, diffuse_tex=t_sphere, roughness_tex=t_rough, normal=(0.1, 0.05, 1.0))
    m_box = b.material(_abi.MAT_MATTE, diffuse=(0.5, 0.5, 0.5), diffuse_tex=t_box)
    gv = np.array([[-5, -1, 5], [5, -1, 5], [5, -1, -5], [-5, -1, -5]], np.float64)
    guv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float64) * 4.0
    b.mesh(gv, np.array([[0, 1, 2], [0, 2, 3]]), m_ground, normals=np.tile([0, 1, 0], (4, 1)), uvs=guv)
    v, f = icosphere(sphere_level)
    b.mesh(v, f, m_sphere, normals=v, object_to_world=translate(-0.6, 0.0, 0.0))
    bv, bf, _ = box_mesh()
    b.mesh(bv, bf, m_box, object_to_world=translate(1.3, -0.55, 0.6) @ rot_y(35.0) @ scale(0.9, 0.9, 0.9))
    b.square_light(translate(-2.0, 3.0, 1.0) @ rot_x(-90.0), 0.5, 0.5, (8.0, 8.0, 8.0), 0.0)
    b.sphere_light((2.2, 1.2, 1.5), 0.3, (30.0, 24.0, 18.0), 0.0)
    return b.build(render=dict(spp=spp, max_depth=max_depth, min_depth=max_depth, seed=seed))


def sphere_rays(n=1 << 20, seed=3, center=None) -> np.ndarray:
    """Hit-ID ray set: origins uniform in [-3,3]^3 around `center`, directions uniform on the sphere,
    mint 0, maxt 1e30. Returns (n, 8) float32 aur_ray records."""
    r = np.random.default_rng(seed)
    o = r.uniform(-3.0, 3.0, size=(n, 3))
    if center is not None:
        o = o + np.asarray(center, np.float64)
    d = r.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 3], rays[:, 4:7], rays[:, 7] = o, 0.0, d, 1e30
    return rays


def sphere_center_camera(data: SceneData) -> np.ndarray:
    """Camera-space centre of the icosphere object (object index 1) of sphere_scene."""
    sel = data.tri_attr == 1
    v = data.verts[data.tri_vidx[sel].ravel()]
    return 0.5 * (v.min(0) + v.max(0))


def terrain_scene(width=1920, height=1080, spp=64, max_depth=8, grid=1024, spheres=256, sphere_level=4,
                  seed=4, sphere_seed=5, render_seed=9) -> SceneData:
    """Large scene: a grid x grid heightfield with 5-octave fBm heights (amplitude 0.3, seed 4) plus
    `spheres` level-4 icospheres (radii U[0.05,0.4], seed 5); 16 materials drawn from Lambert /
    Cook-Torrance / Kelemen (roughness U[0.05,0.9], albedo U[0.1,0.9]); 4 quad lights; roulette
    when bounces > 2 (from the third bounce)."""
    b = SceneBuilder(width, height, FOV40 * 1.3, world_to_camera=look_at((0, 3.2, 9.5), (0, 0, -1.0)),
                     name="terrain")
    mr = np.random.default_rng(seed + 1000)
    mats = []
    for k in range(16):
        alb = tuple(mr.uniform(0.1, 0.9, 3))
        rough = float(mr.uniform(0.05, 0.9))
        kind = k % 3
        if kind == 0:
            mats.append(b.material(_abi.MAT_MATTE, diffuse=alb))
        elif kind == 1:
            mats.append(b.material(_abi.MAT_COOKTORRANCE, specular=alb, roughness=rough, reflectance=0.04))
        else:
            mats.append(b.material(_abi.MAT_KELEMEN, diffuse=alb, specular=(1.0, 1.0, 1.0), roughness=rough,
                                   reflectance=0.04))
    ext = 8.0
    xs = np.linspace(-ext, ext, grid)
    X, Z = np.meshgrid(xs, xs, indexing="xy")
    H = value_noise_fbm(X, Z, 5, 0.3, seed)
    # vertex normals from central differences
    dx = np.gradient(H, xs, axis=1)
    dz = np.gradient(H, xs, axis=0)
    N = np.stack([-dx, np.ones_like(H), -dz], -1)
    N /= np.linalg.norm(N, axis=-1, keepdims=True)
    V = np.stack([X, H, Z], -1).reshape(-1, 3)
    N = N.reshape(-1, 3)
    i = np.arange(grid - 1)
    I, J = np.meshgrid(i, i, indexing="xy")
    a = (J * grid + I).ravel()
    f = np.concatenate([np.stack([a, a + grid, a + 1], 1), np.stack([a + 1, a + grid, a + grid + 1], 1)])
    # 4 x 4 material tiles over the terrain: one object per tile
    cx = (I.ravel() * 4) // (grid - 1)
    cz = (J.ravel() * 4) // (grid - 1)
    tile = np.concatenate([cz * 4 + cx, cz * 4 + cx])
    for t in range(16):
        sel = f[tile == t]
        b.mesh(V, sel, mats[t], normals=N)
    sr = np.random.default_rng(sphere_seed)
    sv, sf = icosphere(sphere_level)
    for _ in range(spheres):
        rad = float(sr.uniform(0.05, 0.4))
        px, pz = sr.uniform(-ext * 0.9, ext * 0.9, 2)
        gx = int(round((px + ext) / (2 * ext) * (grid - 1)))
        gz = int(round((pz + ext) / (2 * ext) * (grid - 1)))
        py = H[gz, gx] + rad * 0.8
        b.mesh(sv * rad + np.array([px, py, pz]), sf, mats[int(sr.integers(0, 16))], normals=sv)
    for (lx, lz, col) in ((-4.0, -4.0, (14.0, 12.0, 10.0)), (4.0, -4.0, (10.0, 12.0, 14.0)),
                          (-4.0, 4.0, (12.0, 12.0, 12.0)), (4.0, 4.0, (14.0, 10.0, 8.0))):
        b.square_light(translate(lx, 5.0, lz) @ rot_x(-90.0), 0.75, 0.75, col, 0.0)
    return b.build(render=dict(spp=spp, max_depth=max_depth, min_depth=2, seed=render_seed))


def batch_scenes(n=64, base_seed=6):
    """64 box scenes with seeded poses/materials; resolution from {128..512}^2, spp from {4,16,64},
    depth from {3,5,8} per scene (seed 6+i)."""
    out = []
    for i in range(n):
        r = np.random.default_rng(base_seed + i)
        res = int(r.choice([128, 192, 256, 384, 512]))
        spp = int(r.choice([4, 16, 64]))
        depth = int(r.choice([3, 5, 8]))
        d = box_scene(res, res, spp, depth, seed=base_seed + i, rng_seed=10_000 + base_seed + i)
        d.name = f"box{i}"
        out.append(d)
    return out


def texture_scene(width=256, height=256, spp=256, max_depth=6, seed=2, tex_seed=7) -> SceneData:
    """Differentiable workload: sphere_scene at 256x256 with the ground albedo replaced by a 64x64 RGB
    texture (uniform 0.2-0.8, seed 7)."""
    tex = np.random.default_rng(tex_seed).uniform(0.2, 0.8, size=(64, 64, 3)).astype(F32)
    d = sphere_scene(width, height, spp, max_depth, seed, ground_texture=tex)
    d.name = "texture"
    return d

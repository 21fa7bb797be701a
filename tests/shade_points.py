"""Shading points for the probe's `shade_point` kind (10) and an independent float64
restatement of what the reference computes there: the interpolated face-forwarded
normal, Material::runNormalShader (material.cpp:27-40), the back-facing fix
(integrator.cpp:132-150), and the texture shaders (texture2DShader.h:28-31,
triplanarTextureShader.h:29-93, Texture2D::read with filter 0, texture2D.cpp:48-72)."""
import numpy as np

from aurora_b200 import _abi


def hit_records(data, n, seed, lobe_u=None):
    """n records (triangle, t, u, v, o3, d3, matte, lobe_u) of rays that hit a random point of a
    random triangle of a random attribute at t = 2 from either side."""
    r = np.random.default_rng(seed)
    attrs = np.unique(data.tri_attr)                 # each attribute equally often
    pick = attrs[r.integers(0, attrs.size, n)]
    prim = np.zeros(n, np.int64)
    for a in attrs:
        sel = np.nonzero(pick == a)[0]
        tris = np.nonzero(data.tri_attr == a)[0]
        prim[sel] = tris[r.integers(0, tris.size, sel.size)]
    tri = data.verts[data.tri_vidx[prim].astype(np.int64)].astype(np.float64)
    u, v = r.uniform(0, 1, n), r.uniform(0, 1, n)
    flip = u + v > 1
    u[flip], v[flip] = 1 - u[flip], 1 - v[flip]
    P = (1 - u - v)[:, None] * tri[:, 0] + u[:, None] * tri[:, 1] + v[:, None] * tri[:, 2]
    d = r.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t = np.full(n, 2.0)
    o = P - d * t[:, None]
    lu = r.integers(0, 2, n).astype(np.float64) if lobe_u is None else np.full(n, lobe_u)
    return np.concatenate([prim[:, None], t[:, None], u[:, None], v[:, None], o, d, np.zeros((n, 1)),
                           lu[:, None]], 1).astype(np.float32)


def _norm(x):
    return x / np.linalg.norm(x)


def _texel(img, s, t):
    h, w = img.shape[:2]
    x = min(max(int(np.floor(s * w)), 0), w - 1)
    y = min(max(int(np.floor(t * h)), 0), h - 1)
    return img[y, x].astype(np.float64)


def _shader(data, tex, P, Ng, su, sv, attr, float_shader):
    img = data.textures[tex]
    scales = data.tex_triplanar_scale
    scale = 0.0 if scales is None else float(scales[tex])
    if scale == 0.0:
        fs, ft = su - np.floor(su), 1.0 - (sv - np.floor(sv))
        c = _texel(img, fs, ft)
        return c[0] if float_shader else c
    m = np.eye(4) if data.attr_c2o is None else data.attr_c2o[attr].reshape(4, 4).astype(np.float64)
    if float_shader:
        w = np.maximum(np.abs(Ng) - 0.2, 0.0)
    else:
        w = np.maximum(np.abs(_norm(m[:3, :3] @ Ng)) - 0.25, 0.0)
    w = w / w.sum()
    Po = (m[:3, :3] @ P + m[:3, 3]) / scale
    out = np.zeros(3)
    for i in range(3):
        if w[i] > 0:
            out += _texel(img, abs(np.fmod(Po[(i + 1) % 3], 1.0)), abs(np.fmod(Po[(i + 2) % 3], 1.0))) * w[i]
    return out[0] if float_shader else out


def expected(data, rec):
    """(N3, Ng3, lobe, color3, rough) per record, for matte, Kelemen (all-zero albedo tables:
    lobe_u 1 picks the diffuse lobe, 0 the specular one) and Cook-Torrance materials."""
    out = np.zeros((rec.shape[0], 11))
    for k, q in enumerate(rec.astype(np.float64)):
        prim, t, u, v = int(q[0]), q[1], q[2], q[3]
        o, d = q[4:7], q[7:10]
        cn = data.corner_normals[prim].reshape(3, 3).astype(np.float64)
        w = 1.0 - u - v
        nn = w * cn[0] + u * cn[1] + v * cn[2]
        if nn @ d > 0:
            nn = -nn
        Ng = _norm(nn)
        P = o + d * t
        uv = data.corner_uvs[prim].reshape(3, 2).astype(np.float64)
        su, sv = w * uv[0] + u * uv[1] + v * uv[2]
        attr = int(data.tri_attr[prim])
        m = data.materials[int(data.attr_material[attr])]
        N = Ng
        if m.normal_kind != _abi.NORMAL_NONE:
            c = np.array(m.normal, np.float64) if m.normal_kind == _abi.NORMAL_CONSTANT else \
                _shader(data, m.normal_tex, P, Ng, su, sv, attr, False)
            a = np.cross(Ng, [1.0, 0, 0]) if (Ng[0] == 0 and Ng[1] != 0 and Ng[2] == 0) else np.cross(Ng, [0, 1.0, 0])
            b = np.cross(Ng, a)
            ns = _norm(a) * c[0] + _norm(b) * c[1] + Ng * c[2]
            N = _norm(ns) if np.any(ns != 0) else Ng
        V = -_norm(d)
        if V @ N <= 0:
            N = _norm(np.cross(V, np.cross(N, V)))
        diff = _shader(data, m.diffuse_tex, P, Ng, su, sv, attr, False) if m.diffuse_tex >= 0 else np.array(m.diffuse)
        if m.type == _abi.MAT_CONSTANT:
            lobe, col, rough = 3, np.zeros(3), 0.0
        elif m.type == _abi.MAT_MATTE or (m.type == _abi.MAT_KELEMEN and q[11] > 0):
            lobe, col, rough = 0, diff, 0.0
        else:
            rough = _shader(data, m.roughness_tex, P, Ng, su, sv, attr, True) if m.roughness_tex >= 0 else m.roughness
            spec = _shader(data, m.specular_tex, P, Ng, su, sv, attr, False) if m.specular_tex >= 0 \
                else np.array(m.specular)
            lobe, col = 1, spec
        out[k] = np.concatenate([N, Ng, [lobe], col, [rough]])
    return out

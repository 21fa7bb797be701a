"""Pins the oracle's FP64 adjoint (oracle_adjoint, forward-mode) against central finite
differences of the oracle's own renderer.

With roulette off, a diffuse colour or a texel enters each path sample polynomially
(Lambert sampling does not depend on it), so with common random numbers the central
difference of the rendered loss equals the adjoint sample by sample up to O(h^2) and
float rounding. Tolerance: 1% of the finite difference plus 1e-6 absolute.
"""
import copy

import numpy as np
import pytest


def _loss(oracle_lib, data, tables, w, spp, crop, seed, light_samples=1):
    osc = oracle_lib.OracleScene(data, tables, use_bvh=True)
    mean, _, _ = osc.render(spp, data.render["max_depth"], data.render["min_depth"], seed, crop=crop, want_m2=False,
                            light_samples=light_samples)
    x0, y0, cw, ch = crop
    return float(np.sum(mean[..., :3] * w[y0:y0 + ch, x0:x0 + cw, :3]))


def _perturbed_material(data, m, c, h):
    d = copy.copy(data)
    d.materials = list(data.materials)
    md = copy.copy(data.materials[m])
    md.diffuse[c] = md.diffuse[c] + h
    d.materials[m] = md
    return d


def _perturbed_texel(data, i, h):
    d = copy.copy(data)
    tex = [np.array(t, np.float32, copy=True) for t in data.textures]
    flat = tex[0].reshape(-1)
    flat[i] = flat[i] + h
    d.textures = tex
    return d


def test_oracle_adjoint_albedo_matches_fd(oracle_lib):
    from aurora_b200 import scenes
    data = scenes.box_scene(64, 64, spp=8)
    tables = np.zeros((21, 64, 32), np.float32)
    w = np.random.default_rng(5).normal(size=(64, 64, 4)).astype(np.float32)
    w[..., 3] = 0.0
    crop, spp, seed = (16, 16, 32, 32), 8, 1
    osc = oracle_lib.OracleScene(data, tables, use_bvh=True)
    gm, gt = osc.adjoint(spp, 5, 5, seed, w, crop=crop)
    assert gt.size == 0
    h = 1e-2
    for m, c in [(0, 0), (0, 2), (1, 0), (2, 1)]:     # walls, red wall, green wall
        fd = (_loss(oracle_lib, _perturbed_material(data, m, c, h), tables, w, spp, crop, seed) -
              _loss(oracle_lib, _perturbed_material(data, m, c, -h), tables, w, spp, crop, seed)) / (2 * h)
        assert abs(gm[m, c] - fd) <= 0.01 * abs(fd) + 1e-6, (m, c, gm[m, c], fd)
    # the Cook-Torrance boxes' albedo is not a parameter; the lights' constant material neither
    assert np.all(gm[4:, :3] == 0.0)


def test_oracle_adjoint_texel_matches_fd(oracle_lib):
    from aurora_b200 import scenes
    data = scenes.texture_scene(128, 128, spp=4)
    tables = np.zeros((21, 64, 32), np.float32)
    tables[10] = oracle_lib.kelemen_table(0.5, 400)          # the sphere's Kelemen material (reflectance 0.5)
    w = np.random.default_rng(6).normal(size=(128, 128, 4)).astype(np.float32)
    w[..., 3] = 0.0
    crop, spp, seed = (48, 88, 32, 32), 4, 2                  # ground in front of the sphere
    osc = oracle_lib.OracleScene(data, tables, use_bvh=True)
    gm, gt = osc.adjoint(spp, 6, 6, seed, w, crop=crop)
    assert gt.size == data.texels().size and np.count_nonzero(gt) > 0
    i = int(np.argmax(np.abs(gt)))
    h = 1e-2
    fd = (_loss(oracle_lib, _perturbed_texel(data, i, h), tables, w, spp, crop, seed) -
          _loss(oracle_lib, _perturbed_texel(data, i, -h), tables, w, spp, crop, seed)) / (2 * h)
    assert abs(gt[i] - fd) <= 0.01 * abs(fd) + 1e-6, (i, gt[i], fd)
    # the textured ground owns no constant diffuse gradient
    assert np.all(gm[0, :3] == 0.0)


def test_oracle_adjoint_through_glass_matches_fd(oracle_lib):
    """Glass boxes (mirror and transmission vertices, emission seen through them): the
    wall albedo gradients against central differences, roulette off."""
    from aurora_b200 import _abi, scenes
    glass = dict(type_=_abi.MAT_GLASS, specular=(1.0, 1.0, 1.0), diffuse=(0.95, 0.9, 0.85), reflectance=0.04,
                 ior=1.5)
    data = scenes.box_scene(64, 64, spp=8, max_depth=6, box_mat=glass, lift=0.01)
    tables = np.zeros((21, 64, 32), np.float32)
    w = np.random.default_rng(9).normal(size=(64, 64, 4)).astype(np.float32)
    w[..., 3] = 0.0
    crop, spp, seed = (16, 24, 32, 32), 8, 1
    gm, _ = oracle_lib.OracleScene(data, tables).adjoint(spp, 6, 6, seed, w, crop=crop)
    h = 1e-2
    for m, c in [(0, 1), (1, 0), (2, 2)]:
        fd = (_loss(oracle_lib, _perturbed_material(data, m, c, h), tables, w, spp, crop, seed) -
              _loss(oracle_lib, _perturbed_material(data, m, c, -h), tables, w, spp, crop, seed)) / (2 * h)
        assert abs(gm[m, c] - fd) <= 0.01 * abs(fd) + 1e-6, (m, c, gm[m, c], fd)


def test_oracle_adjoint_triplanar_texel_matches_fd(oracle_lib):
    """A texel of a triplanar diffuse shader (blended with its neighbours on the other
    projection axes) under a normal map, against central differences."""
    from aurora_b200 import scenes
    data = scenes.shader_scene(64, 64, spp=4, sphere_level=3)
    tables = np.zeros((21, 64, 32), np.float32)
    w = np.random.default_rng(8).normal(size=(64, 64, 4)).astype(np.float32)
    w[..., 3] = 0.0
    crop, spp, seed = (20, 30, 32, 32), 4, 3
    osc = oracle_lib.OracleScene(data, tables, use_bvh=True)
    gm, gt = osc.adjoint(spp, 6, 6, seed, w, crop=crop)
    sizes = [t.size for t in data.textures]
    first = np.cumsum([0] + sizes)
    for tex in (0, 2, 4):                                   # ground, sphere and box shaders (triplanar)
        block = gt[first[tex]:first[tex + 1]]
        assert np.count_nonzero(block) > 0
        i = first[tex] + int(np.argmax(np.abs(block)))
        h = 1e-2
        fd = (_loss(oracle_lib, _perturbed_texel_any(data, i, h), tables, w, spp, crop, seed) -
              _loss(oracle_lib, _perturbed_texel_any(data, i, -h), tables, w, spp, crop, seed)) / (2 * h)
        assert abs(gt[i] - fd) <= 0.01 * abs(fd) + 1e-6, (tex, i, gt[i], fd)


def _perturbed_texel_any(data, i, h):
    d = copy.copy(data)
    tex = [np.array(t, np.float32, copy=True) for t in data.textures]
    sizes = np.cumsum([0] + [t.size for t in tex])
    k = int(np.searchsorted(sizes, i, side="right") - 1)
    flat = tex[k].reshape(-1)
    flat[i - sizes[k]] = flat[i - sizes[k]] + h
    d.textures = tex
    return d


def test_oracle_adjoint_escape_after_last_vertex_matches_fd(oracle_lib):
    """Depth 2, a glass sphere on a Lambert ground under a constant environment light: paths
    camera -> ground -> glass whose mirror or transmission ray escapes after the LAST vertex
    see the environment (integrator.cpp:255-274), so the ground albedo's gradient carries that
    term. Checked against central differences of the oracle's renderer."""
    from aurora_b200 import _abi, scenes
    glass = dict(type_=_abi.MAT_GLASS, specular=(1.0, 1.0, 1.0), diffuse=(0.9, 0.95, 1.0), reflectance=0.04, ior=1.5)
    data = scenes.sphere_scene(48, 48, 8, 2, 2, env=dict(color=(0.8, 0.9, 1.0)), sphere_mat=glass)
    tables = np.zeros((21, 64, 32), np.float32)
    w = np.random.default_rng(10).normal(size=(48, 48, 4)).astype(np.float32)
    w[..., 3] = 0.0
    crop, spp, seed = (8, 24, 32, 24), 8, 2
    gm, _ = oracle_lib.OracleScene(data, tables).adjoint(spp, 2, 2, seed, w, crop=crop)
    h = 1e-2
    for c in range(3):
        fd = (_loss(oracle_lib, _perturbed_material(data, 0, c, h), tables, w, spp, crop, seed) -
              _loss(oracle_lib, _perturbed_material(data, 0, c, -h), tables, w, spp, crop, seed)) / (2 * h)
        assert abs(gm[0, c] - fd) <= 0.01 * abs(fd) + 1e-6, (c, gm[0, c], fd)


def test_oracle_adjoint_light_samples_matches_fd(oracle_lib):
    """light_samples 3 (integrateCameraSample(sample, 3) after the first pass): the wall albedo
    gradients of the oracle's adjoint against central differences of its renderer."""
    from aurora_b200 import scenes
    data = scenes.box_scene(48, 48, spp=4)
    tables = np.zeros((21, 64, 32), np.float32)
    w = np.random.default_rng(12).normal(size=(48, 48, 4)).astype(np.float32)
    w[..., 3] = 0.0
    crop, spp, seed = (8, 8, 32, 32), 4, 1
    gm, _ = oracle_lib.OracleScene(data, tables).adjoint(spp, 5, 5, seed, w, crop=crop, light_samples=3)
    h = 1e-2
    for m, c in [(0, 0), (1, 0), (2, 1)]:
        fd = (_loss(oracle_lib, _perturbed_material(data, m, c, h), tables, w, spp, crop, seed, 3) -
              _loss(oracle_lib, _perturbed_material(data, m, c, -h), tables, w, spp, crop, seed, 3)) / (2 * h)
        assert abs(gm[m, c] - fd) <= 0.01 * abs(fd) + 1e-6, (m, c, gm[m, c], fd)


def test_oracle_adjoint_albedo_matches_the_analytic_gradient(oracle_lib):
    """Closed form: on a Lambert plane under a square light at max_depth 1 the pixel is
    albedo * E, E = integral of Le cos(theta) cos(theta_l) / (pi r^2) over the light, so
    d pixel / d albedo = E (the quadrature of test_oracle's plane cases)."""
    import math
    from test_oracle import _plane_under_light, _light_integrals
    albedo, h, s, le, px = 0.6, 1.0, 0.25, 4.0, 0.8
    data = _plane_under_light(albedo, h, s, (le, le, le), px)
    want = _light_integrals(0.3, 1.0, np.array([0.0, 1.0, 0.0]), h, s, le, px, 600)[2]
    osc = oracle_lib.OracleScene(data, use_bvh=False)
    w = np.zeros((16, 16, 4), np.float32)
    w[8, 8, 0] = 1.0
    spp, seed = 4096, 3
    gm, gt = osc.adjoint(spp, 1, 1, seed, w, crop=(8, 8, 1, 1))
    mean, m2, _ = osc.render(spp, 1, 1, seed, crop=(8, 8, 1, 1))
    sigma = math.sqrt(m2[0, 0, 0] / (spp - 1)) / math.sqrt(spp) / albedo
    assert abs(gm[0, 0] - want) < 4 * sigma + 1e-3 * want, (gm[0, 0], want, sigma)
    assert abs(gm[0, 0] - mean[0, 0, 0] / albedo) < 1e-5 * want    # the same paths, linear in the albedo
    assert np.all(gm[0, 1:3] == 0.0)

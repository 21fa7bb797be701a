"""Pins the CPU oracle (oracle/aurora_oracle.cpp) with hand-derived known answers.

The reference ships no tests or golden vectors and cannot be built here, so the
oracle is checked against independent float64 restatements of the reference
formulas and against analytic light-transport integrals.
"""
import math

import numpy as np
import pytest


def splitmix_u01(seed, pixel, sample, dim):
    M = (1 << 64) - 1

    def fin(z):
        z = ((z ^ (z >> 30)) * 0xbf58476d1ce4e5b9) & M
        z = ((z ^ (z >> 27)) * 0x94d049bb133111eb) & M
        return z ^ (z >> 31)
    key = fin((seed * 0x9e3779b97f4a7c15 + 0x632be59bd9b4e019) & M)
    counter = (pixel << 32) | (sample << 12) | dim
    z = fin((key + counter * 0x9e3779b97f4a7c15) & M)
    return (z >> 40) / 16777216.0


def test_rng_matches_splitmix64(oracle_lib):
    for seed, px, s, d in [(1, 0, 0, 0), (1, 65535, 15, 41), (7, 123456, 1000, 3), (3, 2**31, 2**19, 4095)]:
        assert oracle_lib.rng_u01(seed, px, s, d) == splitmix_u01(seed, px, s, d)


def test_rng_uniformity(oracle_lib):
    u = np.array([oracle_lib.rng_u01(5, p, 0, 2) for p in range(20000)])
    assert 0.0 <= u.min() and u.max() < 1.0
    hist, _ = np.histogram(u, bins=10, range=(0, 1))
    assert np.all(np.abs(hist - 2000) < 6 * math.sqrt(2000))


def tri_soup():
    verts = np.array([[0, 0, -2], [1, 0, -2], [0, 1, -2], [0, 0, -3], [1, 0, -3], [0, 1, -3]], np.float32)
    idx = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    return verts, idx


def ray(o, d, mint=0.0, maxt=1e30):
    return np.array([*o, mint, *d, maxt], np.float32)


def test_moller_trumbore_known_answers(oracle_lib):
    v, i = tri_soup()
    rays = np.stack([ray((0.25, 0.25, 0), (0, 0, -1)),        # hits both, nearest is prim 0 at t=2
                     ray((0.25, 0.25, 0), (0, 0, 1)),         # behind the origin
                     ray((0.25, 0.25, 0), (1, 0, 0)),         # parallel to both
                     ray((0.25, 0.25, 0), (0, 0, -1), 2.5),   # mint skips prim 0
                     ray((0.25, 0.25, 0), (0, 0, -1), 0, 1.5),  # maxt before prim 0
                     ray((0.0, 0.0, 0), (0, 0, -1)),          # exactly on a vertex (b1 = b2 = 0)
                     ray((0.6, 0.6, 0), (0, 0, -1))])         # outside (b1 + b2 > 1)
    hits, ties = oracle_lib.trace_brute(v, i, np.array([7, 9], np.int32), rays)
    assert hits["prim"].tolist() == [0, -1, -1, 1, -1, 0, -1]
    assert hits["attr"][0] == 7 and hits["attr"][3] == 9
    assert hits["t"][0] == 2.0 and hits["t"][3] == 3.0
    assert abs(hits["u"][0] - 0.25) < 1e-7 and abs(hits["v"][0] - 0.25) < 1e-7
    occ = oracle_lib.occluded_brute(v, i, rays)
    assert occ.tolist() == [1, 0, 0, 1, 0, 1, 0]


def test_exact_ties_are_counted(oracle_lib):
    v, i = tri_soup()
    v2 = np.concatenate([v, v[:3]])
    i2 = np.concatenate([i, np.array([[6, 7, 8]], np.uint32)])
    hits, ties = oracle_lib.trace_brute(v2, i2, None, np.stack([ray((0.25, 0.25, 0), (0, 0, -1))]))
    assert ties[0] == 2 and hits["prim"][0] == 2     # the later duplicate wins, as with maxt=t replacement


def test_cpu_bvh_equals_brute_force(oracle_lib):
    from aurora_b200 import scenes
    r = np.random.default_rng(11)
    n = 3000
    c = r.uniform(-2, 2, (n, 1, 3))
    verts = (c + r.normal(0, 0.15, (n, 3, 3))).reshape(-1, 3).astype(np.float32)
    idx = np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)
    b = scenes.SceneBuilder(8, 8, 0.5)
    m = b.material(0, diffuse=(0.5, 0.5, 0.5))
    b.mesh(verts, idx, m)
    data = b.build()
    rays = scenes.sphere_rays(20000, seed=12)
    brute, ties = oracle_lib.trace_brute(data.verts, data.tri_vidx, data.tri_attr, rays)
    sc = oracle_lib.OracleScene(data, use_bvh=True)
    fast = sc.trace(rays)
    ok = ties <= 1
    assert np.array_equal(fast["prim"][ok], brute["prim"][ok])
    assert np.array_equal(fast["t"][ok & (brute["prim"] >= 0)], brute["t"][ok & (brute["prim"] >= 0)])


def test_brdf_known_values(oracle_lib):
    """Lambert and Cook-Torrance (Beckmann) against float64 restatements of lambert.h / cookTorrance.cpp."""
    rng = np.random.default_rng(3)
    recs, want_eval, want_pdf = [], [], []
    for _ in range(200):
        N = np.array([0.0, 0.0, 1.0])
        V = rng.normal(size=3); V[2] = abs(V[2]) + 0.3; V /= np.linalg.norm(V)
        L = rng.normal(size=3); L[2] = abs(L[2]) + 0.3; L /= np.linalg.norm(L)
        col = rng.uniform(0.1, 0.9, 3)
        rough = rng.uniform(0.1, 0.8)
        H = (L + V) / np.linalg.norm(L + V)
        vh, vn, nh, ln = V @ H, V @ N, H @ N, L @ N
        r2 = rough * rough
        D = 1.0 / (r2 * math.pi * nh ** 3) * math.exp(-math.tan(math.acos(nh)) ** 2 / r2)
        ok = vh > 0.001 and ln > 0.001 and vn > 0.001
        want_eval.append(col * D / (4 * vh * vh) if ok else np.zeros(3))
        rr = max(0.001, r2)
        Dp = math.exp(-math.tan(math.acos(nh)) ** 2 / rr) / (rr * math.pi * nh ** 3)
        want_pdf.append(Dp / (4 * vh))
        recs.append([1, *col, rough, *L, *V, *N])
    recs = np.array(recs, np.float32)
    ev = oracle_lib.probe(1, recs)
    pdf = oracle_lib.probe(2, recs)[:, 0]
    np.testing.assert_allclose(ev, np.array(want_eval), rtol=2e-5, atol=1e-7)
    np.testing.assert_allclose(pdf, np.array(want_pdf), rtol=2e-5, atol=1e-10)
    lam = recs.copy(); lam[:, 0] = 0
    np.testing.assert_allclose(oracle_lib.probe(1, lam), recs[:, 1:4] / math.pi, rtol=1e-6)
    np.testing.assert_allclose(oracle_lib.probe(2, lam)[:, 0], 0.5 / math.pi, rtol=1e-6)


def test_ct_sample_is_a_reflection(oracle_lib):
    rng = np.random.default_rng(5)
    recs = []
    for _ in range(500):
        N = rng.normal(size=3); N /= np.linalg.norm(N)
        V = rng.normal(size=3); V /= np.linalg.norm(V)
        if V @ N < 0.2:
            V = V - 2 * (V @ N) * N + 0.2 * N
            V /= np.linalg.norm(V)
        recs.append([1, 0.5, 0.6, 0.7, rng.uniform(0.1, 0.9), *V, *N, rng.uniform(), rng.uniform()])
    recs = np.array(recs, np.float32)
    out = oracle_lib.probe(0, recs)
    L = out[:, :3].astype(np.float64)
    np.testing.assert_allclose(np.linalg.norm(L, axis=1), 1.0, atol=1e-5)
    V, N = recs[:, 5:8].astype(np.float64), recs[:, 8:11].astype(np.float64)
    H = (L + V) / np.linalg.norm(L + V, axis=1, keepdims=True)
    vh = np.sum(V * H, 1)
    pdf = out[:, 3]
    # sample colour = colour * D / (4 vh^2) with pdf = D / (4 vh): colour * pdf / vh
    good = (pdf > 0) & (pdf < 1000) & (vh > 0.01) & (out[:, 4] > 0)   # samples with v.h <= 1e-4 are black (pdf 1)
    np.testing.assert_allclose(out[good, 4], recs[good, 1] * pdf[good] / vh[good], rtol=2e-4)


def test_camera_and_power_heuristic(oracle_lib):
    out = oracle_lib.probe(4, np.array([[0.36397, 256, 256, 128, 128, 0.0, 0.0],
                                        [0.36397, 256, 256, 0, 0, 0.0, 0.0]], np.float32))
    np.testing.assert_allclose(out[0], [0, 0, -1], atol=1e-7)
    d = np.array([-0.36397, 0.36397, -1.0]); d /= np.linalg.norm(d)
    np.testing.assert_allclose(out[1], d, rtol=1e-6)
    w = oracle_lib.probe(5, np.array([[2.0, 1.0], [0.5, 0.5]], np.float32))[:, 0]
    np.testing.assert_allclose(w, [0.8, 0.5], rtol=1e-7)


def _plane_under_light(albedo=0.6, h=1.0, s=0.25, le=(4.0, 4.0, 4.0), px=0.8, fov=0.01):
    from aurora_b200 import scenes
    from aurora_b200 import _abi
    b = scenes.SceneBuilder(16, 16, fov, world_to_camera=scenes.look_at((px, 3, 0.001), (px, 0, 0)))
    m = b.material(_abi.MAT_MATTE, diffuse=(albedo,) * 3)
    v, f = scenes.quad((-5, 0, 5), (5, 0, 5), (5, 0, -5), (-5, 0, -5))
    b.mesh(v, f, m, normals=np.tile([0, 1, 0], (4, 1)))
    b.square_light(scenes.translate(0, h, 0) @ scenes.rot_x(-90.0), s, s, le, 0.0)
    return b.build()


def test_direct_lighting_matches_the_analytic_integral(oracle_lib):
    """Lambert plane under a square light: L = rho/pi * Le * integral cos cos' / r^2 dA (float64 quadrature)."""
    albedo, h, s, px = 0.6, 1.0, 0.25, 0.8
    data = _plane_under_light(albedo, h, s, px=px)
    sc = oracle_lib.OracleScene(data, use_bvh=False)
    mean, m2, counts = sc.render(4096, 1, 1, seed=3, crop=(8, 8, 1, 1))
    # the pixel at (8,8) looks (straight down, tiny fov) at the plane point (px, 0, 0) beside the light
    n = 400
    g = (np.arange(n) + 0.5) / n * 2 * s - s
    X, Z = np.meshgrid(g, g)
    r2 = (X - px) ** 2 + Z ** 2 + h ** 2
    integral = np.sum((h / np.sqrt(r2)) ** 2 / r2) * (2 * s / n) ** 2
    want = albedo / math.pi * 4.0 * integral
    got = mean[0, 0, 0]
    sigma = math.sqrt(m2[0, 0, 0] / 4095) / math.sqrt(4096)
    assert abs(got - want) < 4 * sigma + 1e-3 * want, (got, want, sigma)


def _glossy_plane_scene(material, h, s, le, px, eye_dist):
    """The plane y = 0 with `material` (a builder -> material index callable) under a
    downward square light centred at (0, h, 0), seen by the 16 x 16 pixels of a camera at
    fov slope 1e-4 that looks at P = (px, 0, 0) from the mirror side of the light's centre.
    Returns the scene and the view direction V."""
    from aurora_b200 import scenes
    P = np.array([px, 0.0, 0.0])
    mirror = np.array([px, h, 0.0]) / math.hypot(px, h)   # reflection of the light centre's direction
    eye = P + eye_dist * mirror
    b = scenes.SceneBuilder(16, 16, 1e-4, world_to_camera=scenes.look_at(tuple(eye), tuple(P)))
    m = material(b)
    v, f = scenes.quad((-5, 0, 5), (5, 0, 5), (5, 0, -5), (-5, 0, -5))
    b.mesh(v, f, m, normals=np.tile([0, 1, 0], (4, 1)))
    b.square_light(scenes.translate(0, h, 0) @ scenes.rot_x(-90.0), s, s, (le, le, le), 0.0)
    return b.build(), mirror


def _light_integrals(rough, spec, V, h, s, le, px, n):
    """Float64 quadrature over the light square of next-event estimates at P for view V.

    Returns (expect, plain, lambert). plain is the Cook-Torrance integral of Le f(L, V)
    cos(theta) cos(theta_l) / r^2 dA, with f = colour D / (4 (V.H)^2), D = exp(-tan^2 a / m^2)
    / (m^2 pi cos^3 a), zero unless V.H, L.N and V.N exceed 1e-3 (cookTorrance.cpp:125-144).
    The reference's estimator converges to it except in one place: its sampler sets
    tan a = 0 where N.H > 0.999 (cookTorrance.cpp:79), so inside that 2.6-degree cap the pdf
    it reports for a sampled direction exceeds pdf() (cookTorrance.cpp:101-117) for the same
    direction, and the two power-heuristic weights (integrator.cpp:56-98) sum to more than
    one there. expect takes each strategy with its own weights: the light sample's
    w_l = p_l^2 / (p_l^2 + p_b^2) on f, the BRDF sample's w_b = p_s^2 / (p_s^2 + p_l^2) on the
    sampled f / pdf ratio, which is f / p_b for the Beckmann density it draws. lambert is
    the integral of Le cos(theta) cos(theta_l) / (pi r^2) dA: the Lambert estimate per unit
    albedo (integrator.cpp:33-54, lambert.h:68-80)."""
    g = (np.arange(n) + 0.5) / n * 2 * s - s
    X, Z = np.meshgrid(g, g)
    d = np.stack([X - px, np.full_like(X, h), Z], -1)
    r = np.linalg.norm(d, axis=-1)
    L = d / r[..., None]
    Hv = L + V
    Hv /= np.linalg.norm(Hv, axis=-1, keepdims=True)
    vh, ln, vn, nh = Hv @ V, L[..., 1], V[1], Hv[..., 1]
    cos_l = h / r
    m2 = rough * rough
    tan2 = (1.0 - nh * nh) / (nh * nh)
    D = np.exp(-tan2 / m2) / (m2 * math.pi * nh ** 3)
    f_all = spec * D / (4 * vh * vh)
    f_eval = np.where((vh > 1e-3) & (ln > 1e-3) & (vn > 1e-3), f_all, 0.0)
    mc = max(1e-3, m2)                                     # ctD floors m^2 at 0.001
    p_b = np.exp(-tan2 / mc) / (mc * math.pi * nh ** 3) / (4 * vh)
    D_s = np.where(nh > 0.999, 1.0, np.exp(-tan2 / mc)) / (mc * math.pi * nh ** 3)
    p_s = np.minimum(D_s, 1000.0) / (4 * vh)
    p_l = r * r / (cos_l * 4 * s * s)                      # solid-angle pdf of the area sample
    w_l = p_l ** 2 / (p_l ** 2 + p_b ** 2)
    w_b = p_s ** 2 / (p_s ** 2 + p_l ** 2)
    dA = (2 * s / n) ** 2
    geo = le * ln * cos_l / (r * r)
    return (float(np.sum(geo * (f_eval * w_l + f_all * w_b)) * dA), float(np.sum(geo * f_eval) * dA),
            float(np.sum(geo) * dA / math.pi))


def ct_plane_under_light(rough, spec=0.7, h=1.0, s=0.25, le=4.0, px=0.8, eye_dist=3.0, n=1200):
    """A Cook-Torrance (Beckmann) plane under a square light: the scene, the float64
    expectation of every pixel at max_depth 1, and the plain integral (_light_integrals)."""
    from aurora_b200 import _abi
    data, V = _glossy_plane_scene(
        lambda b: b.material(_abi.MAT_COOKTORRANCE, specular=(spec,) * 3, roughness=rough, reflectance=0.04),
        h, s, le, px, eye_dist)
    expect, plain, _ = _light_integrals(rough, spec, V, h, s, le, px, n)
    return data, expect, plain


def kelemen_albedo_lookup(table, costheta, rough):
    """KelemenMaterial::getAlbedo's bilinear lookup (kelemenMaterial.cpp:180-212) of a 64 x 32
    table, with its second roughness column always the last one, in float64."""
    i = min(max(int(math.floor(costheta * 63)), 0), 63)
    ra = min(max(int(math.floor(rough * 31)), 0), 31)
    rb = 31
    i1 = min(i + 1, 63)
    mixc = costheta * 63 - i
    res_a = (1 - mixc) * table[i, ra] + mixc * table[i1, ra]
    res_b = (1 - mixc) * table[i, rb] + mixc * table[i1, rb]
    rmix = rough * 31 - ra
    return (1 - rmix) * res_a + rmix * res_b


def kelemen_plane_under_light(tables, rough=0.3, spec=0.6, diff=0.5, refl=0.75, h=1.0, s=0.25, le=4.0, px=0.8,
                              eye_dist=3.0, n=1200):
    """A Kelemen plane under a square light. At the camera vertex the material takes the
    Cook-Torrance lobe (spec) with probability A = its table albedo at (N.V, roughness) and
    otherwise the Lambert lobe (diff), without reweighting (kelemenMaterial.cpp:228-255), so
    the pixel's expectation is A E_ct + (1 - A) diff E_lambert. Returns the scene, that
    expectation and A."""
    from aurora_b200 import _abi
    data, V = _glossy_plane_scene(
        lambda b: b.material(_abi.MAT_KELEMEN, diffuse=(diff,) * 3, specular=(spec,) * 3, roughness=rough,
                             reflectance=refl),
        h, s, le, px, eye_dist)
    e_ct, _, e_lam = _light_integrals(rough, spec, V, h, s, le, px, n)
    A = kelemen_albedo_lookup(tables[int(round(refl * 20))], float(V[1]), rough)
    return data, A * e_ct + (1 - A) * diff * e_lam, A


@pytest.mark.parametrize("rough", [0.15, 0.4])
def test_ct_direct_lighting_matches_the_analytic_integral(oracle_lib, rough):
    """Multiple importance sampling of a glossy lobe against its closed-form expectation."""
    data, want, plain = ct_plane_under_light(rough)
    sc = oracle_lib.OracleScene(data, use_bvh=False)
    spp = 65536
    mean, m2, counts = sc.render(spp, 1, 1, seed=5, crop=(8, 8, 1, 1))
    got = mean[0, 0, :3]
    sigma = np.sqrt(m2[0, 0, :3] / (spp - 1)) / math.sqrt(spp)
    assert np.all(np.abs(got - want) < 4 * sigma + 1e-4 * want), (got, want, plain, sigma)
    assert sigma[0] < 0.0015 * want      # the check resolves the 0.3% the cap adds at roughness 0.15
    if rough < 0.2:
        assert want - plain > 0.002 * plain


def metal_plane_under_light(refl=(0.9, 0.6, 0.3), gain=(1.0, 0.8, 1.2), rough_a=0.2, rough_b=0.5, mix=0.3, h=1.0,
                            s=0.25, le=4.0, px=0.8, eye_dist=3.0, n=1200):
    """A metal plane under a square light. MetalMaterial::getBrdf (metalMaterial.cpp:32-62)
    takes Cook-Torrance with colour schlick(V.N, reflectance) * gain per channel, and
    roughness A when its lobe number exceeds mix, else roughness B: the pixel's expectation
    is (1 - mix) E_ct(A) + mix E_ct(B) at that colour. Returns the scene and the RGB
    expectation."""
    from aurora_b200 import _abi
    data, V = _glossy_plane_scene(
        lambda b: b.material(_abi.MAT_METAL, specular=refl, gain=gain, roughness=rough_a, roughness_b=rough_b,
                             mix=mix),
        h, s, le, px, eye_dist)
    vn = float(V[1])
    col = np.array([(r + (1 - vn) ** 5 * (1 - r)) * g for r, g in zip(refl, gain)])
    e_a = _light_integrals(rough_a, 1.0, V, h, s, le, px, n)[0]
    e_b = _light_integrals(rough_b, 1.0, V, h, s, le, px, n)[0]
    return data, col * ((1 - mix) * e_a + mix * e_b)


def test_metal_matches_the_analytic_mixture(oracle_lib):
    """Metal's Schlick tint per channel and its two-roughness mixture against the closed form."""
    data, want = metal_plane_under_light()
    sc = oracle_lib.OracleScene(data, use_bvh=False)
    spp = 65536
    mean, m2, counts = sc.render(spp, 1, 1, seed=11, crop=(8, 8, 1, 1))
    got = mean[0, 0, :3]
    sigma = np.sqrt(m2[0, 0, :3] / (spp - 1)) / math.sqrt(spp)
    assert np.all(np.abs(got - want) < 4 * sigma + 1e-4 * want), (got, want, sigma)
    assert np.all(sigma < 0.005 * want)


def test_kelemen_lobe_choice_matches_the_analytic_mixture(oracle_lib):
    """The Kelemen lobe choice against A E_ct + (1 - A) E_lambert, with a constant albedo table
    (A = 0.35 wherever it is read) as the oracle's input."""
    tables = np.full((21, 64, 32), 0.35, np.float32)
    data, want, A = kelemen_plane_under_light(tables)
    assert abs(A - 0.35) < 1e-7
    sc = oracle_lib.OracleScene(data, tables, use_bvh=False)
    spp = 65536
    mean, m2, counts = sc.render(spp, 1, 1, seed=7, crop=(8, 8, 1, 1))
    got = mean[0, 0, :3]
    sigma = np.sqrt(m2[0, 0, :3] / (spp - 1)) / math.sqrt(spp)
    assert np.all(np.abs(got - want) < 4 * sigma + 1e-4 * want), (got, want, sigma)
    assert sigma[0] < 0.005 * want       # a lobe reweighted by 1/A or 1/(1-A) would move it by tens of percent


def lambert_plane_under_sphere(albedo=0.6, h=1.0, radius=0.25, le=4.0, px=0.8):
    """A Lambert plane y = 0 under a sphere light centred at (0, h, 0), seen straight down by
    the pixels of a 16 x 16 film at fov slope 1e-4, all at P = (px, 0, 0). The sphere lies
    wholly above P's horizon, so the irradiance at P is pi Le (R/d)^2 cos(theta) and the
    pixel's expectation at max_depth 1 is albedo Le R^2 h / d^3 (d = |centre - P|)."""
    from aurora_b200 import scenes
    from aurora_b200 import _abi
    b = scenes.SceneBuilder(16, 16, 1e-4, world_to_camera=scenes.look_at((px, 3, 0.001), (px, 0, 0)))
    m = b.material(_abi.MAT_MATTE, diffuse=(albedo,) * 3)
    v, f = scenes.quad((-5, 0, 5), (5, 0, 5), (5, 0, -5), (-5, 0, -5))
    b.mesh(v, f, m, normals=np.tile([0, 1, 0], (4, 1)))
    b.sphere_light((0.0, h, 0.0), radius, (le, le, le), 0.0)
    d = math.hypot(px, h)
    return b.build(), albedo * le * radius * radius * h / d ** 3


def test_sphere_light_matches_the_analytic_irradiance(oracle_lib):
    """Cone sampling of the sphere light (an extension of the reference) against its closed form."""
    data, want = lambert_plane_under_sphere()
    sc = oracle_lib.OracleScene(data, use_bvh=False)
    spp = 16384
    mean, m2, counts = sc.render(spp, 1, 1, seed=9, crop=(8, 8, 1, 1))
    got = mean[0, 0, :3]
    sigma = np.sqrt(m2[0, 0, :3] / (spp - 1)) / math.sqrt(spp)
    assert np.all(np.abs(got - want) < 4 * sigma + 1e-4 * want), (got, want, sigma)
    assert sigma[0] < 0.002 * want


def test_roulette_is_unbiased_where_its_weight_stays_below_one(oracle_lib):
    """Russian roulette (integrator.cpp:221-248) continues with probability cont, the running
    product of lum(colour) cos / pdf, and divides the throughput by it. A Lambert bounce adds
    2 lum(albedo) cos, so with every albedo at most 0.45 cont stays below one and the image
    with roulette from bounce 1 has the expectation of the image without it. (Above 0.5, cont
    can exceed one; the reference then continues and still divides by cont.)"""
    from aurora_b200 import scenes
    from aurora_b200 import _abi
    data = scenes.box_scene(64, 64, wall=(0.45, 0.45, 0.45), red=(0.45, 0.05, 0.05), green=(0.1, 0.4, 0.1),
                            box_mat=dict(type_=_abi.MAT_MATTE, diffuse=(0.4, 0.4, 0.4)))
    sc = oracle_lib.OracleScene(data)
    spp = 512
    full, m2f, cf = sc.render(spp, 5, 5, 3)
    rr, m2r, cr = sc.render(spp, 5, 1, 4)
    assert cr[0] < 0.8 * cf[0]                      # roulette ends paths early
    var = (m2f[..., :3] + m2r[..., :3]) / (spp - 1) / spp
    z = (rr[..., :3] - full[..., :3]) / np.sqrt(np.maximum(var, 1e-30))
    assert np.mean(np.abs(z) > 4) < 0.002
    tot = (rr[..., :3].sum() - full[..., :3].sum()) / math.sqrt(var.sum())
    assert abs(tot) < 4, tot


def test_oracle_render_is_deterministic(oracle_lib):
    from aurora_b200 import scenes
    data = scenes.box_scene(64, 64)
    sc = oracle_lib.OracleScene(data)
    a, _, ca = sc.render(4, 5, 5, 1, crop=(20, 20, 8, 8))
    b, _, cb = sc.render(4, 5, 5, 1, crop=(20, 20, 8, 8))
    assert np.array_equal(a, b) and np.array_equal(ca, cb)
    assert np.all(a[..., 3] == 1.0) and np.all(a[..., :3] > 0)


def test_kelemen_table_restatement(oracle_lib):
    t0 = oracle_lib.kelemen_table(0.0, 2000)
    t1 = oracle_lib.kelemen_table(1.0, 2000)
    assert np.all(t0 >= 0) and np.all(t1 >= t0 - 1e-6)
    # reflectance 1 => F = 1; at normal incidence and low roughness the estimator -> 1
    assert abs(t1[63, 1] - 1.0) < 0.02


def _frame(n):
    """coordinateSystem (math_utils.h:107-129): unnormalised tangents."""
    n = np.asarray(n, np.float64)
    if n[0] == 0 and n[1] != 0 and n[2] == 0:
        v2 = np.cross(n, [1.0, 0, 0])
    else:
        v2 = np.cross(n, [0, 1.0, 0])
    return v2, np.cross(n, v2)


def test_mirror_and_transmission_known_answers(oracle_lib):
    """SpecMirror / SpecTransmit (specMirror.cpp:35-40, specTransmit.cpp:33-56) in float64:
    tangent components taken along the UNNORMALISED frame (worldToTangent) and mapped back
    along the normalised one (tangentToWorld) — an exact reflection only where the frame is
    unit length, a scaled one elsewhere, as the reference computes it."""
    r = np.random.default_rng(12)
    recs, want = [], []
    for k in range(200):
        n = r.normal(size=3); n /= np.linalg.norm(n)
        v = r.normal(size=3); v /= np.linalg.norm(v)
        while v @ n < 0.05:
            v = r.normal(size=3); v /= np.linalg.norm(v)
        lobe, ior = (2, 0.0) if k % 2 == 0 else (4, 1.5)
        du, dv = _frame(n)
        vt = np.array([v @ du, v @ dv, v @ n])
        if lobe == 2:
            t = np.array([-vt[0], -vt[1], vt[2]])
        else:
            eta = 1 / ior
            cost = -np.sqrt(max(0.0, 1 - eta * eta * (1 - (v @ n) ** 2)))
            t = np.array([eta * -vt[0], eta * -vt[1], cost])
        d = t[0] * du / np.linalg.norm(du) + t[1] * dv / np.linalg.norm(dv) + t[2] * n
        want.append(d / np.linalg.norm(d))
        recs.append([lobe, 0.9, 0.8, 0.7, ior, *v, *n, 0.5, 0.5])
    out = oracle_lib.probe(0, np.array(recs, np.float32))
    np.testing.assert_allclose(out[:, :3], np.array(want), atol=2e-6)
    assert np.all(out[:, 3] == 1.0) and np.allclose(out[:, 4:7], [0.9, 0.8, 0.7])
    # V below the surface: ei = ior, et = 1 and a grazing angle reflects totally (pdf 0)
    tir = oracle_lib.probe(0, np.array([[4, 1, 1, 1, 1.5, 0.99, 0, -0.141, 0, 0, 1, 0.5, 0.5]], np.float32))
    assert tir[0, 3] == 0.0 and np.all(tir[0, 4:7] == 0.0)
    # an exact mirror where the frame is unit length (N orthogonal to y)
    m = oracle_lib.probe(0, np.array([[2, 1, 1, 1, 0, 0.6, 0, 0.8, 0, 0, 1, 0.5, 0.5]], np.float32))
    np.testing.assert_allclose(m[0, :3], [-0.6, 0, 0.8], atol=1e-7)


def _plane_under_sky(env, albedo=0.5):
    """A Lambert plane filling the view under an environment light (nothing else)."""
    from aurora_b200 import _abi, scenes
    b = scenes.SceneBuilder(32, 32, 0.3, world_to_camera=scenes.look_at((0, 3, 0.01), (0, 0, 0)), name="plane")
    m = b.material(_abi.MAT_MATTE, diffuse=(albedo, albedo, albedo))
    v = np.array([[-50, 0, 50], [50, 0, 50], [50, 0, -50], [-50, 0, -50]], np.float64)
    b.mesh(v, np.array([[0, 1, 2], [0, 2, 3]]), m, normals=np.tile([0, 1.0, 0], (4, 1)))
    b.env_light(**env)
    return b.build(render=dict(spp=64, max_depth=1, min_depth=1, seed=3))


@pytest.mark.parametrize("env", [dict(color=(2.0, 1.0, 0.5), exposure=1.0),
                                 dict(color=(1, 1, 1), exposure=0.0,
                                      texture=np.full((16, 32, 3), 1.5, np.float32))],
                         ids=["constant", "uniform-map"])
def test_env_light_lambert_plane(oracle_lib, env):
    """Next-event estimation of a constant sky above a Lambert plane: a*E in expectation, both
    with uniform hemisphere sampling (pdf 1/2pi) and with the env map's uniform-sphere
    sampling weighted by the map pdf (texel luminance / mean = 1 here, pdf 1/4pi)."""
    from aurora_b200 import scenes
    data = _plane_under_sky(env)
    E = np.array(env["color"]) * 2.0 ** env["exposure"] * (1.5 if "texture" in env else 1.0)
    mean, m2, _ = oracle_lib.OracleScene(data).render(256, 1, 1, 3)
    got = mean[..., :3].mean((0, 1))
    np.testing.assert_allclose(got, 0.5 * E, rtol=0.01)


def test_env_light_seen_by_camera(oracle_lib):
    """Camera rays that miss see the environment (alpha 1), unfiltered."""
    from aurora_b200 import _abi, scenes
    b = scenes.SceneBuilder(8, 8, 0.3, world_to_camera=scenes.look_at((0, 3, 0.01), (0, 0, 0)))
    m = b.material(_abi.MAT_MATTE, diffuse=(0.5, 0.5, 0.5))
    v = np.array([[100, -5, 100], [101, -5, 100], [100, -5, 101]], np.float64)   # out of view
    b.mesh(v, np.array([[0, 1, 2]]), m)
    b.env_light(color=(300.0, 2.0, 1.0))
    data = b.build(render=dict(spp=4, max_depth=3, min_depth=3, seed=1))
    mean, _, _ = oracle_lib.OracleScene(data).render(4, 3, 3, 1)
    np.testing.assert_allclose(mean[..., :3], np.broadcast_to([300.0, 2.0, 1.0], (8, 8, 3)), rtol=1e-6)
    assert np.all(mean[..., 3] == 1.0)


def test_texture_shaders_and_normal_maps_known_answers(oracle_lib):
    """Triplanar colour and float shaders (object-space and camera-space weights), the uv
    shader, a normal-map texture and a constant normal map at random hits of the
    shader workload, against an independent float64 restatement (texel choices may flip
    where float rounding crosses a texel edge: at most 1% of the records)."""
    from aurora_b200 import scenes
    from shade_points import expected, hit_records
    data = scenes.shader_scene(32, 32, sphere_level=2)
    rec = hit_records(data, 3000, 41)
    got = oracle_lib.OracleScene(data, np.zeros((21, 64, 32), np.float32)).probe(10, rec)
    want = expected(data, rec)
    bad = np.any(np.abs(got - want) > 2e-5 + 2e-5 * np.abs(want), axis=1)
    assert bad.mean() <= 0.01, (bad.sum(), got[bad][:2], want[bad][:2])
    # every kind of shading point was exercised
    attr = data.tri_attr[rec[:, 0].astype(np.int64)]
    assert all(np.count_nonzero(attr == a) > 300 for a in range(5))
    # the normal maps tilt the shading normal away from Ng
    assert np.mean(np.sum(got[:, :3] * got[:, 3:6], 1) < 0.999) > 0.3


def test_light_samples_passes(oracle_lib):
    """lightsamples (Integrator::integrateCameraSample's numSamples): the first pass traces one
    path per camera sample, later passes L paths from the camera ray's first hit, averaged;
    the estimate stays unbiased."""
    from aurora_b200 import scenes
    data = scenes.box_scene(16, 16, spp=8)
    osc = oracle_lib.OracleScene(data, np.zeros((21, 64, 32), np.float32))
    one, _, c1 = osc.render(1, 5, 5, 1, want_m2=False)
    four, _, c4 = osc.render(1, 5, 5, 1, want_m2=False, light_samples=4)
    np.testing.assert_array_equal(one, four)                 # pass 0: one path either way
    _, _, c = osc.render(3, 5, 5, 1, want_m2=False, light_samples=4)
    assert int(c[2]) == 16 * 16 * (1 + 4 + 4)
    a, m2a, _ = osc.render(64, 5, 5, 3)
    b, m2b, _ = osc.render(64, 5, 5, 3, light_samples=4)
    np.testing.assert_array_equal(a[..., 3], b[..., 3])       # the same camera rays
    sig = np.sqrt(m2a / 63 / 64 + m2b / 63 / 64)
    assert np.mean(np.abs(a[..., :3] - b[..., :3]) <= 4 * sig + 1e-6) > 0.98
    # L paths per pass lower the pass variance (the median pixel's: pixels that see the light
    # keep the camera jitter's variance, which the sub-paths share)
    assert np.median(m2b[..., :3]) < 0.6 * np.median(m2a[..., :3])


@pytest.mark.parametrize("max_depth", [1, 2, 3])
def test_mirror_escape_sees_environment(oracle_lib, max_depth):
    """integrator.cpp:255-274: the ray after a mirror vertex that escapes adds the environment,
    evaluated along the camera ray, times the throughput; this includes the ray after the LAST
    shaded vertex (max_depth 1). A mirror quad (specular colour s) that fills the view under a
    constant environment E * 2^x: every pixel is exactly E * 2^x * s, with alpha 1, and every
    path traces two closest-hit rays (the camera ray and the escaping reflection)."""
    from aurora_b200 import scenes
    spec, env, x = (0.8, 0.6, 0.4), (0.5, 1.0, 2.0), 1.0
    data = scenes.mirror_quad_scene(max_depth=max_depth, spec=spec, env=env, exposure=x)
    mean, m2, counts = oracle_lib.OracleScene(data).render(4, max_depth, max_depth, 9)
    want = np.array(env, np.float64) * 2.0 ** x * np.array(spec, np.float64)
    np.testing.assert_allclose(mean[..., :3], np.broadcast_to(want, mean[..., :3].shape), rtol=1e-6)
    assert (mean[..., 3] == 1.0).all()
    assert int(counts[0]) == 2 * 16 * 16 * 4 and int(counts[1]) == 0

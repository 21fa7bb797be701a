"""Rendered images of the plain renderer against the CPU restatement at equal spp:
per-pixel mean within 3 sigma (criterion c). Both sides consume the same
counter-based random numbers, so the images agree far more tightly than 3 sigma."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def compare(gpu, mean, m2, spp, max_frac=0.005):
    var = m2 / max(spp - 1, 1)
    sig = np.sqrt(var / spp)
    d = np.abs(gpu[..., :3].astype(np.float64) - mean[..., :3])
    bad = d > 3 * sig + 1e-4 * (1 + np.abs(mean[..., :3]))
    frac = bad.any(-1).mean()
    assert frac <= max_frac, (frac, np.argwhere(bad.any(-1))[:5])
    assert np.array_equal(gpu[..., 3], mean[..., 3].astype(np.float32))
    return frac, float(d.max())


def render_both(ctx, oracle_lib, data, tables, spp, crop=None, mode=0):
    import aurora_b200 as ab
    r = data.render
    scene = ab.Scene(ctx, data)
    res = scene.render(ab.render_opts(spp, r["max_depth"], r["min_depth"], r["seed"], mode=mode))
    osc = oracle_lib.OracleScene(data, tables)
    mean, m2, counts = osc.render(spp, r["max_depth"], r["min_depth"], r["seed"], crop=crop)
    g = res.film if crop is None else res.film[crop[1]:crop[1] + crop[3], crop[0]:crop[0] + crop[2]]
    return g, mean, m2, counts, res.stats


def test_box_scene_256_16spp(ctx, oracle_lib, kelemen_tables):
    from aurora_b200 import scenes
    data = scenes.box_scene()
    g, mean, m2, counts, stats = render_both(ctx, oracle_lib, data, kelemen_tables, 16)
    frac, dmax = compare(g, mean, m2, 16)
    assert stats["paths"] == 256 * 256 * 16
    assert abs(stats["closest_rays"] - int(counts[0])) <= 1e-3 * counts[0]
    assert abs(stats["shadow_rays"] - int(counts[1])) <= 1e-3 * counts[1]
    print(f"\nbox: {frac:.5f} of pixels beyond 3 sigma, max |diff| {dmax:.3g}")


def test_sphere_scene_crop(ctx, oracle_lib, kelemen_tables):
    from aurora_b200 import scenes
    data = scenes.sphere_scene(256, 256)
    g, mean, m2, counts, stats = render_both(ctx, oracle_lib, data, kelemen_tables, 16, crop=(64, 64, 128, 128))
    compare(g, mean, m2, 16)


def test_texture_scene(ctx, oracle_lib, kelemen_tables):
    from aurora_b200 import scenes
    data = scenes.texture_scene(96, 96)
    g, mean, m2, counts, stats = render_both(ctx, oracle_lib, data, kelemen_tables, 8)
    compare(g, mean, m2, 8)


GLASS = dict(type_=5, specular=(1.0, 1.0, 1.0), diffuse=(0.95, 0.9, 0.85), reflectance=0.04, ior=1.5)


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_glass_boxes(ctx, oracle_lib, kelemen_tables, mode):
    """glassMaterial boxes: Fresnel-chosen mirror / transmission lobes, the MirrorRay branch
    (emission seen through glass, no next-event estimate, no roulette depth), with
    roulette from the second bounce."""
    from aurora_b200 import scenes
    data = scenes.box_scene(128, 128, max_depth=8, box_mat=GLASS, lift=0.01)
    data.render["min_depth"] = 1
    g, mean, m2, counts, stats = render_both(ctx, oracle_lib, data, kelemen_tables, 16, mode=mode)
    compare(g, mean, m2, 16)


ENV_MAP = np.random.default_rng(15).uniform(0.05, 4.0, (32, 64, 3)).astype(np.float32)


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
@pytest.mark.parametrize("env", [dict(color=(0.4, 0.5, 0.7), exposure=0.0),
                                 dict(color=(1, 1, 1), exposure=-1.0, texture=ENV_MAP)], ids=["constant", "map"])
def test_environment_light(ctx, oracle_lib, kelemen_tables, mode, env):
    """InfiniteAreaLight: seen by camera rays that miss (alpha 1), sampled by next-event
    estimation and weighted against BRDF samples by MIS, and seen through a glass sphere by
    mirror rays that escape (evaluated along the camera ray, as the reference does)."""
    from aurora_b200 import scenes
    glass = dict(type_=5, specular=(1.0, 1.0, 1.0), diffuse=(0.9, 0.95, 1.0), reflectance=0.04, ior=1.5)
    data = scenes.sphere_scene(96, 96, env=env, sphere_mat=glass)
    g, mean, m2, counts, stats = render_both(ctx, oracle_lib, data, kelemen_tables, 16, mode=mode)
    compare(g, mean, m2, 16)
    assert (mean[..., 3] == 1.0).all()     # every pixel sees geometry or the environment


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
@pytest.mark.parametrize("max_depth", [1, 2])
def test_mirror_escape_after_last_vertex(ctx, mode, max_depth):
    """A mirror quad filling the view under a constant environment light: the reflection of every
    camera ray escapes, after the last shaded vertex at max_depth 1 (integrator.cpp:255-274), so
    every pixel is exactly env * 2^exposure * specular colour."""
    import aurora_b200 as ab
    from aurora_b200 import scenes
    spec, env, x = (0.8, 0.6, 0.4), (0.5, 1.0, 2.0), 1.0
    data = scenes.mirror_quad_scene(max_depth=max_depth, spec=spec, env=env, exposure=x)
    scene = ab.Scene(ctx, data)
    res = scene.render(ab.render_opts(4, max_depth, max_depth, 9, mode=mode))
    want = np.array(env, np.float64) * 2.0 ** x * np.array(spec, np.float64)
    np.testing.assert_allclose(res.film[..., :3], np.broadcast_to(want, res.film[..., :3].shape), rtol=1e-6)
    assert (res.film[..., 3] == 1.0).all()
    assert res.stats["closest_rays"] == 2 * 16 * 16 * 4
    scene.close()


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
@pytest.mark.parametrize("max_depth", [2, 3])
def test_glass_under_env_map_shallow(ctx, oracle_lib, kelemen_tables, mode, max_depth):
    """A glass sphere under an environment map at depth 2 and 3: many mirror and transmission
    rays escape right after the last shaded vertex and add the map along the camera ray."""
    from aurora_b200 import scenes
    glass = dict(type_=5, specular=(1.0, 1.0, 1.0), diffuse=(0.9, 0.95, 1.0), reflectance=0.04, ior=1.5)
    data = scenes.sphere_scene(96, 96, max_depth=max_depth, env=dict(color=(1, 1, 1), exposure=-1.0, texture=ENV_MAP),
                               sphere_mat=glass)
    g, mean, m2, counts, stats = render_both(ctx, oracle_lib, data, kelemen_tables, 16, mode=mode)
    compare(g, mean, m2, 16)
    if mode == 0:
        assert stats["closest_rays"] == int(counts[0])


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_environment_map_with_kelemen(ctx, oracle_lib, kelemen_tables, mode):
    from aurora_b200 import scenes
    data = scenes.sphere_scene(96, 96, env=dict(color=(1, 1, 1), exposure=0.0, texture=ENV_MAP))
    g, mean, m2, counts, stats = render_both(ctx, oracle_lib, data, kelemen_tables, 16, mode=mode)
    compare(g, mean, m2, 16)


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_texture_shaders_and_normal_maps(ctx, oracle_lib, kelemen_tables, mode):
    """Triplanar colour and roughness shaders, a normal-map texture and a constant normal map."""
    from aurora_b200 import scenes
    data = scenes.shader_scene(96, 96)
    g, mean, m2, counts, stats = render_both(ctx, oracle_lib, data, kelemen_tables, 8, mode=mode)
    compare(g, mean, m2, 8)


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_progressive_passes(ctx, mode):
    """aur_render_progressive: passes of 5 samples give the running mean after each pass and,
    complete, the single render's film; a callback that returns True stops the render."""
    import aurora_b200 as ab
    from aurora_b200 import scenes
    data = scenes.box_scene(64, 64, spp=16)
    r = data.render
    scene = ab.Scene(ctx, data)
    whole = scene.render(ab.render_opts(16, r["max_depth"], r["min_depth"], r["seed"], mode=mode)).film
    seen = []
    res = scene.render_progressive(ab.render_opts(16, r["max_depth"], r["min_depth"], r["seed"], mode=mode), 5,
                                   lambda img, done: seen.append((done, img)) and False)
    assert [d for d, _ in seen] == [5, 10, 15, 16] and res.stats["paths"] == 64 * 64 * 16
    np.testing.assert_allclose(res.film, whole, rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(seen[-1][1], res.film)
    ten = scene.render(ab.render_opts(10, r["max_depth"], r["min_depth"], r["seed"], mode=mode)).film
    stopped = scene.render_progressive(ab.render_opts(16, r["max_depth"], r["min_depth"], r["seed"], mode=mode), 5,
                                       lambda img, done: done >= 10)
    np.testing.assert_allclose(stopped.film, ten, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(seen[1][1], ten, rtol=1e-5, atol=1e-6)
    scene.close()


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_light_samples(ctx, oracle_lib, kelemen_tables, mode):
    """light_samples 4: passes after the first trace four paths from the camera ray's first
    hit, each firefly-filtered and added as Lo / 4, on the device as in the oracle; the plain
    and the wavefront renderer give the same film. Also from a sample offset (no first pass)."""
    import aurora_b200 as ab
    from aurora_b200 import scenes
    data = scenes.sphere_scene(48, 48, env=dict(color=(0.3, 0.35, 0.4)))
    scene = ab.Scene(ctx, data)
    osc = oracle_lib.OracleScene(data, kelemen_tables)
    for offset in (0, 5):
        res = scene.render(ab.render_opts(8, 6, 6, 2, mode=mode, light_samples=4, sample_offset=offset))
        mean, m2, counts = osc.render(8, 6, 6, 2, light_samples=4, sample_offset=offset)
        compare(res.film, mean, m2, 8)          # 8 passes: the alpha means are exact in float
        assert res.stats["paths"] == 48 * 48 * (8 * 4 - (3 if offset == 0 else 0)) == int(counts[2])
        if mode == 1:
            plain = scene.render(ab.render_opts(8, 6, 6, 2, light_samples=4, sample_offset=offset)).film
            np.testing.assert_allclose(res.film, plain, rtol=1e-6, atol=1e-7)
    scene.close()


def test_terrain_small(ctx, oracle_lib, kelemen_tables):
    """The large-scene generator at reduced size (roulette, 16 materials, 4 lights, depth 8)."""
    from aurora_b200 import scenes
    data = scenes.terrain_scene(160, 90, grid=129, spheres=32, sphere_level=2)
    g, mean, m2, counts, stats = render_both(ctx, oracle_lib, data, kelemen_tables, 8)
    compare(g, mean, m2, 8)


def test_progressive_and_fp64(ctx):
    import aurora_b200 as ab
    from aurora_b200 import scenes
    data = scenes.box_scene(64, 64)
    scene = ab.Scene(ctx, data)
    full = scene.render(ab.render_opts(16, 5, 5, 1)).film
    a = scene.render(ab.render_opts(8, 5, 5, 1, sample_offset=0)).film
    b = scene.render(ab.render_opts(8, 5, 5, 1, sample_offset=8)).film
    np.testing.assert_allclose((a + b) / 2, full, rtol=1e-5, atol=1e-6)
    f64 = scene.render_f64(ab.render_opts(16, 5, 5, 1)).film
    np.testing.assert_allclose(f64, full, rtol=1e-5, atol=1e-6)
    c = scene.render(ab.render_opts(16, 5, 5, 1)).film
    assert np.array_equal(c, full)    # deterministic


def test_invalid_options(ctx):
    import aurora_b200 as ab
    from aurora_b200 import scenes
    scene = ab.Scene(ctx, scenes.box_scene(16, 16))
    for bad in (ab.render_opts(0, 5, 5, 1), ab.render_opts(4, 0, 5, 1), ab.render_opts(4, 5, 5, 1, sample_offset=-1),
                ab.render_opts(4, 5, 5, 1, mode=7)):
        with pytest.raises(ab.AuroraError):
            scene.render(bad)


@pytest.mark.parametrize("rough", [0.15, 0.4])
@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_ct_direct_lighting_known_answer(ctx, mode, rough):
    """Glossy next-event estimation with MIS on the device against the closed-form expectation
    of the reference's estimator (the sampler's N.H > 0.999 cap included). Every pixel of the
    16 x 16 film sees the same point at fov slope 1e-4, so the pixels are independent
    estimates of one value and their spread gives the standard error."""
    import aurora_b200 as ab
    from test_oracle import ct_plane_under_light
    data, want, plain = ct_plane_under_light(rough)
    spp = 16384
    res = ab.Scene(ctx, data).render(ab.render_opts(spp, 1, 1, 5, mode=mode))
    px = res.film[..., 0].astype(np.float64).ravel()
    got, se = px.mean(), px.std(ddof=1) / np.sqrt(px.size)
    assert abs(got - want) < 4 * se + 1e-4 * want, (got, want, plain, se)
    assert se < 0.0015 * want


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_sphere_light_known_answer(ctx, mode):
    """The sphere light's cone sampling on the device against the closed-form irradiance."""
    import aurora_b200 as ab
    from test_oracle import lambert_plane_under_sphere
    data, want = lambert_plane_under_sphere()
    res = ab.Scene(ctx, data).render(ab.render_opts(4096, 1, 1, 9, mode=mode))
    px = res.film[..., 0].astype(np.float64).ravel()
    got, se = px.mean(), px.std(ddof=1) / np.sqrt(px.size)
    assert abs(got - want) < 4 * se + 1e-4 * want, (got, want, se)
    assert se < 0.002 * want


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_kelemen_lobe_choice_known_answer(ctx, kelemen_tables, mode):
    """The Kelemen lobe choice on the device (its own albedo tables) against
    A E_ct + (1 - A) E_lambert, A read from those tables at (N.V, roughness)."""
    import aurora_b200 as ab
    from test_oracle import kelemen_plane_under_light
    data, want, A = kelemen_plane_under_light(kelemen_tables)
    assert 0.05 < A < 0.95
    res = ab.Scene(ctx, data).render(ab.render_opts(16384, 1, 1, 7, mode=mode))
    px = res.film[..., 0].astype(np.float64).ravel()
    got, se = px.mean(), px.std(ddof=1) / np.sqrt(px.size)
    assert abs(got - want) < 4 * se + 1e-4 * want, (got, want, A, se)
    assert se < 0.005 * want


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_metal_known_answer(ctx, mode):
    """Metal's Schlick tint and two-roughness mixture on the device against the closed form."""
    import aurora_b200 as ab
    from test_oracle import metal_plane_under_light
    data, want = metal_plane_under_light()
    res = ab.Scene(ctx, data).render(ab.render_opts(16384, 1, 1, 11, mode=mode))
    px = res.film[..., :3].astype(np.float64).reshape(-1, 3)
    got, se = px.mean(0), px.std(0, ddof=1) / np.sqrt(px.shape[0])
    assert np.all(np.abs(got - want) < 4 * se + 1e-4 * want), (got, want, se)
    assert np.all(se < 0.005 * want)

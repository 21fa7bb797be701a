"""The wavefront (batched) renderer against the plain renderer: same estimator, same
random numbers, same compensated accumulation order -> the same film; and the
64-scene batch against rendering each scene alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def both(ctx, data, spp, **wf):
    import aurora_b200 as ab
    from aurora_b200 import _abi
    r = data.render
    scene = ab.Scene(ctx, data)
    plain = scene.render(ab.render_opts(spp, r["max_depth"], r["min_depth"], r["seed"]))
    wave = scene.render(ab.render_opts(spp, r["max_depth"], r["min_depth"], r["seed"], mode=_abi.RENDER_WAVEFRONT,
                                       **wf))
    scene.close()
    return plain, wave


@pytest.mark.parametrize("cfg", [dict(wf_sort=0), dict(wf_sort=1), dict(wf_pool=2048, wf_block=64, wf_sort=1),
                                 dict(wf_pool=1 << 16, wf_block=256, wf_sort=0)])
def test_box_matches_plain(ctx, kelemen_tables, cfg):
    from aurora_b200 import scenes
    plain, wave = both(ctx, scenes.box_scene(128, 128), 16, **cfg)
    np.testing.assert_allclose(wave.film, plain.film, rtol=1e-6, atol=1e-7)
    assert wave.stats["paths"] == 128 * 128 * 16


def test_sphere_and_terrain_match_plain(ctx, kelemen_tables):
    from aurora_b200 import scenes
    for data, spp in ((scenes.sphere_scene(96, 96), 8),
                      (scenes.terrain_scene(160, 90, grid=129, spheres=32, sphere_level=2), 8),
                      (scenes.texture_scene(64, 64), 4)):
        plain, wave = both(ctx, data, spp)
        np.testing.assert_allclose(wave.film, plain.film, rtol=1e-6, atol=1e-7)


def test_batch_matches_single_renders(ctx):
    """12 scenes of the batch against their single renders on the same (4-wide) tree."""
    import aurora_b200 as ab
    from aurora_b200 import scenes, _abi
    datas = scenes.batch_scenes(12)
    objs = [ab.Scene(ctx, d) for d in datas]
    opts = [ab.render_opts(d.render["spp"], d.render["max_depth"], d.render["min_depth"], d.render["seed"],
                           mode=_abi.RENDER_WAVEFRONT) for d in datas]
    films, stats = ab.render_batch(objs, opts)
    assert stats["paths"] == sum(d.width * d.height * d.render["spp"] for d in datas)
    for d, s, f in zip(datas, objs, films):
        alone = s.render(ab.render_opts(d.render["spp"], d.render["max_depth"], d.render["min_depth"],
                                        d.render["seed"], mode=_abi.RENDER_WAVEFRONT)).film
        np.testing.assert_allclose(f, alone, rtol=1e-6, atol=1e-7)
    for s in objs:
        s.close()


def test_invalid_wavefront_configs(ctx):
    import aurora_b200 as ab
    from aurora_b200 import scenes, _abi
    scene = ab.Scene(ctx, scenes.box_scene(16, 16))
    for bad in (dict(wf_pool=1000), dict(wf_block=100), dict(wf_block=512), dict(wf_pool=1 << 27)):
        with pytest.raises(ab.AuroraError):
            scene.render(ab.render_opts(1, 5, 5, 1, mode=_abi.RENDER_WAVEFRONT, **bad))


def test_autotuned_config(ctx):
    """Default options autotune pool size, block size and the sort switch once per scene."""
    import aurora_b200 as ab
    from aurora_b200 import scenes, _abi
    data = scenes.box_scene(96, 96)
    scene = ab.Scene(ctx, data)
    r = data.render
    plain = scene.render(ab.render_opts(8, r["max_depth"], r["min_depth"], r["seed"]))
    a = scene.render(ab.render_opts(8, r["max_depth"], r["min_depth"], r["seed"], mode=_abi.RENDER_WAVEFRONT))
    b = scene.render(ab.render_opts(8, r["max_depth"], r["min_depth"], r["seed"], mode=_abi.RENDER_WAVEFRONT))
    cfg = a.stats["wf_config"]
    assert cfg["pool"] in (1 << 20, 1 << 21, 1 << 22) and cfg["block"] in (128, 256) and cfg["sort"] in (0, 1)
    assert b.stats["wf_config"] == cfg
    np.testing.assert_allclose(a.film, plain.film, rtol=1e-6, atol=1e-7)
    assert sum(a.stats["stage_ms"].values()) > 0
    scene.close()


def test_batch_with_light_samples(ctx):
    """Scenes of one batch may use different light_samples: each film equals its single
    wavefront render."""
    import aurora_b200 as ab
    from aurora_b200 import scenes, _abi
    datas = [scenes.box_scene(64, 64, spp=6), scenes.sphere_scene(48, 48, spp=5), scenes.box_scene(32, 48, spp=4)]
    ls = [1, 3, 2]
    objs = [ab.Scene(ctx, d) for d in datas]
    opts = [ab.render_opts(d.render["spp"], d.render["max_depth"], d.render["min_depth"], d.render["seed"],
                           mode=_abi.RENDER_WAVEFRONT, light_samples=l) for d, l in zip(datas, ls)]
    films, stats = ab.render_batch(objs, opts)
    want = sum(d.width * d.height * (d.render["spp"] * l - (l - 1)) for d, l in zip(datas, ls))
    assert stats["paths"] == want
    for s, o, f in zip(objs, opts, films):
        np.testing.assert_allclose(f, s.render(o).film, rtol=1e-6, atol=1e-7)
    for s in objs:
        s.close()

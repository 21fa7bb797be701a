"""Parity at the full sizes of the stated workloads: the device films against the CPU
oracle at equal spp (per-pixel mean within 3 sigma, the oracle's Welford variance), the
64-scene batch against single renders, and the differentiable workload's gradients
against central finite differences at h = 1e-3, 4096 spp, common random numbers.

  sphere    Kelemen icosphere, 512x512, 64 spp, depth 6 (whole image)
  terrain   3.4 M triangles, 1920x1080, 64 spp, depth 8, roulette after bounce 2
            (32 full-width rows spread over the frame; the GPU renders the whole frame)
  batch     64 box scenes of uneven resolution, spp and depth in one wavefront launch
            (all 64 against single renders; 8 against the oracle)
  texture   the differentiable workload, 256x256, 256 spp (forward), 4096 spp (gradients)
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _beyond_3sigma(gpu, mean, m2, spp):
    """Fraction of pixels with a channel beyond 3 sigma of the oracle's mean (plus a 1e-4
    relative floor for pixels whose samples are all equal)."""
    sig = np.sqrt(m2 / max(spp - 1, 1) / spp)
    d = np.abs(gpu[..., :3].astype(np.float64) - mean[..., :3])
    bad = d > 3 * sig + 1e-4 * (1 + np.abs(mean[..., :3]))
    return float(bad.any(-1).mean()), float(d.max())


def _same_film(a, b, max_frac=1e-5):
    """Films of two renderers that trace the same paths: equal (rtol 1e-6) except where a ray hits
    two triangles at exactly the same distance (a shared edge, a face lying in another's plane),
    which the binary tree (plain renderer) and the 4-wide tree (wavefront renderer) may resolve to
    different triangles; such pixels are at most max_frac of the film."""
    bad = ~np.isclose(a, b, rtol=1e-6, atol=1e-7).all(-1)
    assert bad.mean() <= max_frac, (int(bad.sum()), bad.size)
    return int(bad.sum())


def _render(ctx, data, spp, mode, **kw):
    import aurora_b200 as ab
    r = data.render
    scene = ab.Scene(ctx, data)
    res = scene.render(ab.render_opts(spp, r["max_depth"], r["min_depth"], r["seed"], mode=mode, **kw))
    scene.close()
    return res


def test_sphere_512_64spp_whole_image(ctx, oracle_lib, kelemen_tables):
    from aurora_b200 import _abi, scenes
    data = scenes.sphere_scene()
    assert (data.width, data.height, data.render["spp"], data.render["max_depth"]) == (512, 512, 64, 6)
    plain = _render(ctx, data, 64, _abi.RENDER_PLAIN)
    wave = _render(ctx, data, 64, _abi.RENDER_WAVEFRONT)
    _same_film(wave.film, plain.film)
    r = data.render
    mean, m2, counts = oracle_lib.OracleScene(data, kelemen_tables).render(64, r["max_depth"], r["min_depth"],
                                                                          r["seed"])
    frac, dmax = _beyond_3sigma(plain.film, mean, m2, 64)
    print(f"\nsphere 512^2 64 spp: {frac:.5f} of pixels beyond 3 sigma, max |diff| {dmax:.3g}")
    assert frac <= 0.005
    assert np.array_equal(plain.film[..., 3], mean[..., 3].astype(np.float32))
    assert plain.stats["paths"] == int(counts[2]) == 512 * 512 * 64
    assert plain.stats["closest_rays"] == int(counts[0]) and plain.stats["shadow_rays"] == int(counts[1])


def test_terrain_1080p_rows_64spp(ctx, oracle_lib, kelemen_tables):
    from aurora_b200 import _abi, scenes
    data = scenes.terrain_scene()
    W, H, r = data.width, data.height, data.render
    assert (W, H, r["spp"], r["max_depth"], r["min_depth"]) == (1920, 1080, 64, 8, 2)
    wave = _render(ctx, data, 64, _abi.RENDER_WAVEFRONT, wf_pool=1 << 22, wf_block=256, wf_sort=1)
    plain = _render(ctx, data, 64, _abi.RENDER_PLAIN)
    ties = _same_film(wave.film, plain.film)
    print(f"\nterrain: {ties} pixels differ between the plain and wavefront films (exact-distance ties)")
    osc = oracle_lib.OracleScene(data, kelemen_tables)
    rows = sorted({int(j * H / 32) + 7 for j in range(32)})
    worst = 0.0
    for y in rows:
        mean, m2, _ = osc.render(64, r["max_depth"], r["min_depth"], r["seed"], crop=(0, y, W, 1))
        frac, dmax = _beyond_3sigma(wave.film[y:y + 1], mean, m2, 64)
        worst = max(worst, frac)
        assert np.array_equal(wave.film[y:y + 1, :, 3], mean[..., 3].astype(np.float32)), y
    print(f"\nterrain rows {len(rows)}: worst row {worst:.5f} of pixels beyond 3 sigma")
    assert worst <= 0.01


def test_batch_of_64_scenes(ctx, oracle_lib, kelemen_tables):
    """All 64 scenes (seed 6+i) in one wavefront launch equal their single wavefront renders (the
    same tree and arithmetic: rtol 1e-6 everywhere) and their single plain renders up to
    exact-distance ties; the 8 cheapest (plus one of each depth) also against the oracle."""
    import aurora_b200 as ab
    from aurora_b200 import _abi, scenes
    datas = scenes.batch_scenes(64)
    assert len({(d.width, d.render["spp"], d.render["max_depth"]) for d in datas}) > 20
    objs = [ab.Scene(ctx, d) for d in datas]
    opts = [ab.render_opts(d.render["spp"], d.render["max_depth"], d.render["min_depth"], d.render["seed"],
                           mode=_abi.RENDER_WAVEFRONT) for d in datas]
    films, stats = ab.render_batch(objs, opts)
    assert stats["paths"] == sum(d.width * d.height * d.render["spp"] for d in datas)
    for d, s, f in zip(datas, objs, films):
        r = d.render
        alone = s.render(ab.render_opts(r["spp"], r["max_depth"], r["min_depth"], r["seed"],
                                        mode=_abi.RENDER_WAVEFRONT)).film
        np.testing.assert_allclose(f, alone, rtol=1e-6, atol=1e-7, err_msg=d.name)
        plain = s.render(ab.render_opts(r["spp"], r["max_depth"], r["min_depth"], r["seed"])).film
        _same_film(f, plain, max_frac=1e-4)
    for s in objs:
        s.close()
    cost = [d.width * d.height * d.render["spp"] * d.render["max_depth"] for d in datas]
    picks = list(np.argsort(cost)[:8])
    for depth in (3, 5, 8):   # at least one scene of each depth
        if not any(datas[i].render["max_depth"] == depth for i in picks):
            picks.append(min((i for i, d in enumerate(datas) if d.render["max_depth"] == depth),
                             key=lambda i: cost[i]))
    for i in picks:
        d = datas[i]
        r = d.render
        mean, m2, _ = oracle_lib.OracleScene(d, kelemen_tables).render(r["spp"], r["max_depth"], r["min_depth"],
                                                                      r["seed"])
        frac, dmax = _beyond_3sigma(films[i], mean, m2, r["spp"])
        print(f"\n{d.name} {d.width}^2 {r['spp']} spp depth {r['max_depth']}: {frac:.5f} beyond 3 sigma")
        assert frac <= 0.005, d.name


def test_texture_256_256spp_forward(ctx, oracle_lib, kelemen_tables):
    from aurora_b200 import _abi, scenes
    data = scenes.texture_scene()
    assert (data.width, data.render["spp"]) == (256, 256)
    r = data.render
    wave = _render(ctx, data, 256, _abi.RENDER_WAVEFRONT)
    mean, m2, counts = oracle_lib.OracleScene(data, kelemen_tables).render(256, r["max_depth"], r["min_depth"],
                                                                          r["seed"])
    frac, dmax = _beyond_3sigma(wave.film, mean, m2, 256)
    print(f"\ntexture 256^2 256 spp: {frac:.5f} of pixels beyond 3 sigma, max |diff| {dmax:.3g}")
    assert frac <= 0.005
    assert wave.stats["paths"] == int(counts[2])


def test_texture_gradients_match_fd_h1e3_4096spp(ctx):
    """Gradients of L = sum(w * image) with respect to the sphere's diffuse colour and to texels of
    the ground's texture against central differences at h = 1e-3 with 4096 spp and common random
    numbers. Roulette is off and Lambert sampling does not depend on the diffuse colour, so the
    estimator is smooth in these parameters: within 2%."""
    import aurora_b200 as ab
    from aurora_b200 import _abi, scenes
    data = scenes.texture_scene()
    r = data.render
    scene = ab.Scene(ctx, data)
    spp, h = 4096, 1e-3
    w = np.random.default_rng(31).normal(size=(256, 256, 4)).astype(np.float32)
    w[..., 3] = 0.0
    p0, t0 = data.material_params(), data.texels()

    def loss(p, t):
        scene.set_params(p, t)
        film = scene.render(ab.render_opts(spp, r["max_depth"], r["min_depth"], r["seed"],
                                           mode=_abi.RENDER_WAVEFRONT)).film
        return float(np.sum(film.astype(np.float64) * w))

    scene.set_params(p0, t0)
    gm, gt, _ = scene.adjoint(ab.render_opts(spp, r["max_depth"], r["min_depth"], r["seed"],
                                             mode=_abi.RENDER_WAVEFRONT), w)
    checks = []
    for c in range(3):                               # the Kelemen sphere's diffuse colour (material 1)
        v = np.zeros_like(p0)
        v[1, c] = 1.0
        checks.append((v, None))
    for i in np.argsort(-np.abs(gt))[:4]:            # the texels with the largest gradients
        vt = np.zeros_like(t0)
        vt[i] = 1.0
        checks.append((None, vt))
    for v, vt in checks:
        pp, pm = (p0 + h * v, p0 - h * v) if v is not None else (p0, p0)
        tp, tm = (t0 + h * vt, t0 - h * vt) if vt is not None else (t0, t0)
        fd = (loss(pp, tp) - loss(pm, tm)) / (2 * h)
        ad = float(np.sum(gm * v)) if v is not None else float(np.sum(gt * vt))
        print(f"\nadjoint {ad:.6g} fd {fd:.6g}")
        assert abs(ad - fd) <= 0.02 * abs(fd), (ad, fd)
    scene.set_params(p0, t0)
    scene.close()

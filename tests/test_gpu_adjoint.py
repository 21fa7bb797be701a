"""Path-replay adjoint against central finite differences with common random numbers,
and the torch.autograd binding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def setup(ctx, res=48):
    import aurora_b200 as ab
    from aurora_b200 import scenes
    data = scenes.texture_scene(res, res)
    scene = ab.Scene(ctx, data)
    rng = np.random.default_rng(17)
    w = rng.normal(size=(res, res, 4)).astype(np.float32)
    w[..., 3] = 0.0
    return data, scene, w


def loss(scene, params, texels, w, spp, seed=2):
    import aurora_b200 as ab
    from aurora_b200 import _abi
    scene.set_params(params, texels)
    film = scene.render(ab.render_opts(spp, 6, 6, seed, mode=_abi.RENDER_WAVEFRONT)).film
    return float(np.sum(film.astype(np.float64) * w))


def adjoint(scene, w, spp, seed=2, mode=0):
    import aurora_b200 as ab
    gm, gt, stats = scene.adjoint(ab.render_opts(spp, 6, 6, seed, mode=mode), w)
    return gm.astype(np.float64), gt.astype(np.float64), stats


def test_albedo_and_texel_gradients_match_fd(ctx):
    """Lambert sampling does not depend on the diffuse colour, so with common random numbers the
    estimator is smooth in it and the adjoint equals the finite difference sample by sample."""
    data, scene, w = setup(ctx)
    p0, t0 = data.material_params(), data.texels()
    spp = 16
    gm, gt, stats = adjoint(scene, w, spp)
    assert stats["paths"] == 48 * 48 * spp
    h = 1e-3
    rng = np.random.default_rng(5)
    checks = []
    for c in range(3):                      # Kelemen sphere diffuse colour (material 1)
        v = np.zeros_like(p0); v[1, c] = 1.0
        checks.append((v, None))
    for _ in range(2):                      # random texel directions
        vt = rng.normal(size=t0.shape).astype(np.float32)
        checks.append((None, vt))
    for v, vt in checks:
        pp = p0 + h * v if v is not None else p0
        pm = p0 - h * v if v is not None else p0
        tp = t0 + h * vt if vt is not None else t0
        tm = t0 - h * vt if vt is not None else t0
        fd = (loss(scene, pp, tp, w, spp) - loss(scene, pm, tm, w, spp)) / (2 * h)
        ad = (np.sum(gm * v) if v is not None else 0.0) + (np.sum(gt * vt) if vt is not None else 0.0)
        assert abs(ad - fd) <= 0.02 * abs(fd) + 1e-3, (ad, fd)
    scene.set_params(p0, t0)


def test_roughness_gradient_matches_fd(ctx):
    """Roughness changes the sampled directions and the Kelemen lobe choice, so the adjoint
    and the finite difference agree in expectation only: both are estimated over 8
    independent sample batches and compared within 3 standard errors. h = 1e-3 keeps
    r +- h inside one cell of the albedo table (the reference's lookup jumps at r = k/31)."""
    import aurora_b200 as ab
    from aurora_b200 import _abi
    data, scene, w = setup(ctx, res=32)
    p0, t0 = data.material_params(), data.texels()
    h, spp, batches = 1e-3, 512, 8
    v = np.zeros_like(p0); v[1, 3] = 1.0
    ads, fds = [], []
    for b in range(batches):
        o = dict(sample_offset=b * spp)
        gm, _, _ = scene.adjoint(ab.render_opts(spp, 6, 6, 2, **o), w)
        ads.append(float(gm[1, 3]))
        vals = []
        for sgn in (1, -1):
            scene.set_params(p0 + sgn * h * v, t0)
            film = scene.render(ab.render_opts(spp, 6, 6, 2, mode=_abi.RENDER_WAVEFRONT, **o)).film
            vals.append(float(np.sum(film.astype(np.float64) * w)))
        scene.set_params(p0, t0)
        fds.append((vals[0] - vals[1]) / (2 * h))
    ad, fd = np.mean(ads), np.mean(fds)
    se = np.sqrt(np.var(ads, ddof=1) / batches + np.var(fds, ddof=1) / batches)
    print(f"\nroughness: adjoint {ad:.5g} +- {np.std(ads, ddof=1) / np.sqrt(batches):.3g}, "
          f"fd {fd:.5g} +- {np.std(fds, ddof=1) / np.sqrt(batches):.3g}")
    assert abs(ad - fd) <= 3 * se + 0.02 * abs(fd), (ad, fd, se)


def test_autograd_function(ctx):
    import torch
    from aurora_b200.pyaurora import AuroraRender
    data, scene, w = setup(ctx, res=32)
    params = torch.tensor(data.material_params(), device="cuda", requires_grad=True)
    texels = torch.tensor(data.texels(), device="cuda", requires_grad=True)
    opts = dict(spp=8, max_depth=6, seed=2)
    img = AuroraRender.apply(params, texels, scene, opts)
    wt = torch.tensor(w, device="cuda")
    (img * wt).sum().backward()
    gm, gt, _ = adjoint(scene, w, 8, mode=1)     # the binding's default mode is wavefront
    np.testing.assert_allclose(params.grad.cpu().numpy(), gm, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(texels.grad.cpu().numpy(), gt, rtol=1e-5, atol=1e-6)
    assert img.shape == (32, 32, 4)


def test_autograd_backward_uses_the_forward_parameters(ctx):
    """forward(A), forward(B), then the backward of A's image: the adjoint replays A's paths under
    A's parameters (not B's, which the scene holds by then) and leaves the scene holding B."""
    import torch
    from aurora_b200.pyaurora import AuroraRender
    data, scene, w = setup(ctx, res=32)
    pa = data.material_params()
    ta = data.texels()
    rng = np.random.default_rng(3)
    pb = np.clip(pa + rng.normal(0, 0.1, pa.shape), 0.05, 0.95).astype(np.float32)
    tb = np.clip(ta + rng.normal(0, 0.1, ta.shape), 0.05, 0.95).astype(np.float32)
    params_a = torch.tensor(pa, device="cuda", requires_grad=True)
    texels_a = torch.tensor(ta, device="cuda", requires_grad=True)
    opts = dict(spp=8, max_depth=6, seed=2)
    img_a = AuroraRender.apply(params_a, texels_a, scene, opts)
    with torch.no_grad():
        AuroraRender.apply(torch.tensor(pb, device="cuda"), torch.tensor(tb, device="cuda"), scene, opts)
    (img_a * torch.tensor(w, device="cuda")).sum().backward()
    held_p, held_t = scene.get_params()
    np.testing.assert_array_equal(held_p, pb)
    np.testing.assert_array_equal(held_t, tb)
    scene.set_params(pa, ta)
    gm, gt, _ = adjoint(scene, w, 8, mode=1)
    np.testing.assert_allclose(params_a.grad.cpu().numpy(), gm, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(texels_a.grad.cpu().numpy(), gt, rtol=1e-5, atol=1e-6)
    scene.set_params(pb, tb)
    gm_b, _, _ = adjoint(scene, w, 8, mode=1)
    assert not np.allclose(gm_b, gm, rtol=1e-3)      # B's gradients differ: the check has teeth


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_adjoint_is_deterministic(ctx, mode):
    data, scene, w = setup(ctx, res=32)
    a = adjoint(scene, w, 8, mode=mode)
    b = adjoint(scene, w, 8, mode=mode)
    assert np.allclose(a[0], b[0], rtol=1e-5, atol=1e-7) and np.allclose(a[1], b[1], rtol=1e-5, atol=1e-7)


def test_wavefront_adjoint_equals_plain_adjoint(ctx):
    """Record pass on the wavefront engine + replay kernel against the megakernel: the same
    paths and the same per-vertex arithmetic, summed in a different order."""
    data, scene, w = setup(ctx, res=48)
    a = adjoint(scene, w, 16, mode=0)
    b = adjoint(scene, w, 16, mode=1)
    assert b[2]["launches"] > 2 and b[2]["closest_rays"] == a[2]["closest_rays"]
    assert b[2]["shadow_rays"] == a[2]["shadow_rays"]
    for x, y in ((a[0], b[0]), (a[1], b[1])):
        np.testing.assert_allclose(y, x, rtol=1e-4, atol=1e-5 * float(np.max(np.abs(x))))


@pytest.mark.parametrize("mode", [0, 1], ids=["megakernel", "wavefront"])
def test_albedo_gradient_known_answer(ctx, mode):
    """Closed form: a Lambert plane under a square light at max_depth 1, seen by all 16 x 16
    pixels at one point (fov slope 1e-4). Each pixel is albedo * E, so the gradient of the
    film's red sum with respect to the red albedo is the sum over the albedo path by path, and
    its expectation is 256 E (E: the quadrature of test_oracle's plane cases)."""
    import math
    import aurora_b200 as ab
    from test_oracle import _plane_under_light, _light_integrals
    albedo, h, s, le, px = 0.6, 1.0, 0.25, 4.0, 0.8
    data = _plane_under_light(albedo, h, s, (le, le, le), px, fov=1e-4)
    want = _light_integrals(0.3, 1.0, np.array([0.0, 1.0, 0.0]), h, s, le, px, 600)[2]
    scene = ab.Scene(ctx, data)
    spp, seed = 4096, 3
    film = scene.render(ab.render_opts(spp, 1, 1, seed, mode=mode)).film
    w = np.zeros((16, 16, 4), np.float32)
    w[..., 0] = 1.0
    gm, gt, _ = scene.adjoint(ab.render_opts(spp, 1, 1, seed, mode=mode), w)
    red = film[..., 0].astype(np.float64).ravel()
    assert abs(gm[0, 0] - red.sum() / albedo) < 1e-4 * gm[0, 0]
    se = red.std(ddof=1) / math.sqrt(red.size) / albedo
    assert abs(gm[0, 0] / red.size - want) < 4 * se + 1e-4 * want, (gm[0, 0] / red.size, want, se)
    assert np.all(gm[0, 1:3] == 0.0)


def test_adjoint_sharded_one_rank_equals_adjoint(ctx):
    """aurora_b200.shard.adjoint_sharded in a one-rank gloo group (its combine is then the
    identity) gives the device adjoint of the whole sample range."""
    import datetime
    import socket
    import torch.distributed as dist
    import aurora_b200 as ab
    from aurora_b200 import scenes
    from aurora_b200.shard import adjoint_sharded
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        data = scenes.texture_scene(64, 64)
        scene = ab.Scene(ctx, data)
        w = np.random.default_rng(4).normal(size=(64, 64, 4)).astype(np.float32)
        opts = ab.render_opts(16, 6, 6, 2, mode=1)
        gm, gt = adjoint_sharded(scene, opts, w)
        gm1, gt1, _ = scene.adjoint(ab.render_opts(16, 6, 6, 2, mode=1), w)
        np.testing.assert_allclose(gm, gm1, rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(gt, gt1, rtol=1e-6, atol=1e-7)
        assert np.any(gm != 0)
    finally:
        dist.destroy_process_group()

"""The device path-replay adjoint against the oracle's FP64 forward-mode adjoint on a
32x32 crop: same paths (same counter-based random numbers), derivatives formed in
reverse in FP32 on the device and forward in FP64 on the CPU.

Tolerance per parameter: |gpu - cpu| <= 2e-3 |cpu| + 2e-4 max|cpu| (the FP32
derivative of the Beckmann term, 2 tan^2/r^3 - 2/r, cancels near the lobe peak).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _compare(gpu, cpu, what):
    gpu = np.asarray(gpu, np.float64).ravel()
    cpu = np.asarray(cpu, np.float64).ravel()
    scale = float(np.max(np.abs(cpu))) if cpu.size else 0.0
    err = np.abs(gpu - cpu)
    bound = 2e-3 * np.abs(cpu) + 2e-4 * scale
    worst = int(np.argmax(err - bound)) if cpu.size else 0
    print(f"\n{what}: max |cpu| {scale:.4g}, max err {err.max() if err.size else 0:.3g}, "
          f"worst #{worst} gpu {gpu[worst] if gpu.size else 0:.6g} cpu {cpu[worst] if cpu.size else 0:.6g}")
    assert np.all(err <= bound), what


def _run(ctx, kelemen_tables, oracle_lib, data, crop, spp, seed, wseed, mode, light_samples=1):
    import aurora_b200 as ab
    H, W = data.height, data.width
    w = np.zeros((H, W, 4), np.float32)
    x0, y0, cw, ch = crop
    w[y0:y0 + ch, x0:x0 + cw, :3] = np.random.default_rng(wseed).normal(size=(ch, cw, 3))
    depth, mind = data.render["max_depth"], data.render["min_depth"]
    scene = ab.Scene(ctx, data)
    gm, gt, _ = scene.adjoint(ab.render_opts(spp, depth, mind, seed, mode=mode, light_samples=light_samples), w)
    scene.close()
    osc = oracle_lib.OracleScene(data, kelemen_tables, use_bvh=True)
    cm, ct = osc.adjoint(spp, depth, mind, seed, w, crop=crop, light_samples=light_samples)
    return gm, gt, cm, ct


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_adjoint_matches_fp64_oracle_texture_scene(ctx, kelemen_tables, oracle_lib, mode):
    """Differentiable workload at 256x256: Kelemen sphere (diffuse + roughness with the lobe
    score term) over the textured ground (texel gradients)."""
    from aurora_b200 import scenes
    data = scenes.texture_scene()
    gm, gt, cm, ct = _run(ctx, kelemen_tables, oracle_lib, data, (112, 180, 32, 32), 64, 2, 21, mode)
    assert np.count_nonzero(ct) > 100 and cm[1, 3] != 0.0
    _compare(gm, cm, "materials (diffuse rgb, roughness)")
    _compare(gt, ct, "texels")


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_adjoint_matches_fp64_oracle_cook_torrance(ctx, kelemen_tables, oracle_lib, mode):
    """Box workload: Cook-Torrance boxes (roughness through eval, MIS and sampled lobes) and
    Lambert walls."""
    from aurora_b200 import scenes
    data = scenes.box_scene(128, 128, spp=64)
    gm, gt, cm, ct = _run(ctx, kelemen_tables, oracle_lib, data, (40, 72, 32, 32), 64, 1, 22, mode)
    assert cm[3, 3] != 0.0
    _compare(gm, cm, "materials (diffuse rgb, roughness)")


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_adjoint_matches_fp64_oracle_through_glass(ctx, kelemen_tables, oracle_lib, mode):
    """Glass boxes in the box workload: the replay follows mirror and transmission vertices
    (T *= colour, no bounce count) to the walls behind them."""
    from aurora_b200 import _abi, scenes
    glass = dict(type_=_abi.MAT_GLASS, specular=(1.0, 1.0, 1.0), diffuse=(0.95, 0.9, 0.85), reflectance=0.04,
                 ior=1.5)
    data = scenes.box_scene(128, 128, spp=64, max_depth=8, box_mat=glass, lift=0.01)
    data.render["min_depth"] = 1
    gm, gt, cm, ct = _run(ctx, kelemen_tables, oracle_lib, data, (40, 72, 32, 32), 64, 1, 23, mode)
    assert np.count_nonzero(cm[:3, :3]) == 9
    _compare(gm, cm, "materials (diffuse rgb, roughness)")


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_adjoint_matches_fp64_oracle_under_an_env_map(ctx, kelemen_tables, oracle_lib, mode):
    """The differentiable workload under an environment map: env next-event estimates and MIS
    weights in dD, and (through a glass sphere) env radiance seen by escaping mirror rays."""
    from aurora_b200 import _abi, scenes
    envmap = np.random.default_rng(16).uniform(0.05, 3.0, (32, 64, 3)).astype(np.float32)
    tex = np.random.default_rng(7).uniform(0.2, 0.8, size=(64, 64, 3)).astype(np.float32)
    data = scenes.sphere_scene(256, 256, 64, 6, 2, ground_texture=tex, env=dict(color=(1, 1, 1), texture=envmap))
    gm, gt, cm, ct = _run(ctx, kelemen_tables, oracle_lib, data, (112, 180, 32, 32), 64, 2, 24, mode)
    _compare(gm, cm, "materials (diffuse rgb, roughness)")
    _compare(gt, ct, "texels")
    glass = dict(type_=_abi.MAT_GLASS, specular=(1.0, 1.0, 1.0), diffuse=(0.9, 0.95, 1.0), reflectance=0.04, ior=1.5)
    data = scenes.sphere_scene(256, 256, 64, 6, 2, ground_texture=tex, env=dict(color=(1, 1, 1), texture=envmap),
                               sphere_mat=glass)
    gm, gt, cm, ct = _run(ctx, kelemen_tables, oracle_lib, data, (112, 150, 32, 32), 64, 2, 25, mode)
    _compare(gm, cm, "materials through glass")
    _compare(gt, ct, "texels through glass")


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_adjoint_matches_fp64_oracle_escape_after_last_vertex(ctx, kelemen_tables, oracle_lib, mode):
    """Depth 2, a glass sphere on the textured ground under an env map: rays that leave the glass
    after the last shaded vertex and escape add the map (integrator.cpp:255-274); their radiance
    enters the gradients of the ground's texels and materials through the replayed throughput."""
    from aurora_b200 import _abi, scenes
    envmap = np.random.default_rng(16).uniform(0.05, 3.0, (32, 64, 3)).astype(np.float32)
    tex = np.random.default_rng(7).uniform(0.2, 0.8, size=(64, 64, 3)).astype(np.float32)
    glass = dict(type_=_abi.MAT_GLASS, specular=(1.0, 1.0, 1.0), diffuse=(0.9, 0.95, 1.0), reflectance=0.04, ior=1.5)
    data = scenes.sphere_scene(256, 256, 64, 2, 2, ground_texture=tex, env=dict(color=(1, 1, 1), texture=envmap),
                               sphere_mat=glass)
    gm, gt, cm, ct = _run(ctx, kelemen_tables, oracle_lib, data, (112, 150, 32, 32), 64, 2, 27, mode)
    assert np.count_nonzero(ct) > 100
    _compare(gm, cm, "materials (depth 2)")
    _compare(gt, ct, "texels (depth 2)")


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_adjoint_matches_fp64_oracle_texture_shaders(ctx, kelemen_tables, oracle_lib, mode):
    """Triplanar diffuse shaders (each texel's gradient weighted by its blend weight) under
    normal maps: the ground, the sphere's diffuse lobe and the box."""
    from aurora_b200 import scenes
    data = scenes.shader_scene(128, 128, spp=64)
    gm, gt, cm, ct = _run(ctx, kelemen_tables, oracle_lib, data, (56, 72, 32, 32), 64, 3, 26, mode)
    assert np.count_nonzero(ct) > 100
    _compare(gm, cm, "materials (diffuse rgb, roughness)")
    _compare(gt, ct, "texels")


@pytest.mark.parametrize("mode", [0, 1], ids=["plain", "wavefront"])
def test_adjoint_matches_fp64_oracle_light_samples(ctx, kelemen_tables, oracle_lib, mode):
    """light_samples 3 on the differentiable workload: every camera sample after the first has
    three paths from its camera ray's first hit, each replayed with weight 1/3."""
    from aurora_b200 import scenes
    data = scenes.texture_scene()
    gm, gt, cm, ct = _run(ctx, kelemen_tables, oracle_lib, data, (112, 180, 32, 32), 16, 2, 28, mode,
                          light_samples=3)
    assert np.count_nonzero(ct) > 100
    _compare(gm, cm, "materials (light samples 3)")
    _compare(gt, ct, "texels (light samples 3)")


def test_adjoint_deeper_than_16_wavefront(ctx, kelemen_tables, oracle_lib):
    """max_depth 20 (glass boxes, roulette from the second bounce): the wavefront adjoint records
    hits in device memory and takes any depth; the megakernel refuses more than 16."""
    import aurora_b200 as ab
    from aurora_b200 import _abi, scenes
    glass = dict(type_=_abi.MAT_GLASS, specular=(1.0, 1.0, 1.0), diffuse=(0.95, 0.9, 0.85), reflectance=0.04,
                 ior=1.5)
    data = scenes.box_scene(128, 128, spp=32, max_depth=20, box_mat=glass, lift=0.01)
    data.render["min_depth"] = 1
    gm, gt, cm, ct = _run(ctx, kelemen_tables, oracle_lib, data, (40, 72, 32, 32), 32, 1, 29, 1)
    _compare(gm, cm, "materials (depth 20)")
    scene = ab.Scene(ctx, data)
    with pytest.raises(ab.AuroraError) as e:
        scene.adjoint(ab.render_opts(4, 20, 1, 1, mode=0), np.zeros((128, 128, 4), np.float32))
    assert e.value.status == _abi.ERR_UNSUPPORTED
    scene.close()

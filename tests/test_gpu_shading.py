"""BRDF values, pdfs, MIS weights, Kelemen lookups, camera and light sampling of the
device against the CPU restatement: within 1e-5 relative (criterion b)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def rand_dirs(r, n, hemi=None):
    d = r.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    if hemi is not None:
        s = np.sign(d @ hemi)
        d *= np.where(s == 0, 1, s)[:, None]
    return d


def close(gpu, cpu, rtol=RTOL, atol=1e-7, frac=0.0):
    """|gpu - cpu| <= atol + rtol |cpu|, allowing a fraction `frac` of records to differ
    (branch flips at the reference's thresholds when the last ulp differs)."""
    err = np.abs(gpu - cpu) > atol + rtol * np.abs(cpu)
    bad = np.any(err.reshape(err.shape[0], -1), axis=1)
    assert bad.mean() <= frac, (bad.sum(), np.nonzero(bad)[0][:5], gpu[bad][:3], cpu[bad][:3])


@pytest.fixture(scope="module")
def brdf_records():
    r = np.random.default_rng(101)
    n = 20000
    N = rand_dirs(r, n)
    V = rand_dirs(r, n, None)
    V = np.where((np.sum(V * N, 1) < 0.05)[:, None], V - 2 * np.sum(V * N, 1)[:, None] * N, V)
    L = rand_dirs(r, n)
    col = r.uniform(0.05, 0.95, (n, 3))
    rough = r.uniform(0.05, 0.95, n)
    lobe = r.integers(0, 2, n)
    ev = np.concatenate([lobe[:, None], col, rough[:, None], L, V, N], 1).astype(np.float32)
    sm = np.concatenate([lobe[:, None], col, rough[:, None], V, N, r.uniform(0, 1, (n, 2))], 1).astype(np.float32)
    return ev, sm


def test_brdf_eval_and_pdf(ctx, oracle_lib, brdf_records):
    ev, _ = brdf_records
    close(ctx.probe(1, ev), oracle_lib.probe(1, ev), frac=1e-3)
    close(ctx.probe(2, ev), oracle_lib.probe(2, ev), atol=1e-6, frac=1e-3)


def test_brdf_sample(ctx, oracle_lib, brdf_records):
    _, sm = brdf_records
    g, c = ctx.probe(0, sm), oracle_lib.probe(0, sm)
    close(g[:, :3], c[:, :3], atol=1e-5, frac=1e-3)     # directions
    close(g[:, 3:], c[:, 3:], atol=1e-6, frac=2e-3)     # pdf, colour


def test_power_heuristic_and_camera(ctx, oracle_lib):
    r = np.random.default_rng(7)
    ph = r.uniform(1e-3, 1e3, (5000, 2)).astype(np.float32)
    close(ctx.probe(5, ph), oracle_lib.probe(5, ph))
    cam = np.stack([np.full(5000, 0.36397), np.full(5000, 1920), np.full(5000, 1080), r.integers(0, 1920, 5000),
                    r.integers(0, 1080, 5000), r.uniform(0, 1, 5000), r.uniform(0, 1, 5000)], 1).astype(np.float32)
    close(ctx.probe(4, cam), oracle_lib.probe(4, cam), atol=1e-7)


def test_kelemen_lookup(ctx, oracle_lib, kelemen_tables):
    r = np.random.default_rng(9)
    rec = np.stack([r.integers(0, 21, 5000), r.uniform(0, 1, 5000), r.uniform(0, 1, 5000)], 1).astype(np.float32)
    close(ctx.probe(3, rec), oracle_lib.probe(3, rec, kelemen_tables))


def test_kelemen_tables_match_restatement(kelemen_tables, oracle_lib):
    """Device tables (250000 samples/entry) vs the CPU restatement of preCalcAlbedo with an
    independent random stream (20000 samples/entry): a coarse whole-table check."""
    for k in (0, 1, 10, 20):
        cpu = oracle_lib.kelemen_table(k / 20.0, 20000)
        gpu = kelemen_tables[k]
        assert np.all(np.isfinite(gpu))
        assert np.max(np.abs(gpu - cpu)) < 0.03 + 0.05 * np.max(np.abs(cpu)), (k, np.max(np.abs(gpu - cpu)))


def _precalc_albedo(reflectance, i, r, n, seed):
    """KelemenMaterial::preCalcAlbedo's estimator (kelemenMaterial.cpp:113-178) for one entry,
    restated in numpy with its own random stream: float32 arithmetic as the reference writes it
    (at grazing cos theta and roughness 1e-5 the sampled half vector rounds to the normal in
    float32, which the estimate depends on), each sample's value accumulated in float64.
    Returns the mean of n samples of F(h.l) max(0, l.n) / v.h and their variance."""
    f = np.float32
    g = np.random.default_rng(seed)
    r1, r2, r3 = ((g.integers(0, 1 << 24, n) / float(1 << 24)).astype(f) for _ in range(3))   # [0, 1) exactly
    rough = f(max(1e-5, r / 31.0))
    z = np.cos(np.arctan(rough * np.sqrt(-np.log(f(1) - r1))))
    rr = np.sqrt(np.maximum(f(0), f(1) - z * z))
    phi = f(np.pi) * f(2) * r2
    H = np.stack([rr * np.cos(phi), rr * np.sin(phi), z], 1)
    H = H / np.sqrt(np.sum(H * H, 1, keepdims=True))
    vz = f(max(1e-4, i / 63.0))
    rv = np.sqrt(np.maximum(f(0), f(1) - vz * vz))
    phi = r3 * f(2) * f(np.pi)
    V = np.stack([rv * np.cos(phi), rv * np.sin(phi), np.full(n, vz, f)], 1)
    V = V / np.sqrt(np.sum(V * V, 1, keepdims=True))
    H = np.where((np.sum(H * V, 1) < 0)[:, None], -H, H)
    vdoth = np.sum(V * H, 1)
    L = H * f(2) * vdoth[:, None] - V
    L = L / np.sqrt(np.sum(L * L, 1, keepdims=True))
    F = f(reflectance) + (f(1) - np.sum(H * L, 1)) ** f(5) * (f(1) - f(reflectance))
    ok = vdoth > 1e-6
    a = np.where(ok, F * np.maximum(f(0), L[:, 2]) / np.where(ok, vdoth, f(1)), f(0)).astype(np.float64)
    return a.mean(), a.var()


def test_kelemen_table_entries_within_monte_carlo_error(kelemen_tables):
    """Entries of three tables (reflectance 0, 0.5, 1) on a grid of cos theta and roughness
    against a numpy restatement with 400000 independent samples each. Both sides estimate
    the same expectation, so they differ by Monte Carlo noise alone: the bound is 5 standard
    errors of the difference (variance / 250000 + variance / 400000) plus the half-precision
    rounding of the stored table (2^-11 relative) and 1e-6."""
    n = 400_000
    worst = 0.0
    for k in (0, 10, 20):
        for i in (0, 1, 8, 21, 40, 63):
            for r in (0, 3, 9, 16, 31):
                mean, var = _precalc_albedo(k / 20.0, i, r, n, seed=1000 * k + 64 * i + r)
                se = np.sqrt(var / 250_000 + var / n)
                dev = float(kelemen_tables[k][i, r])
                bound = 5 * se + 2.0 ** -11 * abs(mean) + 1e-6
                worst = max(worst, abs(dev - mean) / bound)
                assert abs(dev - mean) <= bound, (k, i, r, dev, mean, se)
    print(f"\nKelemen entries: worst |device - restatement| / bound = {worst:.3f}")


def test_lights_and_materials(ctx, oracle_lib, kelemen_tables):
    import aurora_b200 as ab
    from aurora_b200 import scenes
    env = np.random.default_rng(14).uniform(0.1, 3.0, (16, 32, 3)).astype(np.float32)
    data = scenes.sphere_scene(64, 64, env=dict(color=(1, 1, 1), exposure=0.5, texture=env))   # lights: square, sphere, env
    scene = ab.Scene(ctx, data)
    osc = oracle_lib.OracleScene(data, kelemen_tables, use_bvh=False)
    r = np.random.default_rng(13)
    n = 8000
    P = r.uniform(-3, 3, (n, 3)) + scenes.sphere_center_camera(data)
    N = rand_dirs(r, n)
    li = r.integers(0, len(data.lights), n)
    ls = np.concatenate([li[:, None], P, r.uniform(0, 1, (n, 2)), N], 1).astype(np.float32)
    close(ctx.probe(6, ls, scene), osc.probe(6, ls), rtol=2e-5, atol=1e-5, frac=1e-3)
    vis = np.concatenate([li[:, None], P, N], 1).astype(np.float32)
    assert np.array_equal(ctx.probe(8, vis, scene), osc.probe(8, vis))
    D = rand_dirs(r, n)
    lp = np.concatenate([li[:, None], P, D, np.full((n, 1), 0.0005), np.full((n, 1), 1e7)], 1).astype(np.float32)
    g, c = ctx.probe(7, lp, scene), osc.probe(7, lp)
    close(g, c, rtol=2e-5, atol=1e-5, frac=1e-3)
    assert (c[:, 0] > 0).sum() > 10
    mats = np.concatenate([r.integers(0, len(data.materials), n)[:, None], rand_dirs(r, n), N,
                           r.uniform(0, 1, (n, 2)), r.integers(0, 2, n)[:, None], r.uniform(0, 1, n)[:, None]],
                          1).astype(np.float32)
    close(ctx.probe(9, mats, scene), osc.probe(9, mats), frac=1e-3)


def test_shade_points_texture_shaders_and_normal_maps(ctx, oracle_lib, kelemen_tables):
    """The hit's shading frame and Material::getBrdf (probe kind 10): interpolated normal,
    normal-map texture and constant normal map, triplanar colour and float shaders."""
    import aurora_b200 as ab
    from aurora_b200 import scenes
    from shade_points import hit_records
    data = scenes.shader_scene(32, 32)
    scene = ab.Scene(ctx, data)
    rec = hit_records(data, 20000, 43)
    rec[:, 11] = np.random.default_rng(44).uniform(0, 1, rec.shape[0])   # both Kelemen lobes
    close(ctx.probe(10, rec, scene), oracle_lib.OracleScene(data, kelemen_tables).probe(10, rec), frac=1e-3)
    scene.close()


def test_mirror_and_transmission_lobes(ctx, oracle_lib):
    """Glass lobes (SpecMirror, SpecTransmit): sampled directions, pdf 1, colour."""
    r = np.random.default_rng(31)
    n = 4000
    N = rand_dirs(r, n)
    V = rand_dirs(r, n)       # both sides of the surface: transmission enters or reflects totally
    lobe = np.where(r.uniform(size=n) < 0.5, 2, 4)
    ior = np.where(lobe == 4, r.uniform(1.1, 2.4, n), 0.0)
    rec = np.concatenate([lobe[:, None], r.uniform(0.1, 1, (n, 3)), ior[:, None], V, N, r.uniform(0, 1, (n, 2))],
                         1).astype(np.float32)
    close(ctx.probe(0, rec), oracle_lib.probe(0, rec), atol=2e-7)

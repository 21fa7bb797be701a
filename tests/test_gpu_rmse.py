"""RMSE against a 65536-spp reference accumulated in FP64 (the plain renderer's FP64 film):
the batched (wavefront) and plain renderers produce the same film, hence equal RMSE, and
both converge to the reference at the Monte Carlo rate (RMSE ~ spp^-1/2: the estimator
is unbiased with respect to the reference)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_equal_rmse_against_65536spp_fp64_reference(ctx):
    import aurora_b200 as ab
    from aurora_b200 import _abi, scenes
    data = scenes.box_scene(256, 256)
    scene = ab.Scene(ctx, data)
    ref = scene.render_f64(ab.render_opts(65536, 5, 5, 99)).film[..., :3]
    rmse = {}
    for mode, name in ((_abi.RENDER_PLAIN, "plain"), (_abi.RENDER_WAVEFRONT, "wavefront")):
        for spp in (16, 64):
            film = scene.render(ab.render_opts(spp, 5, 5, 1, mode=mode)).film[..., :3].astype(np.float64)
            rmse[(name, spp)] = float(np.sqrt(np.mean((film - ref) ** 2)))
    print("\nRMSE vs 65536-spp FP64 reference:", {f"{k[0]}@{k[1]}": round(v, 6) for k, v in rmse.items()})
    for spp in (16, 64):
        assert abs(rmse[("plain", spp)] - rmse[("wavefront", spp)]) <= 1e-6 * rmse[("plain", spp)]
    ratio = rmse[("plain", 16)] / rmse[("plain", 64)]
    assert 1.8 < ratio < 2.2, ratio
    scene.close()

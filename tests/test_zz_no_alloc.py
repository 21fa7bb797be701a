"""aur_render_fp64acc_noalloc — the renderer for callers that cannot allocate device
memory (hosts that own all GPU memory through their own allocator or budget).

It must reproduce the existing FP64-accumulating entry point (aur_render with
fp64_film=1) on consecutive calls, which share its static scratch array. This
file is collected last so that a failure here leaves every other test run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(scene, opts, film):
    from aurora_b200 import _abi
    st = _abi.RenderStats()
    status = _abi.lib().aur_render_fp64acc_noalloc(scene.handle, C.byref(opts), film.data_ptr(), C.byref(st))
    return status, st


def test_noalloc_matches_fp64_render_twice():
    import torch
    import aurora_b200 as ab
    from aurora_b200 import scenes, _abi
    ctx = ab.Context(0)
    for data, spp in ((scenes.box_scene(128, 96), 16), (scenes.sphere_scene(64, 64), 8)):
        scene = ab.Scene(ctx, data)
        r = data.render
        opts = ab.render_opts(spp, r["max_depth"], r["min_depth"], r["seed"], fp64_film=1)
        ref = scene.render(opts)
        film = torch.zeros((data.height, data.width, 4), dtype=torch.float32, device="cuda")
        for _ in range(2):                       # the second call reuses the static scratch
            film.fill_(-1.0)
            status, st = _noalloc(scene, opts, film)
            _abi.check(status, "aur_render_fp64acc_noalloc")
            got = film.cpu().numpy()
            np.testing.assert_allclose(got, ref.film, rtol=1e-6, atol=1e-7)
            assert st.paths == ref.stats["paths"]
            assert st.closest_rays == ref.stats["closest_rays"]
            assert st.shadow_rays == ref.stats["shadow_rays"]
        scene.close()
    ctx.close()


def test_noalloc_rejects_oversized_and_host_films():
    import torch
    import aurora_b200 as ab
    from aurora_b200 import scenes
    ctx = ab.Context(0)
    big = ab.Scene(ctx, scenes.box_scene(512, 512))
    opts = ab.render_opts(1, 5, 5, 1)
    film = torch.zeros((512, 512, 4), dtype=torch.float32, device="cuda")
    status, _ = _noalloc(big, opts, film)
    assert status == 1     # AUR_ERR_INVALID_ARG: beyond the 65536-pixel scratch
    small = ab.Scene(ctx, scenes.box_scene(32, 32))
    host = torch.zeros((32, 32, 4), dtype=torch.float32)
    status, _ = _noalloc(small, opts, host)
    assert status == 1     # the film must be device memory
    big.close()
    small.close()
    ctx.close()

"""aur_render_fp64acc_noalloc — the renderer for callers that cannot allocate device
memory (hosts that own all GPU memory through their own allocator or budget).

It must reproduce the existing FP64-accumulating entry point (aur_render with
fp64_film=1) on consecutive calls, which share its static scratch array, leave the
device's free memory unchanged, and agree with the CPU oracle. This file is
collected last so that a failure here leaves every other test run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(scene, opts, film):
    from aurora_b200 import _abi
    st = _abi.RenderStats()
    status = _abi.lib().aur_render_fp64acc_noalloc(scene.handle, C.byref(opts), film.data_ptr(), C.byref(st))
    return status, st


@pytest.mark.parametrize("light_samples", [1, 4])
def test_noalloc_matches_fp64_render_twice(light_samples):
    """Two calls in a row equal aur_render(fp64_film=1); light_samples 4 runs the multi-path
    FP64 instantiation. Around the second call the device's free memory does not move."""
    import torch
    import aurora_b200 as ab
    from aurora_b200 import scenes, _abi
    ctx = ab.Context(0)
    for data, spp in ((scenes.box_scene(128, 96), 16), (scenes.sphere_scene(64, 64), 8)):
        scene = ab.Scene(ctx, data)
        r = data.render
        opts = ab.render_opts(spp, r["max_depth"], r["min_depth"], r["seed"], fp64_film=1,
                              light_samples=light_samples)
        ref = scene.render(opts)
        film = torch.zeros((data.height, data.width, 4), dtype=torch.float32, device="cuda")
        for k in range(2):                       # the second call reuses the static scratch
            film.fill_(-1.0)
            torch.cuda.synchronize()
            free0, _ = torch.cuda.mem_get_info()
            status, st = _noalloc(scene, opts, film)
            _abi.check(status, "aur_render_fp64acc_noalloc")
            free1, _ = torch.cuda.mem_get_info()
            if k == 1:     # the first call may still see the driver size the kernel's local memory
                assert free1 == free0, (free0, free1)
            got = film.cpu().numpy()
            np.testing.assert_allclose(got, ref.film, rtol=1e-6, atol=1e-7)
            assert st.paths == ref.stats["paths"]
            assert st.closest_rays == ref.stats["closest_rays"]
            assert st.shadow_rays == ref.stats["shadow_rays"]
        scene.close()
    ctx.close()


def test_noalloc_matches_oracle(oracle_lib, kelemen_tables):
    """The box workload at 128x96, 16 spp: per-pixel means within 3 sigma of the CPU oracle."""
    import torch
    import aurora_b200 as ab
    from aurora_b200 import scenes, _abi
    ctx = ab.Context(0)
    data = scenes.box_scene(128, 96)
    r = data.render
    scene = ab.Scene(ctx, data)
    film = torch.zeros((96, 128, 4), dtype=torch.float32, device="cuda")
    status, st = _noalloc(scene, ab.render_opts(16, r["max_depth"], r["min_depth"], r["seed"], fp64_film=1), film)
    _abi.check(status, "aur_render_fp64acc_noalloc")
    mean, m2, counts = oracle_lib.OracleScene(data, kelemen_tables).render(16, r["max_depth"], r["min_depth"],
                                                                          r["seed"])
    sig = np.sqrt(m2 / 15 / 16)
    got = film.cpu().numpy().astype(np.float64)
    bad = np.abs(got[..., :3] - mean[..., :3]) > 3 * sig + 1e-4 * (1 + np.abs(mean[..., :3]))
    assert bad.any(-1).mean() <= 0.005
    assert st.paths == int(counts[2])
    scene.close()
    ctx.close()


def test_noalloc_rejects_bad_arguments():
    import torch
    import aurora_b200 as ab
    from aurora_b200 import scenes, _abi
    ctx = ab.Context(0)
    big = ab.Scene(ctx, scenes.box_scene(512, 512))
    opts = ab.render_opts(1, 5, 5, 1, fp64_film=1)
    film = torch.zeros((512, 512, 4), dtype=torch.float32, device="cuda")
    status, _ = _noalloc(big, opts, film)
    assert status == _abi.ERR_INVALID_ARG          # beyond the 65536-pixel scratch
    small = ab.Scene(ctx, scenes.box_scene(32, 32))
    for host in (torch.zeros((32, 32, 4), dtype=torch.float32),
                 torch.zeros((32, 32, 4), dtype=torch.float32).pin_memory()):
        status, _ = _noalloc(small, opts, host)
        assert status == _abi.ERR_INVALID_ARG      # the film must be device memory
    dev = torch.zeros((32, 32, 4), dtype=torch.float32, device="cuda")
    status, _ = _noalloc(small, ab.render_opts(1, 5, 5, 1, fp64_film=0), dev)
    assert status == _abi.ERR_UNSUPPORTED          # FP64 accumulation only
    status, _ = _noalloc(small, ab.render_opts(1, 5, 5, 1, fp64_film=1, count_work=1), dev)
    assert status == _abi.ERR_UNSUPPORTED          # no counting pass
    big.close()
    small.close()
    ctx.close()

"""Closest-hit and occlusion parity of the device BVH against the brute-force
FP32 Moller-Trumbore oracle (criterion: bit-exact hit ids, exact-t ties
excluded and counted)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sphere(ctx):
    from aurora_b200 import scenes
    import aurora_b200 as ab
    data = scenes.sphere_scene(64, 64)
    return data, ab.Bvh(ctx, data.verts, data.tri_vidx, data.tri_attr)


def _compare(gpu, cpu, ties):
    ok = ties <= 1
    mism = np.nonzero(ok & (gpu["prim"] != cpu["prim"]))[0]
    hit = ok & (cpu["prim"] >= 0)
    exact = (np.array_equal(gpu["t"][hit], cpu["t"][hit]) and np.array_equal(gpu["u"][hit], cpu["u"][hit])
             and np.array_equal(gpu["v"][hit], cpu["v"][hit]) and np.array_equal(gpu["attr"][hit], cpu["attr"][hit]))
    return mism, int((~ok).sum()), exact


def test_bvh_info(sphere):
    data, bvh = sphere
    info = bvh.info()
    assert 0 < info["depth"] < 64
    assert info["num_nodes"] >= data.ntri // 31
    lo, hi = np.array(info["bounds"][:3]), np.array(info["bounds"][3:])
    assert np.all(lo <= data.verts.min(0)) and np.all(hi >= data.verts.max(0))


@pytest.fixture(scope="module")
def hit_set(sphere, oracle_lib):
    """The 2^20-ray set (origins U[-3,3]^3 around the sphere, directions uniform, seed 3) and the
    brute-force scan's hits and exact-t tie counts for it."""
    from aurora_b200 import scenes
    data, _ = sphere
    n = int(os.environ.get("AURORA_HITID_RAYS", 1 << 20))
    rays = scenes.sphere_rays(n, seed=3, center=scenes.sphere_center_camera(data))
    cpu, ties = oracle_lib.trace_brute(data.verts, data.tri_vidx, data.tri_attr, rays)
    return rays, cpu, ties


def test_hit_ids_bit_exact_2pow20(sphere, hit_set):
    """2^20 rays against the 20804-triangle Kelemen-sphere scene: prim ids, t, u, v identical
    to the brute-force scan."""
    data, bvh = sphere
    rays, cpu, ties = hit_set
    n = rays.shape[0]
    gpu = bvh.trace_closest(rays)
    mism, nties, exact = _compare(gpu, cpu, ties)
    print(f"\nhit-id set: {n} rays, {int((cpu['prim'] >= 0).sum())} hits, {nties} exact-t ties excluded, "
          f"{len(mism)} mismatches")
    assert len(mism) == 0, mism[:10]
    assert exact
    assert int((cpu["prim"] >= 0).sum()) > n // 10


def test_occlusion_parity(sphere, oracle_lib):
    from aurora_b200 import scenes
    data, bvh = sphere
    rays = scenes.sphere_rays(1 << 16, seed=31, center=scenes.sphere_center_camera(data))
    rays[:, 7] = np.random.default_rng(32).uniform(0.1, 6.0, rays.shape[0]).astype(np.float32)
    rays[:, 3] = 0.0005
    gpu = bvh.trace_occluded(rays)
    cpu = oracle_lib.occluded_brute(data.verts, data.tri_vidx, rays)
    assert np.array_equal(gpu, cpu), int((gpu != cpu).sum())
    assert 0 < cpu.sum() < len(cpu)


def test_edge_cases(ctx, oracle_lib):
    import aurora_b200 as ab
    # one triangle; degenerate (zero-area) triangles; axis-aligned and grazing rays
    v = np.array([[0, 0, -2], [1, 0, -2], [0, 1, -2], [0, 0, -3], [0, 0, -3], [0, 0, -3], [2, 2, -4], [3, 2, -4],
                  [2, 2, -4]], np.float32)
    i = np.array([[0, 1, 2], [3, 4, 5], [6, 7, 8]], np.uint32)
    rays = np.array([[0.25, 0.25, 0, 0, 0, 0, -1, 1e30],
                     [0.0, 0.0, 0, 0, 0, 0, -1, 1e30],
                     [0.5, 0.0, -2, 0, 1, 0, 0, 1e30],        # in the triangle's plane
                     [0, 0, 0, 0, 0, 0, -1, 1e30],
                     [2.5, 2, 0, 0, 0, 0, -1, 1e30],
                     [5, 5, 5, 0, 1, 0, 0, 1e30]], np.float32)
    for tris in (i[:1], i):
        bvh = ab.Bvh(ctx, v, tris)
        gpu = bvh.trace_closest(rays)
        cpu, ties = oracle_lib.trace_brute(v, tris, None, rays)
        assert np.array_equal(gpu["prim"], cpu["prim"])
        assert np.array_equal(bvh.trace_occluded(rays), oracle_lib.occluded_brute(v, tris, rays))
    assert bvh.trace_closest(np.zeros((0, 8), np.float32)).shape == (0,)
    with pytest.raises(ab.AuroraError):
        ab.Bvh(ctx, v, np.array([[0, 1, 99]], np.uint32))


def test_device_pointers(sphere):
    """torch CUDA tensors go straight through the ABI (no staging) and give the same hits."""
    import torch
    from aurora_b200 import scenes, _abi
    from aurora_b200.core import HIT_DTYPE
    data, bvh = sphere
    rays = scenes.sphere_rays(4096, seed=5, center=scenes.sphere_center_camera(data))
    host = bvh.trace_closest(rays)
    dr = torch.from_numpy(rays).cuda()
    dh = torch.zeros(4096 * 5, dtype=torch.int32, device="cuda")
    _abi.check(_abi.lib().aur_trace_closest(bvh.handle, dr.data_ptr(), dh.data_ptr(), 4096), "trace")
    dev = dh.cpu().numpy().view(HIT_DTYPE)
    assert np.array_equal(dev["prim"], host["prim"]) and np.array_equal(dev["t"], host["t"])


def test_large_random_soup(ctx, oracle_lib):
    """A 200k-triangle random soup (many overlaps, deep tree) against the CPU BVH oracle,
    which itself is pinned to brute force in test_oracle."""
    import aurora_b200 as ab
    from aurora_b200 import scenes
    r = np.random.default_rng(21)
    n = 200_000
    c = r.uniform(-3, 3, (n, 1, 3))
    v = (c + r.normal(0, 0.05, (n, 3, 3))).reshape(-1, 3).astype(np.float32)
    i = np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)
    bvh = ab.Bvh(ctx, v, i)
    rays = scenes.sphere_rays(1 << 16, seed=22)
    gpu = bvh.trace_closest(rays)
    b = scenes.SceneBuilder(8, 8, 0.5)
    b.mesh(v, i, b.material(0, diffuse=(0.5, 0.5, 0.5)))
    data = b.build()
    cpu = oracle_lib.OracleScene(data).trace(rays)
    bad = np.nonzero(gpu["prim"] != cpu["prim"])[0]
    # differences are only allowed where two triangles give exactly the same t
    for k in bad[:50]:
        assert gpu["t"][k] == cpu["t"][k]
    assert len(bad) <= 5


ISECT_REC = np.dtype([("hit", "u1"), ("maxt", "<f4"), ("attr", "<i4"), ("prim", "<i4"), ("P", "<f4", 3),
                      ("N", "<f4", 3), ("st", "<f4", 2), ("bar", "<f4", 3)])
SHADE_REC = np.dtype([("P", "<f4", 3), ("Ng", "<f4", 3), ("Ns", "<f4", 3), ("st", "<f4", 2), ("id", "<i4")])


def test_gpu_accelerator_adapter_full_contract(sphere, hit_set, oracle_lib, tmp_path):
    """GpuAccelerator (the AccelerationStructure adapter, aurora_b200/adapters) driven by a C++
    program linked against libaurora_b200.so over the 2^20-ray set: the batched intersect gives
    the brute-force scan's triangle, attribute, t and barycentrics, and EmbreeAccelerator's
    post-process bit for bit (hitP, face-forwarded normalised hitN, st, barCoords, maxt shrunk
    to t; embreeAccelerator.cpp:49-90); the one-ray forms agree with the batched ones;
    intersectBinary is "some hit in [mint, maxt]"; getShadingTriangles returns the corners."""
    import subprocess
    from aurora_b200 import _abi, scenes
    data, _ = sphere
    rays, cpu, ties = hit_set
    n, nsingle = rays.shape[0], 512
    shade_ids = np.array([0, 1, data.ntri // 2, data.ntri - 1], np.int32)
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        f.write(np.array([data.verts.shape[0], data.ntri, n, nsingle, len(shade_ids), 1], np.uint32).tobytes())
        for a, t in ((data.verts, np.float32), (data.tri_vidx, np.uint32), (data.tri_attr, np.int32),
                     (data.corner_normals, np.float32), (data.corner_uvs, np.float32), (rays, np.float32),
                     (shade_ids, np.int32)):
            f.write(np.ascontiguousarray(a, t).tobytes())
    exe = os.path.join(os.path.dirname(_abi.LIB_PATH), "test_gpu_accelerator")
    res = subprocess.run([exe, str(inp), str(out)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr
    buf = open(out, "rb").read()
    k = 0
    batch = np.frombuffer(buf, ISECT_REC, n, k); k += n * ISECT_REC.itemsize
    single = np.frombuffer(buf, ISECT_REC, nsingle, k); k += nsingle * ISECT_REC.itemsize
    occ = np.frombuffer(buf, np.uint8, n, k); k += n
    occ1 = np.frombuffer(buf, np.uint8, nsingle, k); k += nsingle
    corners = np.frombuffer(buf, SHADE_REC, 3 * len(shade_ids), k); k += 3 * len(shade_ids) * SHADE_REC.itemsize
    assert k == len(buf)
    ok = ties <= 1
    hit = ok & (cpu["prim"] >= 0)
    assert np.array_equal(batch["prim"][ok], cpu["prim"][ok])
    assert np.array_equal(batch["attr"][hit], cpu["attr"][hit])
    assert np.array_equal(batch["hit"][ok].astype(bool), cpu["prim"][ok] >= 0)
    assert np.array_equal(batch["maxt"][hit], cpu["t"][hit])                    # ray->maxt = t
    assert np.array_equal(batch["maxt"][~(batch["hit"].astype(bool))], rays[~(batch["hit"].astype(bool)), 7])
    u, v = cpu["u"][hit], cpu["v"][hit]
    assert np.array_equal(batch["bar"][hit][:, 0], u) and np.array_equal(batch["bar"][hit][:, 1], v)
    assert np.array_equal(batch["bar"][hit][:, 2], (1.0 - u.astype(np.float64) - v).astype(np.float32))
    post = oracle_lib.OracleScene(data).isect_post(rays, cpu)
    assert np.array_equal(batch["P"][hit], post[hit, 0:3])
    assert np.array_equal(batch["N"][hit], post[hit, 3:6])
    assert np.array_equal(batch["st"][hit], post[hit, 6:8])
    np.testing.assert_allclose(np.linalg.norm(batch["N"][hit], axis=1), 1.0, atol=1e-6)
    assert np.all(np.sum(batch["N"][hit] * rays[hit, 4:7], axis=1) <= 1e-6)     # face-forwarded
    assert single.tobytes() == batch[:nsingle].tobytes()
    assert np.array_equal(occ.astype(bool), batch["hit"].astype(bool))
    assert np.array_equal(occ1, occ[:nsingle])
    for j, t in enumerate(shade_ids):
        c = corners[3 * j:3 * j + 3]
        assert np.all(c["id"] == t)
        assert np.array_equal(c["P"], data.verts[data.tri_vidx[t]])
        assert np.array_equal(c["Ng"], data.corner_normals[t].reshape(3, 3)) and np.array_equal(c["Ns"], c["Ng"])
        assert np.array_equal(c["st"], data.corner_uvs[t].reshape(3, 2))
    print(f"\nadapter: {n} rays, {int(hit.sum())} hits compared, {int((~ok).sum())} exact-t ties excluded")


def test_bvh_intersect_rejects_missing_shading(ctx):
    """aur_bvh_intersect needs the per-corner normals (aur_bvh_set_shading); a scene's BVH has them
    and refuses new ones."""
    import ctypes as C
    import aurora_b200 as ab
    from aurora_b200 import _abi, scenes
    v = np.array([[0, 0, -2], [1, 0, -2], [0, 1, -2]], np.float32)
    bvh = ab.Bvh(ctx, v, np.array([[0, 1, 2]], np.uint32))
    rays = np.array([[0.25, 0.25, 0, 0, 0, 0, -1, 1e30]], np.float32)
    out = (_abi.Isect * 1)()
    assert _abi.lib().aur_bvh_intersect(bvh.handle, rays.ctypes.data, C.addressof(out), 1) == _abi.ERR_INVALID_ARG
    n = np.tile(np.array([0, 0, 1], np.float32), 3)
    _abi.check(_abi.lib().aur_bvh_set_shading(bvh.handle, n.ctypes.data, None), "aur_bvh_set_shading")
    _abi.check(_abi.lib().aur_bvh_intersect(bvh.handle, rays.ctypes.data, C.addressof(out), 1), "aur_bvh_intersect")
    assert out[0].prim == 0 and out[0].t == 2.0 and rays[0, 7] == 2.0 and tuple(out[0].hitN) == (0.0, 0.0, 1.0)
    scene = ab.Scene(ctx, scenes.box_scene(8, 8))
    sb = scene.bvh()
    assert _abi.lib().aur_bvh_set_shading(sb.handle, n.ctypes.data, None) == _abi.ERR_INVALID_ARG
    scene.close()


def test_indices_out_of_range_are_refused(ctx):
    """Vertex indices (aur_bvh_build) and triangle attribute indices (aur_scene_create) are checked
    on the device after their upload, host and device inputs alike, before any kernel reads
    through them."""
    import copy
    import ctypes as C
    import torch
    import aurora_b200 as ab
    from aurora_b200 import _abi, scenes
    v = np.array([[0, 0, -2], [1, 0, -2], [0, 1, -2]], np.float32)
    host = np.array([[0, 1, 3]], np.uint32)
    dev = torch.tensor([[0, 1, 3]], dtype=torch.int32, device="cuda")
    for ptr in (host.ctypes.data, dev.data_ptr()):
        h = C.c_void_p()
        st = _abi.lib().aur_bvh_build(ctx.handle, v.ctypes.data, 3, ptr, None, 1, None, C.byref(h))
        assert st == _abi.ERR_INVALID_ARG and b"vertex index" in _abi.lib().aur_last_error()
    data = scenes.box_scene(16, 16)
    for bad in (-1, len(data.attr_material)):
        d = copy.copy(data)
        d.tri_attr = data.tri_attr.copy()
        d.tri_attr[5] = bad
        with pytest.raises(ab.AuroraError) as e:
            ab.Scene(ctx, d)
        assert e.value.status == _abi.ERR_INVALID_ARG and "attribute" in str(e.value)
    ok = ab.Scene(ctx, data)                     # the context stays usable
    assert ok.render(ab.render_opts(1, 5, 5, 1)).stats["paths"] == 256
    ok.close()

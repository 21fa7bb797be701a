"""Writes tests/golden/golden.npz: small input/output vectors of the CPU oracle that the
CPU tests pin (the oracle must reproduce them exactly) and the GPU tests compare the
device path against.

    python tests/golden/make_golden.py

Contents (all generated from seeded inputs):
  rng_in / rng_out            SplitMix64 draws (seed, pixel, sample, dim) -> u
  ray_in / hit_prim, hit_tuv  4096 rays of the sphere ray set (seed 3, around the icosphere)
                              against the sphere workload's triangles, brute force
  brdf_eval_in / _out         512 Lambert / Cook-Torrance eval records (probe kind 1)
  brdf_pdf_out                their pdfs (probe kind 2)
  brdf_sample_in / _out       512 sample records (probe kind 0)
  kelemen05                   the Kelemen albedo table for reflectance 0.5, 200 samples / entry
  box_mean, box_m2            box workload 16x16, 8 spp, depth 5: per-pixel mean (RGB, alpha)
                              and Welford sums
  box_dfilm, box_grad         a seeded dL/dfilm and the FP64 adjoint for it (materials x 4)
  delta_sample_in / _out      256 mirror / transmission lobe samples (probe kind 0, lobes 2 and 4)
  env_sample_in / _out        256 environment-map light samples of the sphere workload with a
                              16x32 seeded env map (probe kind 6, the env light is light 2)
  shade_point_in / _out       512 shading points of the texture-shader workload (probe kind 10:
                              normal maps, triplanar colour and float shaders)
  glass_mean, glass_m2        box workload 16x16 with glass boxes (lifted 0.01), 8 spp, depth 6
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def make():
    from aurora_b200 import scenes
    from oracle import oracle
    out = {}
    r = np.random.default_rng(2024)
    rng_in = np.stack([r.integers(0, 2**31, 64), r.integers(0, 2**24, 64), r.integers(0, 2**19, 64),
                       r.integers(0, 4096, 64)], 1).astype(np.uint32)
    out["rng_in"] = rng_in
    out["rng_out"] = np.array([oracle.rng_u01(*map(int, x)) for x in rng_in], np.float32)

    sphere = scenes.sphere_scene(64, 64)
    rays = scenes.sphere_rays(4096, seed=3, center=scenes.sphere_center_camera(sphere))
    hits, ties = oracle.trace_brute(sphere.verts, sphere.tri_vidx, sphere.tri_attr, rays)
    out["ray_in"] = rays
    out["hit_prim"] = hits["prim"].astype(np.int32)
    out["hit_tuv"] = np.stack([hits["t"], hits["u"], hits["v"]], 1).astype(np.float32)
    out["hit_ties"] = ties.astype(np.int32)

    n = 512
    N = r.normal(size=(n, 3)); N /= np.linalg.norm(N, axis=1, keepdims=True)
    V = r.normal(size=(n, 3)); V /= np.linalg.norm(V, axis=1, keepdims=True)
    V = np.where((np.sum(V * N, 1) < 0.05)[:, None], V - 2 * np.sum(V * N, 1)[:, None] * N, V)
    L = r.normal(size=(n, 3)); L /= np.linalg.norm(L, axis=1, keepdims=True)
    col = r.uniform(0.05, 0.95, (n, 3))
    rough = r.uniform(0.05, 0.95, n)
    lobe = r.integers(0, 2, n)
    ev = np.concatenate([lobe[:, None], col, rough[:, None], L, V, N], 1).astype(np.float32)
    sm = np.concatenate([lobe[:, None], col, rough[:, None], V, N, r.uniform(0, 1, (n, 2))], 1).astype(np.float32)
    out["brdf_eval_in"] = ev
    out["brdf_eval_out"] = oracle.probe(1, ev)
    out["brdf_pdf_out"] = oracle.probe(2, ev)
    out["brdf_sample_in"] = sm
    out["brdf_sample_out"] = oracle.probe(0, sm)

    out["kelemen05"] = oracle.kelemen_table(0.5, 200)

    box = scenes.box_scene(16, 16, spp=8)
    tables = np.zeros((21, 64, 32), np.float32)
    osc = oracle.OracleScene(box, tables)
    mean, m2, _ = osc.render(8, 5, 5, 1, threads=1)
    out["box_mean"], out["box_m2"] = mean, m2
    dfilm = np.random.default_rng(7).normal(size=(16, 16, 4)).astype(np.float32)
    dfilm[..., 3] = 0
    gm, _ = osc.adjoint(8, 5, 5, 1, dfilm, threads=1)
    out["box_dfilm"], out["box_grad"] = dfilm, gm

    from aurora_b200 import _abi
    m = 256
    Nd = r.normal(size=(m, 3)); Nd /= np.linalg.norm(Nd, axis=1, keepdims=True)
    Vd = r.normal(size=(m, 3)); Vd /= np.linalg.norm(Vd, axis=1, keepdims=True)
    dl = np.where(r.uniform(size=m) < 0.5, 2, 4)
    ior = np.where(dl == 4, r.uniform(1.1, 2.4, m), 0.0)
    ds = np.concatenate([dl[:, None], r.uniform(0.1, 1, (m, 3)), ior[:, None], Vd, Nd, r.uniform(0, 1, (m, 2))],
                        1).astype(np.float32)
    out["delta_sample_in"] = ds
    out["delta_sample_out"] = oracle.probe(0, ds)

    envmap = np.random.default_rng(14).uniform(0.1, 3.0, (16, 32, 3)).astype(np.float32)
    esc = scenes.sphere_scene(32, 32, env=dict(color=(1, 1, 1), exposure=0.5, texture=envmap))
    P = r.uniform(-3, 3, (m, 3))
    Ne = r.normal(size=(m, 3)); Ne /= np.linalg.norm(Ne, axis=1, keepdims=True)
    es = np.concatenate([np.full((m, 1), 2.0), P, r.uniform(0, 1, (m, 2)), Ne], 1).astype(np.float32)
    assert esc.lights[2].type == _abi.LIGHT_ENV
    out["env_sample_in"] = es
    out["env_sample_out"] = oracle.OracleScene(esc, tables).probe(6, es)

    sys.path.insert(0, os.path.dirname(HERE))
    from shade_points import hit_records
    ssc = scenes.shader_scene(32, 32, sphere_level=2)
    sp = hit_records(ssc, 512, 45)
    out["shade_point_in"] = sp
    out["shade_point_out"] = oracle.OracleScene(ssc, tables).probe(10, sp)

    glass = dict(type_=_abi.MAT_GLASS, specular=(1.0, 1.0, 1.0), diffuse=(0.95, 0.9, 0.85), reflectance=0.04,
                 ior=1.5)
    gbox = scenes.box_scene(16, 16, spp=8, max_depth=6, box_mat=glass, lift=0.01)
    gmean, gm2, _ = oracle.OracleScene(gbox, tables).render(8, 6, 6, 1, threads=1)
    out["glass_mean"], out["glass_m2"] = gmean, gm2
    return out


if __name__ == "__main__":
    path = os.path.join(HERE, "golden.npz")
    np.savez_compressed(path, **make())
    print("wrote", path, os.path.getsize(path), "bytes")

"""ctypes wrapper of the CPU oracle (oracle/liboracle.so). TEST INFRASTRUCTURE:
only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as
the checker; the product never imports it."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build() -> str:
    r = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building the oracle failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp, u32, i32 = C.c_void_p, C.c_uint32, C.c_int
        L.oracle_rng_u01.restype = C.c_float
        L.oracle_rng_u01.argtypes = [u32, u32, u32, u32]
        L.oracle_trace_brute.argtypes = [vp, vp, vp, u32, vp, u32, vp, vp, i32]
        L.oracle_occluded_brute.argtypes = [vp, vp, u32, vp, u32, vp, i32]
        L.oracle_scene_create.restype = vp
        L.oracle_scene_create.argtypes = [vp, vp, i32, i32]
        L.oracle_scene_destroy.argtypes = [vp]
        L.oracle_scene_bvh_nodes.argtypes = [vp]
        L.oracle_trace.argtypes = [vp, vp, u32, vp, i32]
        L.oracle_isect_post.argtypes = [vp, vp, vp, u32, vp]
        L.oracle_render.argtypes = [vp, i32, i32, i32, i32, u32, i32, i32, i32, i32, i32, vp, vp, vp, i32]
        L.oracle_kelemen_table.argtypes = [C.c_float, i32, u32, vp, i32]
        L.oracle_shading_probe.argtypes = [vp, i32, vp, u32, vp, vp]
        L.oracle_adjoint.argtypes = [vp, i32, i32, i32, i32, u32, i32, i32, i32, i32, i32, vp, vp, i32]
        _lib = L
    return _lib


HIT_DTYPE = np.dtype([("t", "<f4"), ("u", "<f4"), ("v", "<f4"), ("prim", "<i4"), ("attr", "<i4")])
PROBE_OUT = [7, 3, 1, 1, 3, 1, 8, 2, 1, 5, 11]


def rng_u01(seed, pixel, sample, dim) -> float:
    return lib().oracle_rng_u01(seed, pixel, sample, dim)


def trace_brute(verts, idx, attr, rays, threads=0):
    verts = np.ascontiguousarray(verts, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32)
    attr = None if attr is None else np.ascontiguousarray(attr, np.int32)
    rays = np.ascontiguousarray(rays, np.float32)
    hits = np.zeros(rays.shape[0], HIT_DTYPE)
    ties = np.zeros(rays.shape[0], np.int32)
    lib().oracle_trace_brute(verts.ctypes.data, idx.ctypes.data, None if attr is None else attr.ctypes.data,
                             idx.shape[0], rays.ctypes.data, rays.shape[0], hits.ctypes.data, ties.ctypes.data,
                             threads)
    return hits, ties


def occluded_brute(verts, idx, rays, threads=0):
    verts = np.ascontiguousarray(verts, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32)
    rays = np.ascontiguousarray(rays, np.float32)
    occ = np.zeros(rays.shape[0], np.uint8)
    lib().oracle_occluded_brute(verts.ctypes.data, idx.ctypes.data, idx.shape[0], rays.ctypes.data, rays.shape[0],
                                occ.ctypes.data, threads)
    return occ


def kelemen_table(reflectance, samples, seed=77, threads=0):
    out = np.zeros((64, 32), np.float32)
    lib().oracle_kelemen_table(C.c_float(reflectance), samples, seed, out.ctypes.data, threads)
    return out


class OracleScene:
    """The CPU restatement of a flattened scene (brute force or binned-SAH BVH)."""

    def __init__(self, data, albedo_tables=None, use_bvh=True, max_leaf=4):
        self.data = data
        self._desc = data.desc()
        self.tables = np.ascontiguousarray(albedo_tables if albedo_tables is not None
                                           else np.zeros((21, 64, 32), np.float32), np.float32)
        self.h = lib().oracle_scene_create(C.addressof(self._desc), self.tables.ctypes.data, 1 if use_bvh else 0,
                                           max_leaf)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_scene_destroy(self.h)
            self.h = None

    def trace(self, rays, threads=0):
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros(rays.shape[0], HIT_DTYPE)
        lib().oracle_trace(self.h, rays.ctypes.data, rays.shape[0], hits.ctypes.data, threads)
        return hits

    def isect_post(self, rays, hits):
        """EmbreeAccelerator::intersect's post-process of `hits` (HIT_DTYPE): (n, 8) float32 rows of
        hitP xyz, hitN xyz, st (zeros for misses)."""
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.ascontiguousarray(hits, HIT_DTYPE)
        out = np.zeros((rays.shape[0], 8), np.float32)
        lib().oracle_isect_post(self.h, rays.ctypes.data, hits.ctypes.data, rays.shape[0], out.ctypes.data)
        return out

    def render(self, spp, max_depth, min_depth, seed, crop=None, sample_offset=0, threads=0, want_m2=True,
               light_samples=1):
        """Per-pixel mean (RGB, alpha) of spp passes over the crop, Welford sums of squares of
        the pass values, and counts (closest rays, shadow rays, paths). light_samples > 1:
        passes after the first trace that many paths from the camera ray's first hit."""
        W, H = self.data.width, self.data.height
        x0, y0, w, h = crop if crop is not None else (0, 0, W, H)
        mean = np.zeros((h, w, 4), np.float64)
        m2 = np.zeros((h, w, 3), np.float64) if want_m2 else None
        counts = np.zeros(3, np.uint64)
        lib().oracle_render(self.h, spp, sample_offset, max_depth, min_depth, seed, threads, x0, y0, w, h,
                            mean.ctypes.data, None if m2 is None else m2.ctypes.data, counts.ctypes.data,
                            int(light_samples))
        return mean, m2, counts

    def adjoint(self, spp, max_depth, min_depth, seed, dfilm, crop=None, sample_offset=0, threads=0, light_samples=1):
        """FP64 gradient of <dfilm, image> w.r.t. (per material: diffuse rgb, roughness) and the
        texels, over the crop's pixels. Returns (grad_mat [nmat, 4], grad_tex [ntexel floats])."""
        W, H = self.data.width, self.data.height
        x0, y0, w, h = crop if crop is not None else (0, 0, W, H)
        dfilm = np.ascontiguousarray(dfilm, np.float32).reshape(H * W * 4)
        nmat = len(self.data.materials)
        ntex = int(self.data.texels().size)
        grad = np.zeros(4 * nmat + ntex, np.float64)
        lib().oracle_adjoint(self.h, spp, sample_offset, max_depth, min_depth, seed, threads, x0, y0, w, h,
                             dfilm.ctypes.data, grad.ctypes.data, int(light_samples))
        return grad[:4 * nmat].reshape(nmat, 4), grad[4 * nmat:]

    def probe(self, kind, records):
        records = np.ascontiguousarray(records, np.float32)
        out = np.zeros((records.shape[0], PROBE_OUT[kind]), np.float32)
        rc = lib().oracle_shading_probe(self.h, kind, records.ctypes.data, records.shape[0], out.ctypes.data,
                                        self.tables.ctypes.data)
        assert rc == 0, rc
        return out


def probe(kind, records, tables=None):
    """Scene-free probes (kinds 0-5)."""
    records = np.ascontiguousarray(records, np.float32)
    out = np.zeros((records.shape[0], PROBE_OUT[kind]), np.float32)
    t = None if tables is None else np.ascontiguousarray(tables, np.float32)
    rc = lib().oracle_shading_probe(None, kind, records.ctypes.data, records.shape[0], out.ctypes.data,
                                    None if t is None else t.ctypes.data)
    assert rc == 0, rc
    return out

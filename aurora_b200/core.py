"""Python handles over the C ABI: contexts, BVHs, scenes and the render calls.

Arrays are numpy (host) or anything exposing ``data_ptr()`` (torch CUDA
tensors); the library accepts both host and device pointers.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import check, lib


def _ptr(a) -> int:
    if a is None:
        return 0
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


class Context:
    """aur_ctx: one CUDA device and stream."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().aur_ctx_create(device, C.byref(h)), "aur_ctx_create")
        self.handle = h
        self.device = device
        self._children = weakref.WeakSet()

    def close(self):
        if self.handle:
            for child in list(self._children):     # scenes and BVHs die before their context
                child.close()
            check(lib().aur_ctx_destroy(self.handle), "aur_ctx_destroy")
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        check(lib().aur_ctx_synchronize(self.handle), "aur_ctx_synchronize")

    def kelemen_table(self, reflectance: float) -> np.ndarray:
        out = np.zeros((64, 32), np.float32)
        check(lib().aur_kelemen_table(self.handle, C.c_float(reflectance), _ptr(out)), "aur_kelemen_table")
        return out

    def read_bandwidth(self, nbytes: int, reps: int) -> float:
        """GB/s of `reps` reads of an `nbytes` device buffer (aur_measure_read_bandwidth)."""
        out = C.c_double()
        check(lib().aur_measure_read_bandwidth(self.handle, int(nbytes), int(reps), C.byref(out)),
              "aur_measure_read_bandwidth")
        return out.value

    def probe(self, kind: int, records: np.ndarray, scene: "Scene | None" = None) -> np.ndarray:
        records = np.ascontiguousarray(records, np.float32)
        n = records.shape[0]
        out_w = [7, 3, 1, 1, 3, 1, 8, 2, 1, 5, 11][kind]
        out = np.zeros((n, out_w), np.float32)
        check(lib().aur_shading_probe(self.handle, scene.handle if scene else None, kind, _ptr(records), n,
                                      _ptr(out)), "aur_shading_probe")
        return out


def bvh_opts(max_leaf=0, cost_traverse=0.0, cost_intersect=0.0, ploc_radius=0) -> _abi.BvhOpts:
    return _abi.BvhOpts(max_leaf, cost_traverse, cost_intersect, ploc_radius)


HIT_DTYPE = np.dtype([("t", "<f4"), ("u", "<f4"), ("v", "<f4"), ("prim", "<i4"), ("attr", "<i4")])
# aur_isect: EmbreeAccelerator::intersect's full record
ISECT_DTYPE = np.dtype([("t", "<f4"), ("u", "<f4"), ("v", "<f4"), ("prim", "<i4"), ("attr", "<i4"),
                        ("hitP", "<f4", 3), ("hitN", "<f4", 3), ("st", "<f4", 2), ("bar", "<f4", 3)])


class Bvh:
    """aur_bvh: device BVH over a triangle soup (EmbreeAccelerator replacement)."""

    def __init__(self, ctx: Context, verts, tri_vidx, tri_attr=None, opts: _abi.BvhOpts | None = None,
                 _borrowed=None):
        self.ctx = ctx
        self.owned = _borrowed is None
        if _borrowed is not None:
            self.handle = _borrowed
            return
        verts = np.ascontiguousarray(verts, np.float32)
        tri_vidx = np.ascontiguousarray(tri_vidx, np.uint32)
        attr = None if tri_attr is None else np.ascontiguousarray(tri_attr, np.int32)
        h = C.c_void_p()
        check(lib().aur_bvh_build(ctx.handle, _ptr(verts), verts.shape[0], _ptr(tri_vidx), _ptr(attr),
                                  tri_vidx.shape[0], C.byref(opts) if opts else None, C.byref(h)), "aur_bvh_build")
        self.handle = h
        ctx._children.add(self)

    def close(self):
        if self.owned and self.handle:
            lib().aur_bvh_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        n = C.c_uint32()
        d = C.c_uint32()
        b = (C.c_float * 6)()
        check(lib().aur_bvh_info(self.handle, C.byref(n), C.byref(d), b), "aur_bvh_info")
        return {"num_nodes": n.value, "depth": d.value, "bounds": list(b)}

    def trace_closest(self, rays: np.ndarray) -> np.ndarray:
        """rays: (n, 8) float32 = org xyz, mint, dir xyz, maxt. Returns HIT_DTYPE records."""
        rays = np.ascontiguousarray(rays, np.float32)
        hits = np.zeros(rays.shape[0], HIT_DTYPE)
        check(lib().aur_trace_closest(self.handle, _ptr(rays), _ptr(hits), rays.shape[0]), "aur_trace_closest")
        return hits

    def trace_occluded(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32)
        occ = np.zeros(rays.shape[0], np.uint8)
        check(lib().aur_trace_occluded(self.handle, _ptr(rays), _ptr(occ), rays.shape[0]), "aur_trace_occluded")
        return occ

    def set_shading(self, corner_normals, corner_uvs=None):
        """Per-corner normals (ntri, 9) and uvs (ntri, 6) that intersect() interpolates."""
        n = np.ascontiguousarray(corner_normals, np.float32)
        uv = None if corner_uvs is None else np.ascontiguousarray(corner_uvs, np.float32)
        check(lib().aur_bvh_set_shading(self.handle, _ptr(n), _ptr(uv)), "aur_bvh_set_shading")

    def intersect(self, rays: np.ndarray):
        """EmbreeAccelerator::intersect for (n, 8) rays: (ISECT_DTYPE records, the rays with maxt
        shrunk to t where they hit)."""
        rays = np.array(rays, np.float32, copy=True, order="C")
        out = np.zeros(rays.shape[0], ISECT_DTYPE)
        check(lib().aur_bvh_intersect(self.handle, _ptr(rays), _ptr(out), rays.shape[0]), "aur_bvh_intersect")
        return out, rays


@dataclass
class RenderResult:
    film: np.ndarray          # (H, W, 4) float32 (or float64 for render_f64)
    stats: dict


def render_opts(spp, max_depth, min_depth, seed, mode=_abi.RENDER_PLAIN, sample_offset=0, fp64_film=0,
                wf_pool=0, wf_block=0, wf_sort=-1, count_work=0, light_samples=0) -> _abi.RenderOpts:
    return _abi.RenderOpts(spp, sample_offset, max_depth, min_depth, seed, mode, fp64_film, wf_pool, wf_block,
                           wf_sort, count_work, light_samples)


def _stats(s: _abi.RenderStats) -> dict:
    return {"camera_rays": s.camera_rays, "closest_rays": s.closest_rays, "shadow_rays": s.shadow_rays,
            "paths": s.paths, "node_visits": s.node_visits, "tri_tests": s.tri_tests, "launches": s.launches,
            "kernel_ms": s.kernel_ms, "shadow_node_visits": s.shadow_node_visits,
            "shadow_tri_tests": s.shadow_tri_tests,
            "stage_ms": dict(zip(("regen", "extend", "sort", "shade", "shadow"), list(s.stage_ms))),
            "wf_config": {"pool": s.wf_pool, "block": s.wf_block, "sort": s.wf_sort}, "node_bytes": s.node_bytes}


class Scene:
    """aur_scene: flattened camera-space scene resident on the device."""

    def __init__(self, ctx: Context, data=None, bvh: _abi.BvhOpts | None = None, json_path: str | None = None):
        self.ctx = ctx
        h = C.c_void_p()
        self.file_opts = None
        if json_path is not None:
            o = _abi.RenderOpts()
            check(lib().aur_scene_load_json(ctx.handle, json_path.encode(), C.byref(bvh) if bvh else None, C.byref(h),
                                            C.byref(o)), "aur_scene_load_json")
            self.file_opts = o    # render options from the file's "options"
        else:
            desc = data.desc()
            check(lib().aur_scene_create(ctx.handle, C.byref(desc), C.byref(bvh) if bvh else None, C.byref(h)),
                  "aur_scene_create")
        self.handle = h
        ctx._children.add(self)
        w, hh, ntri, nmat, ntex = C.c_int32(), C.c_int32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib().aur_scene_info(h, C.byref(w), C.byref(hh), C.byref(ntri), C.byref(nmat), C.byref(ntex)),
              "aur_scene_info")
        self.width, self.height, self.ntri, self.nmat, self.ntexel = w.value, hh.value, ntri.value, nmat.value, ntex.value

    def close(self):
        if self.handle:
            lib().aur_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bvh(self) -> Bvh:
        h = C.c_void_p()
        check(lib().aur_scene_bvh(self.handle, C.byref(h)), "aur_scene_bvh")
        return Bvh(self.ctx, None, None, _borrowed=h)

    def render(self, opts: _abi.RenderOpts, out=None) -> RenderResult:
        film = out if out is not None else np.zeros((self.height, self.width, 4), np.float32)
        s = _abi.RenderStats()
        check(lib().aur_render(self.handle, C.byref(opts), _ptr(film), C.byref(s)), "aur_render")
        return RenderResult(film, _stats(s))

    def render_progressive(self, opts: _abi.RenderOpts, pass_spp: int, on_pass=None, out=None) -> RenderResult:
        """Renders opts.spp samples in passes of pass_spp; on_pass(film, samples_done) gets a
        copy of the running mean (H, W, 4) after every pass and may return True to stop."""
        film = out if out is not None else np.zeros((self.height, self.width, 4), np.float32)
        s = _abi.RenderStats()
        h, w = self.height, self.width
        errors = []

        def trampoline(_user, ptr, done):
            try:
                img = np.ctypeslib.as_array(ptr, shape=(h * w * 4,)).reshape(h, w, 4).copy()
                return 1 if (on_pass(img, int(done)) if on_pass else False) else 0
            except Exception as ex:                       # stop the render, re-raise below
                errors.append(ex)
                return 1
        cb = _abi.PASS_FN(trampoline)
        check(lib().aur_render_progressive(self.handle, C.byref(opts), int(pass_spp), C.cast(cb, C.c_void_p), None,
                                           _ptr(film), C.byref(s)), "aur_render_progressive")
        if errors:
            raise errors[0]
        return RenderResult(film, _stats(s))

    def render_f64(self, opts: _abi.RenderOpts) -> RenderResult:
        film = np.zeros((self.height, self.width, 4), np.float64)
        s = _abi.RenderStats()
        check(lib().aur_render_f64(self.handle, C.byref(opts), _ptr(film), C.byref(s)), "aur_render_f64")
        return RenderResult(film, _stats(s))

    def set_params(self, mat_params=None, texels=None):
        mp = None if mat_params is None else (mat_params if hasattr(mat_params, "data_ptr")
                                              else np.ascontiguousarray(mat_params, np.float32))
        tx = None if texels is None else (texels if hasattr(texels, "data_ptr")
                                          else np.ascontiguousarray(texels, np.float32))
        check(lib().aur_scene_set_params(self.handle, _ptr(mp), _ptr(tx)), "aur_scene_set_params")

    def get_params(self):
        mp = np.zeros((self.nmat, 4), np.float32)
        tx = np.zeros(self.ntexel, np.float32)
        check(lib().aur_scene_get_params(self.handle, _ptr(mp), _ptr(tx) if self.ntexel else None),
              "aur_scene_get_params")
        return mp, tx

    def adjoint(self, opts: _abi.RenderOpts, dloss_dfilm, grad_mat=None, grad_tex=None):
        gm = grad_mat if grad_mat is not None else np.zeros((self.nmat, 4), np.float32)
        gt = grad_tex if grad_tex is not None else np.zeros(max(self.ntexel, 1), np.float32)
        d = dloss_dfilm if hasattr(dloss_dfilm, "data_ptr") else np.ascontiguousarray(dloss_dfilm, np.float32)
        s = _abi.RenderStats()
        check(lib().aur_render_adjoint(self.handle, C.byref(opts), _ptr(d), _ptr(gm), _ptr(gt), C.byref(s)),
              "aur_render_adjoint")
        return gm, gt, _stats(s)


def write_film(path: str, film, fmt: int = _abi.FILM_EXR_HALF) -> None:
    """Writes an (H, W, 4) float32 film (numpy or CUDA tensor) as OpenEXR (half or float
    RGBA, uncompressed) or PFM (RGB float)."""
    if hasattr(film, "data_ptr"):
        h, w = int(film.shape[0]), int(film.shape[1])
        f = film.contiguous()
    else:
        f = np.ascontiguousarray(film, np.float32)
        h, w = f.shape[:2]
    check(lib().aur_film_write(path.encode(), _ptr(f), w, h, fmt), "aur_film_write")


def render_batch(scenes: list[Scene], opts: list[_abi.RenderOpts], films=None):
    n = len(scenes)
    if films is None:
        films = [np.zeros((s.height, s.width, 4), np.float32) for s in scenes]
    hs = (C.c_void_p * n)(*[s.handle.value for s in scenes])
    os_ = (_abi.RenderOpts * n)(*opts)
    fs = (C.c_void_p * n)(*[_ptr(f) for f in films])
    st = _abi.RenderStats()
    check(lib().aur_render_batch(hs, os_, n, fs, C.byref(st)), "aur_render_batch")
    return films, _stats(st)

#!/usr/bin/env python
"""Path samples/s of the Aurora path-tracing core on the large terrain workload
(1920x1080, 64 spp, depth 8, roulette from the third bounce, ~3.4M triangles).

One step = one full frame (W*H*spp camera paths) rendered through the C ABI.
`value` is device-timed (CUDA events on the library's stream, inputs resident);
`e2e` runs the public API from host arrays to a host image every step
(scene upload + device BVH build + render + film download). Prints ONE JSON line
on rank 0. `--impl reference` times the CPU restatement of the reference path
(oracle/) on all host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "path samples/s at 1080p d8 (batched vs plain GPU) + adjoint/forward time ratio"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--small", action="store_true", help="reduced workload (smoke runs only)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--mode", default="auto", choices=["auto", "plain", "wavefront"])
    p.add_argument("--profile", action="store_true",
                   help="render two 1-spp frames of the workload with a fixed wavefront configuration "
                        "(pool 2^20, block 128, sort on) and exit: the small case for ncu captures")
    p.add_argument("--profile-adjoint", action="store_true",
                   help="one wavefront path-replay adjoint of the differentiable workload at 64 spp (pool "
                        "2^20, block 128, sort on) and exit: the small case for ncu captures of the adjoint")
    return p.parse_args()


def workload(small: bool):
    from aurora_b200 import scenes
    if small:
        return scenes.terrain_scene(480, 270, spp=8, grid=257, spheres=64, sphere_level=3)
    return scenes.terrain_scene()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().strip().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1])); mx = max(mx, float(r[2]))
                for k, name in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(name)
            except Exception:
                pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def render_opts_for(data, mode, rank=0, count_work=0, spp=None):
    """Options of one step on `rank`: the full frame with the rank's own sample range
    [rank * spp, (rank + 1) * spp) (weak scaling, no data-path collective)."""
    import aurora_b200 as ab
    from aurora_b200.shard import sample_range
    r = data.render
    s = spp or r["spp"]
    first, count = sample_range(rank, rank + 1, s, "weak")
    return ab.render_opts(count, r["max_depth"], r["min_depth"], r["seed"], mode=mode, sample_offset=first,
                          count_work=count_work)


def spread_rows(H, rows, offset=0):
    """`rows` full-width rows spread evenly over the frame (so that sky, terrain and spheres
    enter the sample in the frame's proportions), shifted by `offset` rows."""
    stride = H / rows
    return sorted({(int(j * stride) + offset) % H for j in range(rows)})


def render_rows(osc, data, ys, cores, keep=False):
    """Renders rows `ys` of the workload on the CPU; returns the seconds taken (and, with
    keep, each row's per-pixel mean and Welford sums of squares)."""
    r = data.render
    out = []
    t0 = time.perf_counter()
    for y in ys:
        mean, m2, _ = osc.render(r["spp"], r["max_depth"], r["min_depth"], r["seed"], crop=(0, y, data.width, 1),
                                 threads=cores, want_m2=keep)
        if keep:
            out.append((y, mean, m2))
    dt = time.perf_counter() - t0
    return (dt, out) if keep else dt


# The CPU sample, the same for the cpu_baseline leg and the reference arm: 216 full-width
# rows (a fifth of the 1080) spread evenly over the frame, so that sky, terrain and spheres
# enter it in the frame's proportions; both warm up on the same 8 rows first.
CPU_ROWS, CPU_ROW_OFFSET = 216, 7


def cpu_sample_rows(H):
    return spread_rows(H, min(H, CPU_ROWS), CPU_ROW_OFFSET)


def cpu_warmup(osc, data, cores):
    render_rows(osc, data, spread_rows(data.height, 8, data.height // 16), cores)


def cpu_baseline(data, tables):
    """CPU restatement (oracle, all host threads) on the fixed row sample at the workload's spp.
    Returns (paths/s, sample description, cores, build seconds, rows [(y, mean, m2)])."""
    from oracle import oracle
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    osc = oracle.OracleScene(data, tables, use_bvh=True)
    build_s = time.perf_counter() - t0
    r = data.render
    W, H = data.width, data.height
    ys = cpu_sample_rows(H)
    cpu_warmup(osc, data, cores)
    dt, rows = render_rows(osc, data, ys, cores, keep=True)
    paths = W * len(ys) * r["spp"]
    return (paths / dt, f"{W}x{len(ys)} fixed rows spread over the frame x {r['spp']} spp ({paths} paths, "
            f"{dt:.1f} s)", cores, build_s, rows)


def row_parity(film, rows, spp):
    """Fraction of the sampled pixels whose device mean lies beyond 3 sigma of the oracle's
    (per channel, the oracle's Welford variance; a 1e-4 relative floor)."""
    bad = n = 0
    for y, mean, m2 in rows:
        g = film[y:y + 1, :, :3].astype(np.float64)
        sig = np.sqrt(m2 / max(spp - 1, 1) / spp)
        d = np.abs(g - mean[..., :3])
        bad += int((d > 3 * sig + 1e-4 * (1 + np.abs(mean[..., :3]))).any(-1).sum())
        n += g.shape[1]
    return bad / max(n, 1), n


def adjoint_ratio(ab, _abi, torch, ctx, stream, steps=2, warmup=1):
    """Device time of the path-replay adjoint over the device time of the forward render on
    the differentiable workload (256x256, 256 spp, depth 6, 64x64 RGB texture, 16 materials).
    dL/dfilm is a resident device tensor; the parameter gradients come back to host arrays."""
    from aurora_b200 import scenes
    data = scenes.texture_scene()
    sc = ab.Scene(ctx, data)
    H, W = data.height, data.width
    spp, depth = data.render["spp"], data.render["max_depth"]
    film = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
    g = torch.Generator(device="cpu").manual_seed(8)
    dfilm = torch.randn((H, W, 4), generator=g).to("cuda")
    gm = np.zeros((sc.nmat, 4), np.float32)
    gt = np.zeros(max(sc.ntexel, 1), np.float32)

    def dev_ms(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def fwd(mode):
        return lambda: sc.render(ab.render_opts(spp, depth, depth, data.render["seed"], mode=mode), out=film)

    f_wf = dev_ms(fwd(_abi.RENDER_WAVEFRONT))
    f_plain = dev_ms(fwd(_abi.RENDER_PLAIN))
    def adj(mode):
        return lambda: sc.adjoint(ab.render_opts(spp, depth, depth, data.render["seed"], mode=mode), dfilm, gm, gt)

    a_wf = dev_ms(adj(_abi.RENDER_WAVEFRONT))
    st = sc.adjoint(ab.render_opts(spp, depth, depth, data.render["seed"], mode=_abi.RENDER_WAVEFRONT), dfilm, gm,
                    gt)[2]
    split = {"record_ms": st["stage_ms"]["regen"], "replay_ms": st["stage_ms"]["extend"],
             "wavefront_config": st["wf_config"]}
    a_plain = dev_ms(adj(_abi.RENDER_PLAIN))
    sc.close()
    return {"workload": f"texture {data.ntri} tris {W}x{H} {spp}spp depth {depth}, 16 materials + 64x64x3 texels",
            "forward_ms": f_wf, "adjoint_ms": a_wf, "ratio": a_wf / f_wf,
            "forward_plain_ms": f_plain, "adjoint_plain_ms": a_plain, "ratio_plain": a_plain / f_plain,
            "adjoint_split": split,
            "note": "ratio: wavefront adjoint (record pass on the wavefront engine + replay kernel) over the "
                    "wavefront forward (the autograd pair); ratio_plain: megakernel adjoint over the plain forward"}


def batch_timing(ab, _abi, torch, ctx, stream, steps=3):
    """The 64-scene batched workload: box scenes (seed 6+i) of resolution 128^2..512^2, 4/16/64
    spp and depth 3/5/8 in one wavefront launch (autotuned once, untimed), films resident on
    the device. Device time per launch (CUDA events, mean of `steps`) and path samples/s."""
    from aurora_b200 import scenes
    datas = scenes.batch_scenes(64)
    objs = [ab.Scene(ctx, d) for d in datas]
    opts = [ab.render_opts(d.render["spp"], d.render["max_depth"], d.render["min_depth"], d.render["seed"],
                           mode=_abi.RENDER_WAVEFRONT) for d in datas]
    films = [torch.empty((d.height, d.width, 4), dtype=torch.float32, device="cuda") for d in datas]
    _, st = ab.render_batch(objs, opts, films)                  # autotune + warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        _, st = ab.render_batch(objs, opts, films)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    for o in objs:
        o.close()
    paths = sum(d.width * d.height * d.render["spp"] for d in datas)
    return {"workload": "64 box scenes (seed 6+i), 128^2..512^2, 4/16/64 spp, depth 3/5/8, one wavefront launch",
            "paths": paths, "ms": ms, "value": paths / (ms / 1000.0), "unit": "path samples/s",
            "wavefront_config": st["wf_config"], "launches": st["launches"]}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle
    data = workload(args.small)
    tables = np.stack([oracle.kelemen_table(k / 20.0, 20000) for k in range(21)])
    cores = os.cpu_count() or 1
    osc = oracle.OracleScene(data, tables, use_bvh=True)
    r = data.render
    W, H = data.width, data.height
    ys = cpu_sample_rows(H)                      # the cpu_baseline leg's rows: one fixed sample
    cpu_warmup(osc, data, cores)
    for k in range(args.warmup):                 # warm-up steps: the 8 warm-up rows again
        cpu_warmup(osc, data, cores)
    times = [render_rows(osc, data, ys, cores) for _ in range(args.steps)]
    paths = W * len(ys) * r["spp"]
    ms = 1000 * statistics.mean(times)
    value = paths / (ms / 1000)
    sample = (f"{W}x{len(ys)} fixed full-width rows spread over the frame x {r['spp']} spp per step ({paths} "
              f"paths); C++ restatement with a binned-SAH binary BVH, not Embree")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "path samples/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": {"workload": f"terrain {data.ntri} tris {W}x{H} {r['spp']}spp depth {r['max_depth']}",
                       "sample": sample},
            "cpu_baseline": {"value": value, "unit": "path samples/s", "cores": cores, "kind": "port",
                             "sample": sample, "per_thread": value / cores,
                             "step_ms": [round(1000 * t, 1) for t in times]},
            "e2e": {"value": value, "unit": "path samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_profile_case(args):
    """Two 1-spp frames of the full-size scene (about 1 GB on the device), no timing output."""
    import aurora_b200 as ab
    from aurora_b200 import _abi
    data = workload(args.small)
    ctx = ab.Context(0)
    scene = ab.Scene(ctx, data)
    r = data.render
    mode = _abi.RENDER_PLAIN if args.mode == "plain" else _abi.RENDER_WAVEFRONT
    for k in range(2):
        res = scene.render(ab.render_opts(1, r["max_depth"], r["min_depth"], r["seed"], mode=mode, sample_offset=k,
                                          wf_pool=1 << 20, wf_block=128, wf_sort=1))
    print(json.dumps({"profile_case": data.name, "tris": data.ntri, "mode": args.mode, "stats": res.stats}))
    scene.close()
    ctx.close()
    return 0


def run_profile_adjoint(args):
    """One wavefront adjoint of the differentiable workload (texture scene, 256x256) at 64 spp,
    about 0.6 GB on the device, no timing output."""
    import aurora_b200 as ab
    from aurora_b200 import _abi, scenes
    data = scenes.texture_scene()
    ctx = ab.Context(0)
    scene = ab.Scene(ctx, data)
    dfilm = np.random.default_rng(8).normal(size=(data.height, data.width, 4)).astype(np.float32)
    r = data.render
    gm, gt, st = scene.adjoint(ab.render_opts(64, r["max_depth"], r["max_depth"], r["seed"],
                                              mode=_abi.RENDER_WAVEFRONT, wf_pool=1 << 20, wf_block=128, wf_sort=1),
                               dfilm)
    print(json.dumps({"profile_case": "adjoint " + data.name, "tris": data.ntri, "stats": st}))
    scene.close()
    ctx.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile:
        return run_profile_case(args)
    if args.profile_adjoint:
        return run_profile_adjoint(args)
    import torch
    import aurora_b200 as ab
    from aurora_b200 import _abi
    from aurora_b200.shard import max_over_ranks

    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    data = workload(args.small)
    W, H, spp = data.width, data.height, data.render["spp"]
    ctx = ab.Context(local)
    stream = torch.cuda.Stream()            # the library's kernels run on this stream; events are recorded on it
    torch.cuda.set_stream(stream)
    _abi.check(_abi.lib().aur_ctx_set_stream(ctx.handle, stream.cuda_stream), "aur_ctx_set_stream")
    t0 = time.perf_counter()
    scene = ab.Scene(ctx, data)
    build_s = time.perf_counter() - t0
    film = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")

    def frame(mode, count_work=0, spp_=None):
        return scene.render(render_opts_for(data, mode, rank, count_work, spp_), out=film)

    modes = {"plain": _abi.RENDER_PLAIN, "wavefront": _abi.RENDER_WAVEFRONT}
    have_wf = True
    try:
        frame(_abi.RENDER_WAVEFRONT, spp_=1)
    except ab.AuroraError:
        have_wf = False
    head = args.mode if args.mode != "auto" else ("wavefront" if have_wf else "plain")

    def timed(mode, steps, warmup):
        for _ in range(warmup):
            frame(modes[mode])
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        kernel_ms, launches, stats, host = 0.0, 0, None, []
        e0.record(stream)
        for _ in range(steps):
            t0 = time.perf_counter()
            res = frame(modes[mode])
            host.append((time.perf_counter() - t0) * 1000.0)
            kernel_ms += res.stats["kernel_ms"]
            launches += res.stats["launches"]
            stats = res.stats
        e1.record(stream)
        stats = dict(stats, host_ms_per_call=host)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist:
            ms = max_over_ranks(ms, device="cuda")
            kernel_ms = max_over_ranks(kernel_ms, device="cuda")
        return ms / steps, kernel_ms / steps, launches, stats

    # headline mode, with clocks sampled during the timed region
    clocks = Clocks(local)
    ms_step, kms_step, launches, st = timed(head, args.steps, args.warmup)
    clk = clocks.stop()
    paths_step = W * H * spp
    value = world * paths_step / (ms_step / 1000.0)
    rays_step = st["closest_rays"] + st["shadow_rays"]

    # the other renderer for the batched-vs-plain ratio
    other = {}
    if head == "wavefront":
        pms, _, _, pst = timed("plain", max(1, args.steps // 2), 1)
        other = {"plain_value": world * paths_step / (pms / 1000.0)}
        other["batched_vs_plain"] = value / other["plain_value"]
    else:
        other = {"plain_value": value, "wavefront_value": None, "batched_vs_plain": None}

    # Roofline of the dominant kernel. Algorithmic bytes come from a counting pass of the
    # plain renderer (1 spp, untimed): both renderers trace the same rays through the same
    # tree (the 4-wide one: 128-B node records; the binary one: 64 B), so node visits and
    # triangle tests (48 B) per path are the same.
    cw = frame(_abi.RENDER_PLAIN, count_work=1, spp_=1).stats
    node_b = cw["node_bytes"]
    if st.get("node_bytes", node_b) != node_b:
        raise RuntimeError("the counting pass traversed another tree than the timed renderer")
    npaths = max(cw["paths"], 1)
    closest_bpp = (cw["node_visits"] * node_b + cw["tri_tests"] * 48) / npaths
    shadow_bpp = (cw["shadow_node_visits"] * node_b + cw["shadow_tri_tests"] * 48) / npaths
    peak, peak_kind = peaks()
    if head == "plain":
        kname, kms, kbytes = "k_render_plain", kms_step, (closest_bpp + shadow_bpp) * paths_step
        shares = None
    else:
        stage = st["stage_ms"]
        shares = {k: v / max(sum(stage.values()), 1e-9) for k, v in stage.items()}
        if stage["shadow"] > stage["extend"]:
            kname, kms, kbytes = "k_shadow", stage["shadow"], shadow_bpp * paths_step
        else:
            kname, kms, kbytes = "k_extend", stage["extend"], closest_bpp * paths_step
    achieved = kbytes / (kms / 1000.0) / 1e9
    # The node and triangle records a traversal kernel fetches are served by L1 and L2 for the
    # most part (one BVH shared by every ray): the bound is the L2's read bandwidth, measured here
    # with the library's own kernel on an L2-resident buffer; HBM is the secondary line.
    l2_peak = max(ctx.read_bandwidth(48 << 20, 200) for _ in range(3))
    prof = {}
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            prof = json.load(f).get(kname) or {}
    except Exception:
        pass
    traffic = prof["dram_bytes_per_path"] * paths_step if "dram_bytes_per_path" in prof else None
    l2_traffic = prof["l2_bytes_per_path"] * paths_step if "l2_bytes_per_path" in prof else None
    roof = {"bound": "l2", "achieved": achieved, "peak": l2_peak, "unit": "GB/s", "frac": achieved / l2_peak,
            "traffic": traffic,
            "peak_kind": "measured in this run: aur_measure_read_bandwidth, 48 MiB L2-resident buffer read 200 "
                         "times with 128-bit L1-bypassing loads (best of 3)",
            "kernel": kname, "kernel_ms_per_step": kms,
            "l2_traffic": l2_traffic,
            "l2_achieved": l2_traffic / (kms / 1000.0) / 1e9 if l2_traffic else None,
            "hbm": {"achieved": traffic / (kms / 1000.0) / 1e9 if traffic else None, "peak": peak,
                    "peak_kind": peak_kind, "algorithmic_frac": achieved / peak,
                    "dram_frac": traffic / (kms / 1000.0) / 1e9 / peak if traffic else None},
            "simt_lanes_per_inst": prof.get("lanes_per_inst"), "fma_pipe_pct": prof.get("fma_pipe_pct"),
            "alu_pipe_pct": prof.get("alu_pipe_pct"), "l1tex_throughput_pct": prof.get("l1tex_throughput_pct"),
            "lts_throughput_pct": prof.get("lts_throughput_pct"), "issue_active_pct": prof.get("issue_active_pct"),
            "profile": prof.get("source"),
            "algorithmic_bytes_per_step": kbytes,
            "closest_bytes_per_path": closest_bpp, "shadow_bytes_per_path": shadow_bpp,
            "node_bytes": node_b,
            "closest_nodes_per_ray": cw["node_visits"] / max(cw["closest_rays"], 1),
            "shadow_nodes_per_ray": cw["shadow_node_visits"] / max(cw["shadow_rays"], 1),
            "stage_shares": shares}
    if head == "wavefront":
        roof["wavefront_config"] = st["wf_config"]

    # end to end through the public C ABI with host buffers (scene arrays in, image out)
    e2e = None
    if not args.no_e2e:
        desc_bytes = sum(a.nbytes for a in (data.verts, data.tri_vidx, data.tri_attr, data.corner_normals,
                                            data.corner_uvs, data.attr_material, data.attr_emission))
        # the step's inputs and its image live in pinned (page-locked) host memory, as a host
        # application that streams scenes to the GPU keeps them; filled once, outside the timing
        keep = []

        def pinned(a):
            t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
            keep.append(t)
            v = t.numpy().view(a.dtype).reshape(a.shape)
            v[...] = a
            return v
        import dataclasses
        data_h = dataclasses.replace(data, verts=pinned(data.verts), tri_vidx=pinned(data.tri_vidx),
                                     tri_attr=pinned(data.tri_attr), corner_normals=pinned(data.corner_normals),
                                     corner_uvs=pinned(data.corner_uvs), attr_material=pinned(data.attr_material),
                                     attr_emission=pinned(data.attr_emission))
        host_film = pinned(np.zeros((H, W, 4), np.float32))
        e2e_steps = max(1, args.steps)

        split = {"create": 0.0, "render": 0.0, "close": 0.0}

        def e2e_step():
            t0 = time.perf_counter()
            sc2 = ab.Scene(ctx, data_h)
            t1 = time.perf_counter()
            sc2.render(render_opts_for(data, modes[head], rank), out=host_film)
            t2 = time.perf_counter()
            sc2.close()
            t3 = time.perf_counter()
            for k, v in (("create", t1 - t0), ("render", t2 - t1), ("close", t3 - t2)):
                split[k] += v * 1000.0
        e2e_step()                                  # warm-up (untimed)
        split = dict.fromkeys(split, 0.0)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / e2e_steps
        if dist:
            dt = max_over_ranks(dt, device="cuda")
        e2e = {"value": world * paths_step / dt, "unit": "path samples/s", "h2d_bytes_per_step": int(desc_bytes),
               "d2h_bytes_per_step": int(host_film.nbytes), "ms_per_step": dt * 1000,
               "split_ms": {k: v / e2e_steps for k, v in split.items()},
               "includes": "scene upload + device BVH build + render + film download (pinned host buffers)"}

    adj = None if args.small else adjoint_ratio(ab, _abi, torch, ctx, stream)
    batch = None if args.small else batch_timing(ab, _abi, torch, ctx, stream)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the device film of the headline renderer at the same seed and samples: its rows are
        # compared with the oracle's (per-pixel 3 sigma) after the CPU leg
        frame(modes[head])
        torch.cuda.synchronize()
        gpu_film = film.cpu().numpy()
        tables = np.stack([ctx.kelemen_table(k / 20.0) for k in range(21)])
        v, sample, cores, bs, rows = cpu_baseline(data, tables)
        frac, npx = row_parity(gpu_film, rows, spp)
        cpu = {"value": v, "unit": "path samples/s", "cores": cores, "kind": "port", "sample": sample,
               "per_thread": v / cores, "bvh_build_s": bs,
               "label": "C++ restatement of the reference path with a binned-SAH binary BVH, not Embree's BVH4",
               "parity": {"pixels": npx, "frac_beyond_3sigma": frac,
                          "note": "device film rows vs the oracle's rows at equal spp and seed"}}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "path samples/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, no external data)",
                "config": {"workload": f"terrain {data.ntri} tris {W}x{H} {spp}spp depth {data.render['max_depth']} "
                                       f"roulette>2 ({head})",
                           "renderer": head, "l2": "inputs larger than L2 (BVH+triangles > 126 MB); no flush",
                           "multi_gpu": "each rank renders the full frame with its own sample indices"},
                "rays_per_s": world * rays_step / (ms_step / 1000.0), "kernel_ms_per_step": kms_step,
                "host_ms_per_call": st.get("host_ms_per_call"),
                "bvh_build_s": build_s, "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu,
                "e2e": e2e, "clocks": clk, "adjoint_forward": adj, "batch64": batch}
        line.update(other)
        print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

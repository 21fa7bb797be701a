"""PyAurora: render() and a differentiable render (torch.autograd.Function).

The reference's PyAurora (PyAurora/core.py:106-120) serialises a scene to JSON and
shells out to the renderer. Here the scene is resident on the GPU and the
renderer is called through the C ABI; `AuroraRender` exposes the path-replay
adjoint (aur_render_adjoint) as the backward of the render.

    scene = aurora_b200.Scene(ctx, data)
    params = torch.tensor(data.material_params(), device="cuda", requires_grad=True)
    texels = torch.tensor(data.texels(), device="cuda", requires_grad=True)
    image = AuroraRender.apply(params, texels, scene, dict(spp=256, max_depth=6, seed=2))
    loss = ((image[..., :3] - target) ** 2).sum(); loss.backward()
"""
from __future__ import annotations

import torch

from . import _abi
from .core import Scene, render_opts

_MODES = {"plain": _abi.RENDER_PLAIN, "wavefront": _abi.RENDER_WAVEFRONT}


def _opts(o: dict, adjoint: bool = False):
    spp = int(o.get("adjoint_spp", o["spp"]) if adjoint else o["spp"])
    depth = int(o["max_depth"])
    return render_opts(spp, depth, int(o.get("min_depth", depth)), int(o.get("seed", 0)),
                       mode=_MODES[o.get("mode", "wavefront")],
                       sample_offset=int(o.get("sample_offset", 0)))


def render(scene: Scene, spp: int, max_depth: int, min_depth: int | None = None, seed: int = 0,
           mode: str = "wavefront") -> torch.Tensor:
    """Renders `scene` into a (H, W, 4) CUDA tensor (RGB mean, alpha)."""
    film = torch.empty((scene.height, scene.width, 4), dtype=torch.float32, device=f"cuda:{scene.ctx.device}")
    torch.cuda.synchronize(film.device)
    scene.render(_opts(dict(spp=spp, max_depth=max_depth, min_depth=min_depth if min_depth is not None else max_depth,
                            seed=seed, mode=mode)), out=film)
    return film


class AuroraRender(torch.autograd.Function):
    """image = AuroraRender.apply(mat_params (nmat, 4), texels (ntexel,), scene, options).

    Forward renders with the given per-material (diffuse rgb, roughness) and texels;
    backward runs the path-replay adjoint with the same random numbers (wavefront mode: record
    pass on the wavefront engine + replay kernel; plain mode: one megakernel). options:
    spp, max_depth, min_depth, seed, mode ("wavefront" | "plain"), adjoint_spp.

    The scene holds one set of parameters, and other renders of the same scene (a target
    image, another forward) may change it between this forward and its backward. So the
    forward keeps a copy of the parameters it rendered with; the backward replays the paths
    under that copy and then puts back whatever the scene held when the backward began.
    """

    @staticmethod
    def forward(ctx, mat_params, texels, scene: Scene, options: dict):
        torch.cuda.synchronize()
        mp = mat_params.detach().contiguous().float().clone()
        tx = texels.detach().contiguous().float().clone() if texels is not None and texels.numel() else None
        scene.set_params(mp, tx)
        film = torch.empty((scene.height, scene.width, 4), dtype=torch.float32, device=mat_params.device)
        scene.render(_opts(options), out=film)
        ctx.scene, ctx.options = scene, options
        ctx.has_tex = tx is not None
        ctx.fwd_params = (mp, tx)      # not save_for_backward: the caller may update the inputs in place
        return film

    @staticmethod
    def backward(ctx, grad_film):
        scene = ctx.scene
        g = grad_film.detach().contiguous().float()
        gm = torch.zeros((scene.nmat, 4), dtype=torch.float32, device=g.device)
        gt = torch.zeros(max(scene.ntexel, 1), dtype=torch.float32, device=g.device)
        torch.cuda.synchronize()
        held_mp, held_tx = scene.get_params()
        mp, tx = ctx.fwd_params
        scene.set_params(mp, tx)
        try:
            scene.adjoint(_opts(ctx.options, adjoint=True), g, gm, gt)
        finally:
            scene.set_params(held_mp, held_tx if scene.ntexel else None)
        return gm, (gt[:scene.ntexel] if ctx.has_tex else None), None, None

"""aurora_b200 — B200 (sm_100a) path-tracing core of Aurora behind a C ABI.

The compute path is the in-tree shared library aurora_b200/lib/libaurora_b200.so
(hand-written CUDA for sm_100a); this package only binds it. Importing the
package does not load the library; the first call that needs it does, and
fails loudly if it has not been built.
"""
from ._abi import AuroraError, lib  # noqa: F401
from .core import Bvh, Context, RenderResult, Scene, render_batch, render_opts, bvh_opts, write_film  # noqa: F401

__all__ = ["AuroraError", "Bvh", "Context", "Scene", "RenderResult", "render_batch", "render_opts", "bvh_opts",
           "write_film", "lib"]

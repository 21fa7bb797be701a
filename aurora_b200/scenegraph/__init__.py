"""Scene building in Python with PyAurora's classes (PyAurora/core.py, geometry.py,
lights.py, shaders.py of espennordahl/Aurora): the same class names, constructor
arguments and methods, serialised to the same JSON scene file. `core.render(scene)`
renders it in-process on the GPU instead of writing a file and running the binary.

    from aurora_b200.scenegraph import core, geometry, lights, shaders
"""
from . import core, geometry, lights, shaders  # noqa: F401

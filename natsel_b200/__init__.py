"""natsel_b200: the reference engine's per-step rigid-body solve on one B200.

``World`` (natsel_b200.world) drives libnatsel_gpu.so through the C ABI in
include/natsel_gpu.h; ``scenes`` builds the seeded benchmark scenes.
"""
from . import scenes  # noqa: F401

__all__ = ["scenes", "World", "load_library"]


def __getattr__(name):
    if name in ("World", "load_library", "default_world_def", "NsError"):
        from . import world
        return getattr(world, name)
    raise AttributeError(name)

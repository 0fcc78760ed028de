"""slimtracin_b200 — SlimTracin's per-pixel tracing path and BVH builds on NVIDIA B200 (sm_100a).

    structs   ctypes / numpy mirrors of the reference's data contract
    scenes    seeded synthetic scenes (configs 0-2, example recipes) in that layout
    api       the ctypes binding of libslimtracin_b200.so and a small host (Renderer)
    build     nvcc build of the library
"""
from . import structs, scenes  # noqa: F401

__all__ = ["structs", "scenes", "api", "build"]

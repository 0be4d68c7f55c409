"""untangling26_b200 — B200-native collision-and-untangling hot path of Untangling26.

The compute path is libu26.so (hand-written sm_100a CUDA behind the C ABI in
include/u26.h). This package holds the host-side mirror of the reference's LBVH /
IntersectionResolver interfaces, mesh topology preparation and synthetic scenes.
"""
from ._native import Context, U26Error, load  # noqa: F401

__all__ = ["Context", "U26Error", "load"]

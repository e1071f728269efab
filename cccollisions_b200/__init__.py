"""B200-native collision engine, a drop-in for the ``cccollisions`` torch extension.

``import cccollisions`` (the alias package beside this one) or ``import cccollisions_b200`` gives
the reference's module-level functions
(bvh, bvh_motion, find_collisions, find_collisions_continuous[_partial], find_proximity,
find_mincol_cand, compute_impulses[_partial], compute_impulses_from_collisions).
"""
from .api import (  # noqa: F401
    bvh,
    bvh_motion,
    compute_impulses,
    compute_impulses_from_collisions,
    compute_impulses_partial,
    find_collisions,
    find_collisions_continuous,
    find_collisions_continuous_partial,
    find_mincol_cand,
    find_proximity,
    find_triangle_edge_candidates,
    find_triangle_edge_candidates2,
    find_triangle_edge_collisions,
)

__all__ = [
    "bvh", "bvh_motion", "find_collisions", "find_collisions_continuous", "find_collisions_continuous_partial",
    "find_proximity", "find_mincol_cand", "compute_impulses", "compute_impulses_partial",
    "compute_impulses_from_collisions", "find_triangle_edge_collisions", "find_triangle_edge_candidates",
    "find_triangle_edge_candidates2",
]

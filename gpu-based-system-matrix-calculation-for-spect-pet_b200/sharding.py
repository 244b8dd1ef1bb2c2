"""Work partitioning of a system-matrix job across ranks (one process per GPU).

Matrix elements are independent, so ranks share no data: for the photoelectric matrix each
rank owns whole voxel planes (z) of the image grid for every detector, the unit the benchmark
and the multi-GPU driver hand out.  No collective touches the data path; only the timing
reduction (max over ranks) crosses ranks.

Crystal scatter reads the photoelectric element PE[k, v] of every crystal k at the element's
own voxel v, so a rank that owns a block of voxel columns computes the PE columns of that
block itself and needs nothing from the other ranks: no all-gather of the PE matrix.
"""
from __future__ import annotations


def plane_for_step(step: int, rank: int, world: int, n_planes: int, first: int = 0) -> int:
    """z-plane processed by `rank` at `step`: ranks take interleaved planes starting at
    `first` and wrapping around the image, so every plane lies in [0, n_planes), per-rank work
    is fixed as the world grows (weak scaling) and the ranks of one step take distinct planes
    whenever world <= n_planes."""
    if n_planes < 1:
        raise ValueError("n_planes must be positive")
    return (first + step * world + rank) % n_planes


def detector_slab(n_det: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous detector rows [begin, begin + count) of `rank` when rows are split;
    sizes differ by at most one."""
    base, extra = divmod(n_det, world)
    begin = rank * base + min(rank, extra)
    return begin, base + (1 if rank < extra else 0)


def voxel_block(n_vox: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous voxel columns [begin, begin + count) of `rank` for the scatter path (the
    photoelectric columns it needs are its own); sizes differ by at most one."""
    return detector_slab(n_vox, rank, world)

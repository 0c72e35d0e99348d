"""Per-node geometry on the GPU (mirrors yggdrax/geometry.py:17-75 and
yggdrax/_geometry_impl.py:30-338)."""

from __future__ import annotations

from typing import NamedTuple, Optional

import torch

from . import _lib as L
from .dtypes import INDEX_BITS
from .tree import _dev_of, _host_of, resolve_tree_topology


class TreeGeometry(NamedTuple):
    """Bounding information for every node: ``center`` (M, 3),
    ``half_extent`` (M, 3), ``radius`` (M,), ``max_extent`` (M,)."""

    center: torch.Tensor
    half_extent: torch.Tensor
    radius: torch.Tensor
    max_extent: torch.Tensor


def compute_tree_geometry(tree, positions_sorted: torch.Tensor, *,
                          max_leaf_size: Optional[int] = None,
                          particle_radius: Optional[torch.Tensor] = None) -> TreeGeometry:
    """Per-node boxes, sphere radii and L-infinity extents.

    Leaf boxes come from Morton cells when the topology was built with
    ``use_morton_geometry`` (fixed depth), otherwise from each leaf's
    particle range in ``positions_sorted`` (at most ``max_leaf_size``
    particles per leaf, defaulting to the tree's ``leaf_size``).  Internal
    boxes are the union of their children's.  ``particle_radius`` (LET
    proxies) is outside the GPU pipeline and raises."""
    if particle_radius is not None:
        raise NotImplementedError("particle_radius is outside the GPU tree pipeline")
    topology = resolve_tree_topology(tree)
    total = int(topology.parent.shape[0])
    if int(topology.node_ranges.shape[0]) != total:
        raise ValueError("tree.node_ranges must align with tree.parent shape")
    pos = positions_sorted
    L.require_cuda(pos, "positions_sorted")
    if pos.dim() != 2 or pos.shape[1] != 3:
        raise ValueError("positions must have shape (N, 3)")
    if int(pos.shape[0]) != int(topology.num_particles):
        raise ValueError("positions_sorted must match tree.num_particles")
    if pos.dtype != torch.float32:
        raise TypeError("positions_sorted must be float32")
    pos = pos.contiguous()
    if max_leaf_size is None and getattr(topology, "leaf_size", None) is not None:
        max_leaf_size = int(topology.leaf_size)
    cap = -1 if max_leaf_size is None else int(max_leaf_size)
    use_morton = _host_of(topology).use_morton
    d = _dev_of(topology)
    dev = pos.device
    lib = L.lib()
    center = torch.empty((total, 3), dtype=torch.float32, device=dev)
    half = torch.empty((total, 3), dtype=torch.float32, device=dev)
    radius = torch.empty(total, dtype=torch.float32, device=dev)
    max_extent = torch.empty(total, dtype=torch.float32, device=dev)
    ws = L.workspace(lib.ygx_geometry_workspace_size(total), dev)
    L.check(lib.ygx_tree_geometry(
        L.ptr(topology.node_ranges), total, INDEX_BITS, L.ptr(d.parent32), L.ptr(d.left32),
        L.ptr(d.right32), L.ptr(d.level32), L.ptr(d.tree_flags), L.ptr(pos),
        int(pos.shape[0]), 1 if use_morton else 0, L.ptr(d.bounds), L.ptr(topology.leaf_codes),
        L.ptr(topology.leaf_depths), cap, L.ptr(center), L.ptr(half), L.ptr(radius),
        L.ptr(max_extent), L.ptr(ws), ws.numel(), L.stream_handle(dev)), "ygx_tree_geometry")
    return TreeGeometry(center, half, radius, max_extent)


class LevelMajorTreeGeometry(NamedTuple):
    """Tree geometry in padded level-major buffers (_geometry_impl.py:39-47):
    ``(num_levels, max_nodes_per_level[, 3])``, zero past each level's nodes,
    ``node_indices`` -1 there."""

    centers: torch.Tensor
    half_extents: torch.Tensor
    radii: torch.Tensor
    max_extents: torch.Tensor
    level_counts: torch.Tensor
    node_indices: torch.Tensor


def geometry_to_level_major(tree, geometry: TreeGeometry) -> LevelMajorTreeGeometry:
    """geometry_to_level_major (geometry.py:79-102, _geometry_impl.py:342-420):
    row l holds the geometry of the l-th level's nodes in ``nodes_by_level``
    order; one kernel (``ygx_level_major_geometry``)."""
    from .dtypes import INDEX_DTYPE

    topology = resolve_tree_topology(tree)
    d = _dev_of(topology)
    nlev = _host_of(topology).num_levels
    if nlev <= 0:
        raise ValueError("tree must contain at least one populated level")
    dev = topology.parent.device
    lo = topology.level_offsets.to(INDEX_DTYPE).contiguous()
    counts = (lo[1:] - lo[:-1])[:nlev]
    M = int(torch.clamp(counts, min=1).max())
    f = lambda *s: torch.empty(s, dtype=torch.float32, device=dev)  # noqa: E731
    out = LevelMajorTreeGeometry(
        centers=f(nlev, M, 3), half_extents=f(nlev, M, 3), radii=f(nlev, M),
        max_extents=f(nlev, M), level_counts=counts,
        node_indices=torch.empty((nlev, M), dtype=INDEX_DTYPE, device=dev))
    L.check(L.lib().ygx_level_major_geometry(
        L.ptr(d.nbl32), L.ptr(lo), INDEX_BITS, nlev, M,
        L.ptr(geometry.center.contiguous().float()),
        L.ptr(geometry.half_extent.contiguous().float()),
        L.ptr(geometry.radius.contiguous().float()),
        L.ptr(geometry.max_extent.contiguous().float()), L.ptr(out.centers),
        L.ptr(out.half_extents), L.ptr(out.radii), L.ptr(out.max_extents),
        L.ptr(out.node_indices), L.stream_handle(dev)), "ygx_level_major_geometry")
    return out


__all__ = ["TreeGeometry", "LevelMajorTreeGeometry", "compute_tree_geometry",
           "geometry_to_level_major"]

"""Dense level-major far-field buffers for a level-by-level M2L sweep.

Mirrors ``DenseInteractionBuffers`` / ``densify_interactions`` /
``build_dense_interactions`` (yggdrax/dense_interactions.py:23-254): the
sparse far lists regrouped into ``(num_levels, max_nodes, max_interactions)``
tensors of source ids (-1 padded), a validity mask, per-slot counts and
target-minus-source displacements, written by one kernel
(``ygx_dense_m2l``).  The buffers grow as levels x widest level x longest
row; a request larger than the device's free memory raises ``MemoryError``.
"""

from __future__ import annotations

from typing import NamedTuple, Optional

import torch

from . import _lib as L
from .dtypes import INDEX_BITS, INDEX_DTYPE
from .geometry import LevelMajorTreeGeometry, TreeGeometry, geometry_to_level_major
from .interactions import (DualTreeTraversalConfig, NodeInteractionList,
                           build_interactions_and_neighbors)
from .tree import resolve_tree_topology


class DenseInteractionBuffers(NamedTuple):
    """Dense level-major far-field pairs (dense_interactions.py:23-31)."""

    geometry: LevelMajorTreeGeometry
    m2l_sources: torch.Tensor
    m2l_displacements: torch.Tensor
    m2l_mask: torch.Tensor
    m2l_counts: torch.Tensor
    sparse_interactions: NodeInteractionList


def densify_interactions(tree, geometry: TreeGeometry,
                         interactions: NodeInteractionList) -> DenseInteractionBuffers:
    """densify_interactions (:149-197): slot (l, m) is the m-th node of level l
    (``nodes_by_level`` order); its row of the far list fills
    ``m2l_sources[l, m, :count]``, ``m2l_displacements`` = centre of the
    target minus centre of the source (fp32)."""
    topology = resolve_tree_topology(tree)
    lg = geometry_to_level_major(topology, geometry)
    dev = topology.parent.device
    nlev, M = int(lg.node_indices.shape[0]), int(lg.node_indices.shape[1])
    counts = interactions.counts.to(INDEX_DTYPE).contiguous()
    K = max(1, int(counts.max()) if counts.numel() else 0)
    isz = 4 if INDEX_BITS == 32 else 8
    need = nlev * M * K * (isz + 1 + 12) + nlev * M * isz
    free, _ = torch.cuda.mem_get_info(dev)
    if need > free:
        raise MemoryError(f"dense interaction buffers need {need / 2**30:.1f} GiB "
                          f"({nlev} levels x {M} nodes x {K} interactions); "
                          f"{free / 2**30:.1f} GiB free")
    src = torch.empty((nlev, M, K), dtype=INDEX_DTYPE, device=dev)
    mask = torch.empty((nlev, M, K), dtype=torch.bool, device=dev)
    cnt = torch.empty((nlev, M), dtype=INDEX_DTYPE, device=dev)
    disp = torch.empty((nlev, M, K, 3), dtype=torch.float32, device=dev)
    sources = interactions.sources.to(INDEX_DTYPE).contiguous()
    if sources.numel() == 0:
        sources = torch.zeros(1, dtype=INDEX_DTYPE, device=dev)
    L.check(L.lib().ygx_dense_m2l(
        L.ptr(lg.node_indices), INDEX_BITS, nlev * M, K, L.ptr(counts),
        L.ptr(interactions.offsets.to(INDEX_DTYPE).contiguous()), L.ptr(sources),
        L.ptr(geometry.center.contiguous().float()), int(geometry.center.shape[0]),
        L.ptr(src), L.ptr(mask), L.ptr(cnt), L.ptr(disp), L.stream_handle(dev)),
        "ygx_dense_m2l")
    return DenseInteractionBuffers(geometry=lg, m2l_sources=src, m2l_displacements=disp,
                                   m2l_mask=mask, m2l_counts=cnt,
                                   sparse_interactions=interactions)


def build_dense_interactions(tree, geometry: TreeGeometry, theta: float = 0.5, *,
                             max_pair_queue: Optional[int] = None,
                             process_block: Optional[int] = None,
                             traversal_config: Optional[DualTreeTraversalConfig] = None,
                             retry_logger=None) -> DenseInteractionBuffers:
    """build_dense_interactions (:200-247): the far lists (default MAC, like
    the reference) and their dense view."""
    interactions, _ = build_interactions_and_neighbors(
        tree, geometry, theta=theta, max_pair_queue=max_pair_queue,
        process_block=process_block, traversal_config=traversal_config,
        retry_logger=retry_logger)
    return densify_interactions(tree, geometry, interactions)


__all__ = ["DenseInteractionBuffers", "build_dense_interactions", "densify_interactions"]

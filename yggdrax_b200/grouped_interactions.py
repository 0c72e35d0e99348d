"""Class-major grouping of far-field pairs.

Mirrors ``GroupedInteractionBuffers`` / ``build_grouped_interactions`` /
``build_grouped_interactions_from_pairs`` (yggdrax/grouped_interactions.py:
21-200), which run on the host in NumPy there and on the GPU here
(``csrc/grouped.cu``): every pair's class key is (target level, source
level, displacement in target-level cells per axis, ``rint`` in float64 of
``(c_t - c_s) / max(root_extent / 2^level, 1e-12)``); pairs are ordered
stably by key, a class is a run of equal keys, and each class carries its
key and displacement ``key * cell`` (float64, stored as float32).
"""

from __future__ import annotations

from typing import NamedTuple, Optional

import numpy as np
import torch

from . import _lib as L
from .dtypes import INDEX_BITS, INDEX_DTYPE
from .geometry import TreeGeometry
from .tree import _dev_of, resolve_tree_topology


class GroupedInteractionBuffers(NamedTuple):
    """Class-major grouped far pairs (grouped_interactions.py:21-31)."""

    class_keys: torch.Tensor           # (num_classes, 5) int32
    class_displacements: torch.Tensor  # (num_classes, 3)
    class_offsets: torch.Tensor        # (num_classes + 1,)
    class_sources: torch.Tensor        # (num_pairs,) in class order
    class_targets: torch.Tensor
    class_ids: torch.Tensor            # (num_pairs,) class of each input pair
    level_offsets: torch.Tensor
    level_nodes: torch.Tensor


def build_grouped_interactions(tree, geometry: TreeGeometry, interactions
                               ) -> GroupedInteractionBuffers:
    """build_grouped_interactions (:41-72): the far list's sources / targets."""
    return build_grouped_interactions_from_pairs(
        tree, geometry, interactions.sources, interactions.targets,
        level_offsets=getattr(interactions, "level_offsets", None))


def build_grouped_interactions_from_pairs(tree, geometry: TreeGeometry, sources, targets, *,
                                          level_offsets: Optional[torch.Tensor] = None
                                          ) -> GroupedInteractionBuffers:
    """build_grouped_interactions_from_pairs (:75-200), same keys, order
    and outputs (pairs of equal key keep their input order)."""
    topology = resolve_tree_topology(tree)
    dev = topology.parent.device
    idt = INDEX_DTYPE
    src = torch.as_tensor(sources, device=dev).to(idt).contiguous()
    tgt = torch.as_tensor(targets, device=dev).to(idt).contiguous()
    lo_out = (level_offsets.to(idt) if level_offsets is not None
              else torch.zeros(1, dtype=idt, device=dev))
    P = int(src.shape[0])
    if P == 0:
        return GroupedInteractionBuffers(
            class_keys=torch.zeros((0, 5), dtype=torch.int32, device=dev),
            class_displacements=torch.zeros((0, 3), dtype=geometry.center.dtype, device=dev),
            class_offsets=torch.zeros(1, dtype=idt, device=dev),
            class_sources=torch.zeros(0, dtype=idt, device=dev),
            class_targets=torch.zeros(0, dtype=idt, device=dev),
            class_ids=torch.zeros(0, dtype=idt, device=dev), level_offsets=lo_out,
            level_nodes=topology.nodes_by_level)
    d = _dev_of(topology)
    bmin = topology.bounds_min.detach().double().cpu().numpy()
    bmax = topology.bounds_max.detach().double().cpu().numpy()
    ext = (bmax - bmin) if bmin.ndim == 1 else (bmax[0] - bmin[0])
    ext = np.ascontiguousarray(ext, dtype=np.float64)
    center = geometry.center.contiguous().float()
    lib = L.lib()
    ws = L.workspace(lib.ygx_grouped_workspace_size(P), dev)
    nc = np.zeros(1, np.int64)
    st = L.stream_handle(dev)
    L.check(lib.ygx_grouped_classes(L.ptr(src), L.ptr(tgt), INDEX_BITS, P, L.ptr(d.level32),
                                    L.ptr(center), ext.ctypes.data, nc.ctypes.data, L.ptr(ws),
                                    ws.numel(), st), "ygx_grouped_classes")
    C = int(nc[0])
    keys = torch.empty((C, 5), dtype=torch.int32, device=dev)
    disp = torch.empty((C, 3), dtype=torch.float32, device=dev)
    offsets = torch.empty(C + 1, dtype=idt, device=dev)
    cs = torch.empty(P, dtype=idt, device=dev)
    ct = torch.empty(P, dtype=idt, device=dev)
    ids = torch.empty(P, dtype=idt, device=dev)
    L.check(lib.ygx_grouped_emit(L.ptr(src), L.ptr(tgt), INDEX_BITS, P, ext.ctypes.data,
                                 L.ptr(keys), L.ptr(disp), L.ptr(offsets), L.ptr(cs), L.ptr(ct),
                                 L.ptr(ids), L.ptr(ws), ws.numel(), st), "ygx_grouped_emit")
    return GroupedInteractionBuffers(
        class_keys=keys, class_displacements=disp.to(geometry.center.dtype),
        class_offsets=offsets, class_sources=cs, class_targets=ct, class_ids=ids,
        level_offsets=lo_out, level_nodes=topology.nodes_by_level)


__all__ = ["GroupedInteractionBuffers", "build_grouped_interactions",
           "build_grouped_interactions_from_pairs"]

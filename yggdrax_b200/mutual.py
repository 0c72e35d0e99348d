"""Canonical mutual dual-tree walk on the GPU.

Mirrors ``dual_tree_walk_mutual`` / ``MutualWalkResult``
(yggdrax/_interactions_impl.py:6309-6560, exported by yggdrax/interactions.py):
the symmetric breadth-first walk that emits every unordered node pair once,
with the MAC on caller-supplied centres and radii (for a mutual FMM: centres
of mass and the largest centre-to-particle distance), canonical pairs
``a < b`` in the reference's emission order, ``-1``-padded flat lists and
device-boolean overflow flags.  The kernels are ``csrc/mutual.cu``.
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np
import torch

from . import _lib as L
from .dtypes import INDEX_BITS, INDEX_DTYPE


class MutualWalkResult(NamedTuple):
    """Flat canonical output (:6309-6336): ``far_a``/``far_b`` and
    ``near_a``/``near_b`` padded with -1 to their capacities, ``a < b`` in
    every live slot, ``*_count`` the pairs the lists would hold; the three
    flags are device booleans (a truncated list is not an error here, the
    caller must read them)."""

    far_a: torch.Tensor
    far_b: torch.Tensor
    far_count: torch.Tensor
    near_a: torch.Tensor
    near_b: torch.Tensor
    near_count: torch.Tensor
    far_overflow: torch.Tensor
    near_overflow: torch.Tensor
    queue_overflow: torch.Tensor


def dual_tree_walk_mutual(left_child_full: torch.Tensor, right_child_full: torch.Tensor,
                          centers: torch.Tensor, radii: torch.Tensor, theta: float, root, *,
                          max_pair_queue: int, far_cap: int, near_cap: int) -> MutualWalkResult:
    """Symmetric dual-tree walk emitting each unordered node pair once.

    ``left_child_full`` / ``right_child_full``: ``(total_nodes,)`` children
    with -1 on leaves; ``centers`` ``(total_nodes, 3)``, ``radii``
    ``(total_nodes,)`` float32; a pair is accepted when
    ``theta * |c_b - c_a| > r_a + r_b``; a rejected leaf pair (not a leaf with
    itself) is near; otherwise the larger node splits (both on ties or the
    diagonal).  Same arguments and result as the reference."""
    lib = L.lib()
    dev = centers.device
    total = int(centers.shape[0])
    if max_pair_queue < 1 or far_cap < 1 or near_cap < 1:
        raise ValueError("max_pair_queue, far_cap and near_cap must be >= 1")
    ib, idt = INDEX_BITS, INDEX_DTYPE
    lf = left_child_full.to(device=dev, dtype=idt).contiguous()
    rt = right_child_full.to(device=dev, dtype=idt).contiguous()
    c = centers.to(torch.float32).contiguous()
    r = radii.to(torch.float32).contiguous()
    if lf.shape[0] != total or rt.shape[0] != total or r.shape[0] != total:
        raise ValueError("children, centers and radii must cover the same nodes")
    root_i = int(root.item() if torch.is_tensor(root) else root)
    far_a = torch.empty(far_cap, dtype=idt, device=dev)
    far_b = torch.empty(far_cap, dtype=idt, device=dev)
    near_a = torch.empty(near_cap, dtype=idt, device=dev)
    near_b = torch.empty(near_cap, dtype=idt, device=dev)
    ws = L.workspace(lib.ygx_mutual_walk_workspace_size(total, int(max_pair_queue)), dev)
    counts = np.zeros(2, np.int64)
    flags = np.zeros(1, np.uint32)
    gens = np.zeros(1, np.int32)
    L.check(lib.ygx_mutual_walk(
        L.ptr(lf), L.ptr(rt), ib, L.ptr(c), L.ptr(r), total, float(theta), root_i,
        int(max_pair_queue), int(far_cap), int(near_cap), L.ptr(far_a), L.ptr(far_b),
        L.ptr(near_a), L.ptr(near_b), counts.ctypes.data, flags.ctypes.data, gens.ctypes.data,
        L.ptr(ws), ws.numel(), L.stream_handle(dev)), "ygx_mutual_walk")
    f = int(flags[0])
    b = lambda v: torch.tensor(bool(v), device=dev)  # noqa: E731
    return MutualWalkResult(
        far_a=far_a, far_b=far_b, far_count=torch.tensor(int(counts[0]), dtype=idt, device=dev),
        near_a=near_a, near_b=near_b,
        near_count=torch.tensor(int(counts[1]), dtype=idt, device=dev),
        far_overflow=b(f & 1), near_overflow=b(f & 2), queue_overflow=b(f & 4))


__all__ = ["MutualWalkResult", "dual_tree_walk_mutual"]

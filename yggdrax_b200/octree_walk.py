"""Native octree walk: far pairs in explicit octree node space and near
neighbours in octree leaf space.

Mirrors ``build_octree_native_far_pairs`` / ``build_octree_native_neighbor_lists``
(yggdrax/_interactions_impl.py:5556-5717) over ``_dual_tree_walk_octree_impl``
(:1908-2597), and ``build_explicit_octree_traversal_view`` /
``compute_explicit_octree_box_geometry`` (yggdrax/octree.py:422-704).  The walk,
the cell box geometry and the row sort run as kernels of ``libygx.so``
(``csrc/octwalk.cu``, the onesweep sort); the glue is torch on the device.

Row order: the reference appends each generation's accepted pairs to their
rows, all (first cell -> second cell) entries of the generation before all
(second -> first) entries, and orders the entries of one row inside such a
block by an unstable argsort (:813-873).  Here those blocks keep wavefront
order, so rows equal the reference's as the sequence of (generation, block)
groups, and inside a group as sets.

The reference's refinement takes the first ``child_count`` of a cell's eight
octant slots (:106-165), which skips children stored in later octants when
some earlier octant is empty; and in leaf space every cell carrying a radix
leaf counts as a leaf, the root included when a radix leaf spans it (the
walk then ends at the root).  Both are reproduced.
"""

from __future__ import annotations

from typing import Callable, NamedTuple, Optional

import numpy as np
import torch

from . import _lib as L
from .dtypes import INDEX_BITS, INDEX_DTYPE
from .interactions import (_DEFAULT_MAX_INTERACTIONS, _DEFAULT_MAX_NEIGHBORS, _MAC_CODES,
                           DEFAULT_PAIR_QUEUE_MULTIPLIER, DualTreeRetryEvent,
                           DualTreeTraversalConfig, _target_blocks)
from . import interactions as _inter

_OCT_REQUIRED = ("oct_valid_mask", "oct_parent", "oct_children", "oct_child_counts",
                 "oct_node_codes", "oct_node_depths", "oct_node_ranges", "oct_nodes_by_level",
                 "oct_level_offsets", "oct_num_levels", "oct_leaf_mask", "oct_leaf_nodes",
                 "radix_node_to_oct", "radix_leaf_to_oct", "bounds_min", "bounds_max")

_FLAG_FAR, _FLAG_NEAR, _FLAG_QUEUE, _FLAG_BAD, _FLAG_WF, _FLAG_LOG = 1, 2, 4, 8, 16, 32
_FAR_MSG = ("Native octree interaction list capacity exceeded; increase "
            "max_interactions_per_node and rebuild.")
_NEAR_MSG = ("Native octree neighbor list capacity exceeded; increase max_neighbors_per_leaf "
             "and rebuild.")
_QUEUE_MSG = "Native octree pair queue capacity exceeded; increase max_pair_queue and rebuild."

# Wavefront and log entries per cell that the last walk of a size octave
# needed, so a repeated workload sizes its buffers right the first time.
_OCT_HINTS: dict = {}


class ExplicitOctreeBoxGeometry(NamedTuple):
    """Per-cell box geometry (octree.py:39-46)."""

    centers: torch.Tensor
    half_extents: torch.Tensor
    radii: torch.Tensor
    max_extents: torch.Tensor


class ExplicitOctreeTraversalView(NamedTuple):
    """Octree tables, radix <-> octree maps and box geometry (octree.py:49-70)."""

    valid_mask: torch.Tensor
    parent: torch.Tensor
    children: torch.Tensor
    child_counts: torch.Tensor
    node_codes: torch.Tensor
    node_depths: torch.Tensor
    node_ranges: torch.Tensor
    nodes_by_level: torch.Tensor
    level_offsets: torch.Tensor
    num_levels: torch.Tensor
    leaf_mask: torch.Tensor
    leaf_nodes: torch.Tensor
    radix_node_to_oct: torch.Tensor
    radix_leaf_to_oct: torch.Tensor
    oct_to_radix_node: torch.Tensor
    oct_to_radix_leaf: torch.Tensor
    num_valid_nodes: torch.Tensor
    num_leaf_nodes: torch.Tensor
    box_centers: torch.Tensor
    box_half_extents: torch.Tensor
    box_radii: torch.Tensor
    box_max_extents: torch.Tensor


class CompactTaggedOctreeFarPairs(NamedTuple):
    """Exact-length far pairs in octree node space (:647-652): rows in the
    octree's level order, tags -1 (no pair policy)."""

    sources: torch.Tensor
    targets: torch.Tensor
    tags: torch.Tensor


class OctreeNativeNeighborList(NamedTuple):
    """Near neighbours in octree leaf space (:655-669)."""

    offsets: torch.Tensor
    neighbors: torch.Tensor
    leaf_indices: torch.Tensor
    counts: torch.Tensor
    particle_order_leaf_indices: torch.Tensor
    particle_order_to_native_leaf: torch.Tensor
    neighbor_leaf_positions: torch.Tensor
    target_block_leaf_ids: torch.Tensor
    target_block_source_leaf_ids: torch.Tensor
    target_block_valid_mask: torch.Tensor
    target_block_offsets: torch.Tensor
    target_block_size: int


def compute_explicit_octree_box_geometry(*, valid_mask, node_codes, node_depths, bounds_min,
                                         bounds_max) -> ExplicitOctreeBoxGeometry:
    """Cell boxes from (code, depth) pairs (octree.py:422-476): fp32, every
    operation rounded; zeros on invalid cells (kernel ``k_oct_box``)."""
    lib = L.lib()
    valid = torch.as_tensor(valid_mask).to(torch.uint8).contiguous()
    dev = valid.device
    M = int(valid.shape[0])
    codes = torch.as_tensor(node_codes, device=dev).contiguous()
    codes = codes.view(torch.int64) if codes.dtype == torch.uint64 else codes.to(torch.int64)
    depths = torch.as_tensor(node_depths, device=dev).to(INDEX_DTYPE).contiguous()
    bmin = np.ascontiguousarray(torch.as_tensor(bounds_min).detach().cpu().numpy(), np.float32)
    bmax = np.ascontiguousarray(torch.as_tensor(bounds_max).detach().cpu().numpy(), np.float32)
    centers = torch.empty((M, 3), dtype=torch.float32, device=dev)
    half = torch.empty((M, 3), dtype=torch.float32, device=dev)
    radii = torch.empty(M, dtype=torch.float32, device=dev)
    maxe = torch.empty(M, dtype=torch.float32, device=dev)
    L.check(lib.ygx_octree_box_geometry(
        L.ptr(valid), L.ptr(codes), L.ptr(depths), INDEX_BITS, M, bmin.ctypes.data,
        bmax.ctypes.data, L.ptr(centers), L.ptr(half), L.ptr(radii), L.ptr(maxe),
        L.stream_handle(dev)), "ygx_octree_box_geometry")
    return ExplicitOctreeBoxGeometry(centers=centers, half_extents=half, radii=radii,
                                     max_extents=maxe)


def build_explicit_octree_traversal_view(topology) -> ExplicitOctreeTraversalView:
    """octree.py:577-704: the oct tables, the smallest radix node (leaf)
    carried by each cell (-1 where none, or for invalid / non-leaf cells)
    and the box geometry."""
    missing = tuple(n for n in _OCT_REQUIRED if not hasattr(topology, n))
    if missing:
        raise ValueError("topology is missing explicit octree traversal fields: "
                         + ", ".join(missing))
    t = topology
    idt = INDEX_DTYPE
    valid = t.oct_valid_mask.to(torch.bool)
    leaf = t.oct_leaf_mask.to(torch.bool)
    dev = valid.device
    M = int(valid.shape[0])
    r2o = t.radix_node_to_oct.to(torch.int64)
    nr = int(r2o.shape[0])
    o2r = torch.full((M,), nr, dtype=torch.int64, device=dev)
    o2r.scatter_reduce_(0, r2o, torch.arange(nr, dtype=torch.int64, device=dev), "amin")
    o2r = torch.where(valid & (o2r < nr), o2r, torch.full_like(o2r, -1))
    l2o = t.radix_leaf_to_oct.to(torch.int64)
    ni = int(t.left_child.shape[0])
    lfill = ni + int(l2o.shape[0])
    o2l = torch.full((M,), lfill, dtype=torch.int64, device=dev)
    o2l.scatter_reduce_(0, l2o, torch.arange(ni, lfill, dtype=torch.int64, device=dev), "amin")
    o2l = torch.where(leaf & (o2l < lfill), o2l, torch.full_like(o2l, -1))
    box = compute_explicit_octree_box_geometry(valid_mask=valid, node_codes=t.oct_node_codes,
                                               node_depths=t.oct_node_depths,
                                               bounds_min=t.bounds_min, bounds_max=t.bounds_max)
    return ExplicitOctreeTraversalView(
        valid_mask=valid, parent=t.oct_parent.to(idt), children=t.oct_children.to(idt),
        child_counts=t.oct_child_counts.to(idt), node_codes=t.oct_node_codes,
        node_depths=t.oct_node_depths.to(idt), node_ranges=t.oct_node_ranges.to(idt),
        nodes_by_level=t.oct_nodes_by_level.to(idt), level_offsets=t.oct_level_offsets.to(idt),
        num_levels=torch.as_tensor(t.oct_num_levels).to(idt), leaf_mask=leaf,
        leaf_nodes=t.oct_leaf_nodes.to(idt), radix_node_to_oct=t.radix_node_to_oct.to(idt),
        radix_leaf_to_oct=t.radix_leaf_to_oct.to(idt), oct_to_radix_node=o2r.to(idt),
        oct_to_radix_leaf=o2l.to(idt), num_valid_nodes=valid.sum().to(idt),
        num_leaf_nodes=leaf.sum().to(idt), box_centers=box.centers,
        box_half_extents=box.half_extents, box_radii=box.radii, box_max_extents=box.max_extents)


def _capacities(tree, max_interactions_per_node, max_neighbors_per_leaf, max_pair_queue,
                process_block, traversal_config):
    """:5584-5604 / :5666-5686: the traversal config (or the module default),
    else a queue of 128 x the radix node count and the default row caps."""
    cfg = traversal_config if traversal_config is not None else _inter._GLOBAL_DUAL_TREE_CONFIG
    if cfg is not None:
        return (max(4, int(cfg.max_pair_queue)), int(cfg.max_interactions_per_node),
                int(cfg.max_neighbors_per_leaf))
    q = max(4, int(max_pair_queue) if max_pair_queue is not None
            else int(tree.parent.shape[0]) * DEFAULT_PAIR_QUEUE_MULTIPLIER)
    if process_block is not None and int(process_block) < 1:
        raise ValueError("process_block must be >= 1")
    far = int(max_interactions_per_node if max_interactions_per_node is not None
              else _DEFAULT_MAX_INTERACTIONS)
    return q, far, int(max_neighbors_per_leaf)


def _walk(view: ExplicitOctreeTraversalView, theta: float, mac_type: str,
          dehnen_radius_scale: float, *, far: bool, queue: int, far_cap: int, near_cap: int):
    """One walk collecting far rows (far=True) or near rows, re-run with
    larger buffers when the wavefront or the pair log did not fit.  Returns
    (sorted keys, sorted values, row counts, leaf cells or None, flags,
    stats, row of every cell (int32; level rank for far walks, carrier row or
    -1 for near walks))."""
    if mac_type not in _MAC_CODES:
        raise ValueError(f"Unknown mac_type: {mac_type}")
    if dehnen_radius_scale <= 0:
        raise ValueError("dehnen_radius_scale must be > 0")
    lib = L.lib()
    dev = view.parent.device
    st = L.stream_handle(dev)
    M = int(view.parent.shape[0])
    root = int(torch.argmin(view.parent).item())  # first cell without a parent
    rank = torch.empty(M, dtype=torch.int32, device=dev)
    lws = L.workspace(lib.ygx_layout_workspace_size(M), dev)
    if far:
        # rank of every cell in level order (the far rows' sort key)
        nbl = view.nodes_by_level.to(INDEX_DTYPE).contiguous()
        L.check(lib.ygx_scatter_positions(L.ptr(nbl), INDEX_BITS, M, M, L.ptr(rank), 32,
                                          L.ptr(lws), lws.numel(), st), "ygx_scatter_positions")
        leaf8 = view.leaf_mask.to(torch.uint8).contiguous()
        near_row, cells, rows = None, None, M
    else:
        # the carrier cells (those holding a radix leaf) in cell order, and the
        # row of each (-1 for the others)
        r2o = view.radix_leaf_to_oct.to(INDEX_DTYPE).contiguous()
        cells = torch.empty(M, dtype=INDEX_DTYPE, device=dev)
        nrows = np.zeros(1, np.int64)
        L.check(lib.ygx_flag_compact(L.ptr(r2o), int(r2o.shape[0]), M, INDEX_BITS, L.ptr(rank),
                                     L.ptr(cells), nrows.ctypes.data, L.ptr(lws), lws.numel(),
                                     st), "ygx_flag_compact")
        rows = int(nrows[0])
        cells = cells[:rows]
        leaf8 = (rank >= 0).to(torch.uint8).contiguous()
        near_row = rank
    children = view.children.to(INDEX_DTYPE).contiguous()
    counts = view.child_counts.to(INDEX_DTYPE).contiguous()
    hkey = ("far" if far else "near", M.bit_length())
    h_wf, h_log = _OCT_HINTS.get(hkey, (0.0, 0.0))
    wf = min(queue, max(4096, 8 * M, int(1.25 * h_wf * M)))
    log = max(65536, 16 * M, int(1.1 * h_log * M))
    cnt = torch.empty(max(rows, 1), dtype=torch.int32, device=dev)
    while True:
        key = torch.empty(log, dtype=torch.int64, device=dev)
        val = torch.empty(log, dtype=torch.int32, device=dev)
        ws = L.workspace(lib.ygx_octree_walk_workspace_size(M, wf), dev)
        stats = np.zeros(8, np.int64)
        flags = np.zeros(1, np.uint32)
        rc = lib.ygx_octree_walk(
            L.ptr(children), L.ptr(counts), INDEX_BITS, M, L.ptr(view.box_centers),
            L.ptr(view.box_radii), L.ptr(view.box_max_extents), L.ptr(leaf8),
            L.ptr(rank) if far else None, None if far else L.ptr(near_row), rows, root,
            _MAC_CODES[mac_type], float(theta), float(dehnen_radius_scale), int(queue), wf,
            int(far_cap), int(near_cap), log, L.ptr(key) if far else None,
            L.ptr(val) if far else None, None if far else L.ptr(key),
            None if far else L.ptr(val), L.ptr(cnt) if far else None,
            None if far else L.ptr(cnt), stats.ctypes.data, flags.ctypes.data, L.ptr(ws),
            ws.numel(), st)
        f = int(flags[0])
        if rc == 0 and f & _FLAG_WF:
            wf = min(queue, max(2 * wf, int(stats[6])))
            continue
        L.check(rc, "ygx_octree_walk")
        n = int(stats[0] if far else stats[1])
        stop = f & (_FLAG_FAR | _FLAG_NEAR | _FLAG_QUEUE)
        if not stop and f & _FLAG_LOG:
            log = n + n // 8 + 1024
            continue
        break
    _OCT_HINTS[hkey] = (max(h_wf, int(stats[6]) / M), max(h_log, n / M))
    if stop:
        return None, None, cnt[:rows], cells, f, stats, rank
    ko = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    vo = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
    if n:
        ws = L.workspace(lib.ygx_sort_pairs_workspace_size(n), dev)
        bits = max(1, (max(rows, 2) - 1).bit_length())
        L.check(lib.ygx_sort_pairs(L.ptr(key), L.ptr(val), n, 0, bits, L.ptr(ko), L.ptr(vo),
                                   L.ptr(ws), ws.numel(), st), "ygx_sort_pairs")
    return ko[:n], vo[:n], cnt[:rows], cells, f, stats, rank


def _octree_topology(tree, what: str):
    topo = tree.topology if hasattr(tree, "topology") else tree
    if not (hasattr(topo, "oct_children") and hasattr(topo, "oct_parent")):
        raise ValueError(f"{what} requires an octree topology")
    return topo


def build_octree_native_far_pairs(
    tree: object,
    geometry: object,
    theta: float = 0.5,
    max_interactions_per_node: Optional[int] = None,
    mac_type: str = "bh",
    *,
    pair_policy: Optional[object] = None,
    policy_state: object = None,
    max_pair_queue: Optional[int] = None,
    process_block: Optional[int] = None,
    traversal_config: Optional[DualTreeTraversalConfig] = None,
    retry_logger: Optional[Callable[[DualTreeRetryEvent], None]] = None,
    dehnen_radius_scale: float = 1.0,
) -> CompactTaggedOctreeFarPairs:
    """Exact-length far pairs directly in explicit octree node space
    (:5556-5634); ``geometry`` is unused (the walk uses the cell boxes).
    Raises the reference's ``RuntimeError`` when a row exceeds
    ``max_interactions_per_node`` (default 512) or the wavefront exceeds
    ``max_pair_queue`` (default 128 x the radix node count)."""
    del geometry, retry_logger, policy_state
    topo = _octree_topology(tree, "build_octree_native_far_pairs")
    if pair_policy is not None:
        raise NotImplementedError("pair_policy is not supported on this path")
    q, fcap, ncap = _capacities(topo, max_interactions_per_node, _DEFAULT_MAX_NEIGHBORS,
                                max_pair_queue, process_block, traversal_config)
    view = build_explicit_octree_traversal_view(topo)
    ko, vo, cnt, _, f, _, _ = _walk(view, theta, mac_type, dehnen_radius_scale, far=True,
                                    queue=q, far_cap=fcap, near_cap=ncap)
    if f & _FLAG_FAR:
        raise RuntimeError(_FAR_MSG)
    if f & _FLAG_QUEUE:
        raise RuntimeError(_QUEUE_MSG)
    sources = vo.to(INDEX_DTYPE)
    lib = L.lib()
    dev = sources.device
    nbl = view.nodes_by_level.to(INDEX_DTYPE).contiguous()
    targets = torch.empty_like(sources)
    gws = L.workspace(256, dev)
    L.check(lib.ygx_gather_index(L.ptr(nbl), int(nbl.shape[0]), L.ptr(ko.contiguous()),
                                 int(ko.shape[0]), INDEX_BITS, L.ptr(targets), L.ptr(gws),
                                 gws.numel(), L.stream_handle(dev)), "ygx_gather_index")
    tags = torch.full_like(sources, -1)
    return CompactTaggedOctreeFarPairs(sources=sources, targets=targets, tags=tags)


def build_octree_native_neighbor_lists(
    tree: object,
    geometry: object,
    theta: float = 0.5,
    max_neighbors_per_leaf: int = _DEFAULT_MAX_NEIGHBORS,
    max_interactions_per_node: Optional[int] = None,
    mac_type: str = "bh",
    *,
    pair_policy: Optional[object] = None,
    policy_state: object = None,
    max_pair_queue: Optional[int] = None,
    process_block: Optional[int] = None,
    traversal_config: Optional[DualTreeTraversalConfig] = None,
    retry_logger: Optional[Callable[[DualTreeRetryEvent], None]] = None,
    dehnen_radius_scale: float = 1.0,
) -> OctreeNativeNeighborList:
    """Exact-length near neighbours directly in explicit octree leaf space
    (:5637-5717, converted as ``_raw_to_octree_native_neighbors``
    :5411-5553): rows are the cells that carry a radix leaf, in cell order;
    neighbours are cell ids."""
    del geometry, retry_logger, policy_state
    topo = _octree_topology(tree, "build_octree_native_neighbor_lists")
    if pair_policy is not None:
        raise NotImplementedError("pair_policy is not supported on this path")
    q, fcap, ncap = _capacities(topo, max_interactions_per_node, max_neighbors_per_leaf,
                                max_pair_queue, process_block, traversal_config)
    view = build_explicit_octree_traversal_view(topo)
    ko, vo, counts32, cells, f, _, row_of_cell = _walk(
        view, theta, mac_type, dehnen_radius_scale, far=False, queue=q, far_cap=fcap,
        near_cap=ncap)
    if f & _FLAG_NEAR:
        raise RuntimeError(_NEAR_MSG)
    if f & _FLAG_QUEUE:
        raise RuntimeError(_QUEUE_MSG)
    dev = cells.device
    idt = INDEX_DTYPE
    rows = int(cells.shape[0])
    lib = L.lib()
    st = L.stream_handle(dev)
    leaf_indices = cells.to(idt)
    counts = counts32.to(idt)
    offsets = torch.empty(rows + 1, dtype=idt, device=dev)
    lws = L.workspace(lib.ygx_layout_workspace_size(rows), dev)
    L.check(lib.ygx_counts_to_offsets(L.ptr(counts) if rows else None, rows, INDEX_BITS,
                                      L.ptr(offsets), L.ptr(lws), lws.numel(), st),
            "ygx_counts_to_offsets")
    neighbors = vo.to(idt)
    # particle order of the carrier cells: stable by their first particle
    starts = view.node_ranges[leaf_indices.long(), 0].to(torch.int64).contiguous()
    order32 = torch.empty(max(rows, 1), dtype=torch.int32, device=dev)
    if rows:
        kk = torch.empty_like(starts)
        ws = L.workspace(lib.ygx_sort_pairs_workspace_size(rows), dev)
        L.check(lib.ygx_sort_pairs(L.ptr(starts), None, rows, 0, 64, L.ptr(kk), L.ptr(order32),
                                   L.ptr(ws), ws.numel(), st), "ygx_sort_pairs")
    order = order32[:rows].to(torch.int64)
    po_to_native = torch.empty(rows, dtype=idt, device=dev)
    L.check(lib.ygx_scatter_positions(L.ptr(order32), 32, rows, rows, L.ptr(po_to_native),
                                      INDEX_BITS, L.ptr(lws), lws.numel(), st),
            "ygx_scatter_positions")
    # dense (rows, longest row) table of neighbour row positions, -1 padded
    max_nbr = int(counts.max().item()) if rows else 0
    max_nbr = _inter._dense_table_width(max_nbr, rows, INDEX_BITS, dev)
    pos = torch.full((rows, max_nbr), -1, dtype=idt, device=dev)
    if max_nbr and neighbors.numel():
        # row of every neighbour cell (rank_of_cell from the carrier compaction)
        L.check(lib.ygx_dense_row_table(L.ptr(offsets), L.ptr(counts), rows, L.ptr(neighbors),
                                        L.ptr(row_of_cell), int(row_of_cell.shape[0]),
                                        INDEX_BITS, max_nbr, L.ptr(pos), st),
                "ygx_dense_row_table")
    tb = _target_blocks(counts, offsets, pos, rows, dev)
    return OctreeNativeNeighborList(
        offsets=offsets, neighbors=neighbors, leaf_indices=leaf_indices, counts=counts,
        particle_order_leaf_indices=leaf_indices[order], particle_order_to_native_leaf=po_to_native,
        neighbor_leaf_positions=pos, target_block_leaf_ids=tb[0],
        target_block_source_leaf_ids=tb[1], target_block_valid_mask=tb[2],
        target_block_offsets=tb[3], target_block_size=int(tb[4]))


__all__ = ["CompactTaggedOctreeFarPairs", "ExplicitOctreeBoxGeometry",
           "ExplicitOctreeTraversalView", "OctreeNativeNeighborList",
           "build_explicit_octree_traversal_view", "build_octree_native_far_pairs",
           "build_octree_native_neighbor_lists", "compute_explicit_octree_box_geometry"]

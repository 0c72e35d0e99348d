"""Batched point sets: many independent trees built, measured and walked
together.

Sets are stored back to back in one position / mass array and described by
``offsets`` (``S + 1`` entries, set ``s`` = points ``offsets[s] ..
offsets[s+1]``).  Every stage runs once for all sets: Morton codes with each
set's own bounds, one stable sort by (set, code), the Karras forest (set
``s`` at global node ids ``2 * leaf_off[s] - s`` in the per-tree layout),
bottom-up geometry over the forest, and one dual-tree walk whose first
wavefront holds the root pair of every set.  The per-set accessors return
exactly what the single-set functions (``build_tree``,
``compute_tree_geometry``, ``build_interactions_and_neighbors``) return for
that set alone: local node ids, the set's own offsets.

This has no counterpart in the reference, which builds one set per call.
Adaptive radix trees only (``leaf_size`` partitions).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import _lib as L
from .dtypes import INDEX_BITS, INDEX_DTYPE
from .geometry import TreeGeometry
from .interactions import (_CAPACITY_HINTS, _MAC_CODES, _WF_CAP_MAX, NodeInteractionList,
                           NodeNeighborList, _dense_neighbor_budget, _grow_wf_cap, _hint_key)
from .tree import MAX_TREE_LEVELS, RadixTreeTopology

_GENS_HINTS_BATCH: dict = {}


@dataclass
class BatchedTrees:
    """The forest of S radix trees (packed per-set arrays, local values)."""

    offsets: torch.Tensor            # (S+1,) int64, device
    leaf_off: torch.Tensor           # (S+1,) int64, device
    leaf_size: int
    positions_sorted: torch.Tensor   # (n, 3)
    masses_sorted: torch.Tensor      # (n,)
    inverse_permutation: torch.Tensor
    particle_indices: torch.Tensor   # (n,) local to each set
    morton_codes: torch.Tensor       # (n,) uint64, sets' sorted codes
    bounds: torch.Tensor             # (S, 6)
    leaf_starts: torch.Tensor
    leaf_ends: torch.Tensor
    leaf_codes: torch.Tensor
    leaf_depths: torch.Tensor
    parent: torch.Tensor             # (total,) local parent
    left_child: torch.Tensor         # (total_leaves - S,)
    right_child: torch.Tensor
    left_is_leaf: torch.Tensor
    right_is_leaf: torch.Tensor
    node_ranges: torch.Tensor        # (total, 2) local particle ranges
    node_level: torch.Tensor
    level_offsets: torch.Tensor      # (S, 65)
    nodes_by_level: torch.Tensor     # (total,) local ids
    num_levels: torch.Tensor         # (S,)
    # int32 device copies with global node ids
    parent32: torch.Tensor = field(repr=False, default=None)
    left32: torch.Tensor = field(repr=False, default=None)
    right32: torch.Tensor = field(repr=False, default=None)
    level32: torch.Tensor = field(repr=False, default=None)
    nbl32: torch.Tensor = field(repr=False, default=None)
    node_seg32: torch.Tensor = field(repr=False, default=None)
    leaf_seg32: torch.Tensor = field(repr=False, default=None)
    leafpos32: torch.Tensor = field(repr=False, default=None)
    node_base32: torch.Tensor = field(repr=False, default=None)
    leaf_base32: torch.Tensor = field(repr=False, default=None)
    seg_flags: torch.Tensor = field(repr=False, default=None)
    # host copies for slicing
    offsets_host: np.ndarray = field(repr=False, default=None)
    leaf_off_host: np.ndarray = field(repr=False, default=None)

    @property
    def num_sets(self) -> int:
        return int(self.offsets_host.shape[0]) - 1

    @property
    def total_leaves(self) -> int:
        return int(self.leaf_off_host[-1])

    @property
    def total_nodes(self) -> int:
        return 2 * self.total_leaves - self.num_sets

    def node_block(self, i: int):
        a, b = int(self.leaf_off_host[i]), int(self.leaf_off_host[i + 1])
        return 2 * a - i, 2 * (b - a) - 1

    def tree(self, i: int) -> RadixTreeTopology:
        """Set i's topology, as build_tree gives it for that set alone."""
        a, b = int(self.leaf_off_host[i]), int(self.leaf_off_host[i + 1])
        p0, p1 = int(self.offsets_host[i]), int(self.offsets_host[i + 1])
        no, tot = self.node_block(i)
        io = a - i
        dev = self.parent.device
        t = RadixTreeTopology(
            parent=self.parent[no:no + tot], left_child=self.left_child[io:io + b - a - 1],
            right_child=self.right_child[io:io + b - a - 1],
            left_is_leaf=self.left_is_leaf[io:io + b - a - 1],
            right_is_leaf=self.right_is_leaf[io:io + b - a - 1],
            particle_indices=self.particle_indices[p0:p1], morton_codes=self.morton_codes[p0:p1],
            node_ranges=self.node_ranges[no:no + tot], num_particles=p1 - p0,
            num_internal_nodes=b - a - 1, node_level=self.node_level[no:no + tot],
            level_offsets=self.level_offsets[i], nodes_by_level=self.nodes_by_level[no:no + tot],
            num_levels=self.num_levels[i], bounds_min=self.bounds[i, :3],
            bounds_max=self.bounds[i, 3:], leaf_codes=self.leaf_codes[a:b],
            leaf_depths=self.leaf_depths[a:b],
            use_morton_geometry=torch.zeros((), dtype=torch.bool, device=dev),
            leaf_size=self.leaf_size)
        return t


def shard_sets(offsets, rank: int, world: int):
    """Sets [s0, s1) of this rank when S independent sets are spread over
    ``world`` ranks (one GPU each; the sets need no exchange): contiguous
    ranges cut at the set boundaries nearest to equal point counts, so every
    rank gets a share of the points within one set's size of N / world."""
    off = np.asarray(offsets.cpu() if torch.is_tensor(offsets) else offsets, dtype=np.int64)
    S = off.shape[0] - 1
    if world < 1 or not (0 <= rank < world):
        raise ValueError("need 0 <= rank < world")
    cuts = [0]
    for k in range(1, world):
        target = off[-1] * k / world
        j = int(np.searchsorted(off, target))
        j = j if j <= S and (j == 0 or abs(off[j] - target) <= abs(off[j - 1] - target)) \
            else j - 1
        cuts.append(min(max(j, cuts[-1]), S))
    cuts.append(S)
    return cuts[rank], cuts[rank + 1]


@dataclass
class BatchLayout:
    """Set and leaf offsets of a batch: host copies and device copies.  Leaf
    counts depend only on the set sizes (ceil(n_s / leaf_size) adaptive
    leaves per set), so the whole layout is known before any kernel runs."""

    offsets_host: np.ndarray
    leaf_off_host: np.ndarray
    offsets: torch.Tensor
    leaf_off: torch.Tensor
    leaf_size: int

    @property
    def num_sets(self) -> int:
        return int(self.offsets_host.shape[0]) - 1

    @property
    def num_points(self) -> int:
        return int(self.offsets_host[-1])

    @property
    def total_leaves(self) -> int:
        return int(self.leaf_off_host[-1])


def batch_layout(offsets, n: int, leaf_size: int, dev) -> BatchLayout:
    """Validated layout of S sets over n points (``offsets``: S + 1 entries)."""
    if leaf_size < 1:
        raise ValueError("leaf_size must be >= 1")
    off_host = np.asarray(offsets.cpu() if torch.is_tensor(offsets) else offsets, dtype=np.int64)
    S = int(off_host.shape[0]) - 1
    if S < 1 or S > (1 << 16):
        raise ValueError("between 1 and 65536 sets are supported")
    if off_host[0] != 0 or off_host[-1] != n or np.any(np.diff(off_host) < 1):
        raise ValueError("offsets must start at 0, end at len(positions) and give every set "
                         ">= 1 point")
    leaves = (np.diff(off_host) + leaf_size - 1) // leaf_size
    leaf_off_host = np.concatenate([[0], np.cumsum(leaves)]).astype(np.int64)
    return BatchLayout(offsets_host=off_host, leaf_off_host=leaf_off_host,
                       offsets=torch.from_numpy(off_host).to(dev),
                       leaf_off=torch.from_numpy(leaf_off_host).to(dev), leaf_size=int(leaf_size))


def build_trees_batched(positions: torch.Tensor, masses: torch.Tensor, offsets,
                        *, leaf_size: int = 16) -> BatchedTrees:
    """Adaptive radix trees (``build_tree(..., leaf_size)``) of S point sets."""
    lay = batch_layout(offsets, int(positions.shape[0]), leaf_size, positions.device)
    return _build_on_layout(positions, masses, lay)


def _build_on_layout(positions: torch.Tensor, masses: torch.Tensor,
                     lay: BatchLayout) -> BatchedTrees:
    """The batched build on a known layout: kernel launches only, no host
    synchronization (so a CUDA graph can capture it)."""
    lib = L.lib()
    dev = positions.device
    st = L.stream_handle(dev)
    ib, idt = INDEX_BITS, INDEX_DTYPE
    pos = positions.contiguous().float()
    mass = masses.contiguous().float()
    n = int(pos.shape[0])
    S, off, off_host, leaf_size = lay.num_sets, lay.offsets, lay.offsets_host, lay.leaf_size
    ws = L.workspace(lib.ygx_batch_encode_sort_workspace_size(n), dev)
    bounds = torch.empty((S, 6), dtype=torch.float32, device=dev)
    codes = torch.empty(n, dtype=torch.uint64, device=dev)
    order = torch.empty(n, dtype=torch.int32, device=dev)
    seg_sorted = torch.empty(n, dtype=torch.int32, device=dev)
    L.check(lib.ygx_batch_encode_sort(L.ptr(pos), n, L.ptr(off), S, L.ptr(bounds), L.ptr(codes),
                                      L.ptr(order), L.ptr(seg_sorted), L.ptr(ws), ws.numel(), st),
            "ygx_batch_encode_sort")
    pos_s = torch.empty_like(pos)
    mass_s = torch.empty_like(mass)
    pidx = torch.empty(n, dtype=idt, device=dev)
    inv = torch.empty(n, dtype=idt, device=dev)
    L.check(lib.ygx_batch_reorder(L.ptr(pos), L.ptr(mass), L.ptr(order), L.ptr(seg_sorted),
                                  L.ptr(off), n, ib, L.ptr(pos_s), L.ptr(mass_s), L.ptr(pidx),
                                  L.ptr(inv), st), "ygx_batch_reorder")
    leaf_off = lay.leaf_off
    Lt = lay.total_leaves
    starts = torch.empty(Lt, dtype=idt, device=dev)
    ends = torch.empty(Lt, dtype=idt, device=dev)
    lcodes = torch.empty(Lt, dtype=torch.uint64, device=dev)
    ldepths = torch.empty(Lt, dtype=idt, device=dev)
    leaf_seg = torch.empty(Lt, dtype=torch.int32, device=dev)
    L.check(lib.ygx_batch_leaves(L.ptr(codes), L.ptr(off), L.ptr(leaf_off), S, Lt, int(leaf_size),
                                 ib, L.ptr(starts), L.ptr(ends), L.ptr(lcodes), L.ptr(ldepths),
                                 L.ptr(leaf_seg), st), "ygx_batch_leaves")
    total, ni = 2 * Lt - S, Lt - S
    e = lambda k, dt=idt: torch.empty(k, dtype=dt, device=dev)  # noqa: E731
    i32 = torch.int32
    out = dict(parent=e(total), left=e(max(ni, 0)), right=e(max(ni, 0)),
               lil=e(max(ni, 0), torch.bool), ril=e(max(ni, 0), torch.bool),
               ranges=torch.empty((total, 2), dtype=idt, device=dev), node_level=e(total),
               level_offsets=torch.empty((S, MAX_TREE_LEVELS + 1), dtype=idt, device=dev),
               nbl=e(total), num_levels=e(S), parent32=e(total, i32), left32=e(total, i32),
               right32=e(total, i32), level32=e(total, i32), nbl32=e(total, i32),
               node_seg32=e(total, i32), leafpos32=e(total, i32), node_base32=e(total, i32),
               leaf_base32=e(Lt, i32), seg_flags=e(S, i32), tree_flags=e(1, i32))
    wst = L.workspace(lib.ygx_batch_topology_workspace_size(Lt, S), dev)
    L.check(lib.ygx_batch_build_topology(
        L.ptr(lcodes), L.ptr(starts), L.ptr(ends), L.ptr(leaf_off), L.ptr(leaf_seg), S, Lt, ib,
        *[L.ptr(out[k]) for k in ("parent", "left", "right", "lil", "ril", "ranges", "node_level",
                                  "level_offsets", "nbl", "num_levels", "parent32", "left32",
                                  "right32", "level32", "nbl32", "node_seg32", "leafpos32",
                                  "node_base32", "leaf_base32", "seg_flags", "tree_flags")],
        L.ptr(wst), wst.numel(), st), "ygx_batch_build_topology")
    return BatchedTrees(
        offsets=off, leaf_off=leaf_off, leaf_size=int(leaf_size), positions_sorted=pos_s,
        masses_sorted=mass_s, inverse_permutation=inv, particle_indices=pidx,
        morton_codes=codes, bounds=bounds, leaf_starts=starts, leaf_ends=ends, leaf_codes=lcodes,
        leaf_depths=ldepths, parent=out["parent"], left_child=out["left"],
        right_child=out["right"], left_is_leaf=out["lil"], right_is_leaf=out["ril"],
        node_ranges=out["ranges"], node_level=out["node_level"],
        level_offsets=out["level_offsets"], nodes_by_level=out["nbl"],
        num_levels=out["num_levels"], parent32=out["parent32"], left32=out["left32"],
        right32=out["right32"], level32=out["level32"], nbl32=out["nbl32"],
        node_seg32=out["node_seg32"], leaf_seg32=leaf_seg, leafpos32=out["leafpos32"],
        node_base32=out["node_base32"], leaf_base32=out["leaf_base32"],
        seg_flags=out["seg_flags"].view(torch.int32), offsets_host=off_host,
        leaf_off_host=lay.leaf_off_host)


@dataclass
class BatchedGeometry:
    center: torch.Tensor
    half_extent: torch.Tensor
    radius: torch.Tensor
    max_extent: torch.Tensor

    def geometry(self, batch: BatchedTrees, i: int) -> TreeGeometry:
        no, tot = batch.node_block(i)
        return TreeGeometry(center=self.center[no:no + tot],
                            half_extent=self.half_extent[no:no + tot],
                            radius=self.radius[no:no + tot],
                            max_extent=self.max_extent[no:no + tot])


def compute_tree_geometry_batched(batch: BatchedTrees) -> BatchedGeometry:
    """``compute_tree_geometry(tree_s, positions_sorted_s, max_leaf_size=leaf_size)``
    for every set."""
    lib = L.lib()
    dev = batch.parent.device
    total = batch.total_nodes
    g = BatchedGeometry(center=torch.empty((total, 3), dtype=torch.float32, device=dev),
                        half_extent=torch.empty((total, 3), dtype=torch.float32, device=dev),
                        radius=torch.empty(total, dtype=torch.float32, device=dev),
                        max_extent=torch.empty(total, dtype=torch.float32, device=dev))
    ws = L.workspace(lib.ygx_geometry_workspace_size(total), dev)
    L.check(lib.ygx_batch_tree_geometry(
        L.ptr(batch.node_ranges), total, batch.num_sets, L.ptr(batch.leaf_off),
        L.ptr(batch.leaf_seg32), batch.total_leaves, L.ptr(batch.offsets), INDEX_BITS,
        L.ptr(batch.parent32), L.ptr(batch.left32), L.ptr(batch.right32), L.ptr(batch.level32),
        L.ptr(batch.seg_flags), L.ptr(batch.positions_sorted), int(batch.leaf_size),
        L.ptr(g.center), L.ptr(g.half_extent), L.ptr(g.radius), L.ptr(g.max_extent), L.ptr(ws),
        ws.numel(), L.stream_handle(dev)), "ygx_batch_tree_geometry")
    return g


@dataclass
class BatchedInteractions:
    """Far / near lists of every set, packed: far rows in level-major order
    set after set, near rows leaf by leaf; node ids local to each set."""

    node_offsets: torch.Tensor   # (total+1,) global row starts, node-indexed
    far_counts: torch.Tensor
    sources: torch.Tensor
    targets: torch.Tensor
    target_levels: torch.Tensor
    near_offsets: torch.Tensor   # (total_leaves+1,)
    near_counts: torch.Tensor
    neighbors: torch.Tensor
    stats: dict

    def lists(self, batch: BatchedTrees, i: int):
        """(NodeInteractionList, NodeNeighborList) of set i, as
        build_interactions_and_neighbors gives them for that set alone."""
        no, tot = batch.node_block(i)
        a, b = int(batch.leaf_off_host[i]), int(batch.leaf_off_host[i + 1])
        nl, ni = b - a, b - a - 1
        dev = self.node_offsets.device
        idt = self.node_offsets.dtype
        total = batch.total_nodes
        nbl = batch.nbl32

        def row_start(x):  # start of the x-th node in level-major order
            return int(self.node_offsets[int(nbl[x])]) if x < total else int(self.node_offsets[-1])

        f0, f1 = row_start(no), row_start(no + tot)
        offsets = torch.cat([self.node_offsets[no:no + tot] - f0,
                             torch.tensor([f1 - f0], dtype=idt, device=dev)])
        nlev = int(batch.num_levels[i])
        lo = batch.level_offsets[i].cpu().numpy()
        level_offsets = torch.tensor([row_start(no + int(lo[l])) - f0 for l in range(nlev + 1)],
                                     dtype=idt, device=dev)
        far = NodeInteractionList(
            offsets=offsets, sources=self.sources[f0:f1], targets=self.targets[f0:f1],
            counts=self.far_counts[no:no + tot], level_offsets=level_offsets,
            target_levels=self.target_levels[f0:f1])
        n0, n1 = int(self.near_offsets[a]), int(self.near_offsets[b])
        nb = self.neighbors[n0:n1]
        cnt = self.near_counts[a:b]
        max_nbr = int(cnt.max()) if nl > 0 else 0
        nlp = torch.full((nl, max_nbr), -1, dtype=idt, device=dev)
        if max_nbr > 0 and nl * max_nbr * (4 if INDEX_BITS == 32 else 8) <= \
                _dense_neighbor_budget(dev):
            rows = torch.repeat_interleave(torch.arange(nl, device=dev), cnt.long())
            starts = (self.near_offsets[a:b] - n0).long()
            cols = torch.arange(n1 - n0, device=dev) - starts[rows]
            nlp[rows, cols] = nb - ni
        elif max_nbr > 0:
            nlp = torch.empty((nl, 0), dtype=idt, device=dev)
        ar = torch.arange(nl, dtype=idt, device=dev)
        near = NodeNeighborList(
            offsets=self.near_offsets[a:b + 1] - n0, neighbors=nb,
            leaf_indices=ar + ni, counts=cnt, particle_order_leaf_indices=ar + ni,
            particle_order_to_native_leaf=ar, neighbor_leaf_positions=nlp,
            target_block_leaf_ids=torch.empty(0, dtype=idt, device=dev),
            target_block_source_leaf_ids=torch.empty(0, dtype=idt, device=dev),
            target_block_valid_mask=torch.empty(0, dtype=torch.bool, device=dev),
            target_block_offsets=torch.zeros(1, dtype=idt, device=dev), target_block_size=0)
        return far, near


def build_interactions_and_neighbors_batched(batch: BatchedTrees, geometry: BatchedGeometry, *,
                                             theta: float = 0.5, mac_type: str = "bh",
                                             dehnen_radius_scale: float = 1.0
                                             ) -> BatchedInteractions:
    """The exact far / near lists (count-then-fill semantics, no capacities)
    of every set, from one walk over the whole forest."""
    if mac_type not in _MAC_CODES:
        raise ValueError(f"Unknown mac_type '{mac_type}'")
    if float(dehnen_radius_scale) <= 0.0:
        raise ValueError("dehnen_radius_scale must be > 0")
    lib = L.lib()
    dev = batch.parent.device
    st = L.stream_handle(dev)
    ib, idt = INDEX_BITS, INDEX_DTYPE
    total, Lt, S = batch.total_nodes, batch.total_leaves, batch.num_sets
    ni = Lt - S
    mac = _MAC_CODES[mac_type]
    center = geometry.center.contiguous()
    radius = geometry.radius.contiguous()
    max_extent = geometry.max_extent.contiguous()
    z = lambda *s: torch.zeros(s, dtype=idt, device=dev)  # noqa: E731
    if ni == 0 or total < 3:  # every set is a single leaf: no pairs
        return BatchedInteractions(
            node_offsets=z(total + 1), far_counts=z(total), sources=z(0), targets=z(0),
            target_levels=z(0), near_offsets=z(Lt + 1), near_counts=z(Lt), neighbors=z(0),
            stats={})
    key = _hint_key(mac_type, theta, total, "batch")
    hint_wf, hint_log = _CAPACITY_HINTS.get(key, (0.0, 0.0))
    cap = min(_WF_CAP_MAX, max(32 * total + 65536, int(1.25 * hint_wf * total)))
    log_cap = max(8 * total + 65536, int(1.1 * hint_log * total))
    while True:
        ws = L.workspace(lib.ygx_traverse_workspace_size(total, Lt, cap, log_cap), dev)
        stats = np.zeros(L.TSTAT_WORDS, np.uint64)
        flags = np.zeros(1, np.uint32)
        rc = lib.ygx_batch_traverse_walk(
            L.ptr(center), L.ptr(radius), L.ptr(max_extent), L.ptr(batch.left32),
            L.ptr(batch.right32), L.ptr(batch.leafpos32), L.ptr(batch.parent32), total,
            L.ptr(batch.leaf_off), S, L.ptr(batch.seg_flags), mac, float(theta),
            float(dehnen_radius_scale), _GENS_HINTS_BATCH.get(key, 0), cap, log_cap,
            stats.ctypes.data, flags.ctypes.data, L.ptr(ws), ws.numel(), st)
        f = int(flags[0])
        if f & (L.FLAG_QUEUE_OVERFLOW | L.FLAG_LOG_OVERFLOW) and rc == 0:
            if f & L.FLAG_QUEUE_OVERFLOW:
                cap = _grow_wf_cap(cap, stats)
                log_cap = max(log_cap, int(stats[L.TSTAT["log_need"]]))
            else:
                # the reported need fits the re-run; head-room spares another
                # re-run when the next inputs need a little more
                log_cap = max(int(1.15 * int(stats[L.TSTAT["log_need"]])),
                              log_cap + log_cap // 4)
            continue
        L.check(rc, "ygx_batch_traverse_walk")
        if f & L.FLAG_BAD_INPUT:
            raise ValueError("MAC extents must be positive (geometry has zero or NaN extents)")
        if f:
            raise L.YgxError(f"traversal walk reported flags {f:#x}")
        break
    pw, pl = _CAPACITY_HINTS.get(key, (0.0, 0.0))  # hints only grow
    _CAPACITY_HINTS[key] = (max(pw, int(stats[L.TSTAT["wf_need"]]) / total),
                            max(pl, int(stats[L.TSTAT["log_need"]]) / total))
    _GENS_HINTS_BATCH[key] = int(stats[L.TSTAT["gens"]])
    s = {k: int(stats[v]) for k, v in L.TSTAT.items()}
    P, Q = s["far_total"], s["near_total"]
    node_offsets = torch.empty(total + 1, dtype=idt, device=dev)
    far_counts = torch.empty(total, dtype=idt, device=dev)
    level_dummy = torch.zeros(2, dtype=idt, device=dev)
    level_out = torch.empty(2, dtype=idt, device=dev)
    near_offsets = torch.empty(Lt + 1, dtype=idt, device=dev)
    near_counts = torch.empty(Lt, dtype=idt, device=dev)
    far_src32 = torch.empty(max(P, 1), dtype=torch.int32, device=dev)
    near_nbr32 = torch.empty(max(Q, 1), dtype=torch.int32, device=dev)
    L.check(lib.ygx_traverse_fill(
        total, ni, cap, log_cap, P, Q, L.ptr(batch.nbl32), L.ptr(batch.leafpos32),
        L.ptr(level_dummy), 0, ib, L.ptr(node_offsets), L.ptr(far_counts), L.ptr(level_out),
        L.ptr(near_offsets), L.ptr(near_counts), L.ptr(far_src32), L.ptr(near_nbr32), L.ptr(ws),
        ws.numel(), st), "ygx_traverse_fill")
    sources = torch.empty(P, dtype=idt, device=dev)
    targets = torch.empty(P, dtype=idt, device=dev)
    target_levels = torch.empty(P, dtype=idt, device=dev)
    neighbors = torch.empty(Q, dtype=idt, device=dev)
    L.check(lib.ygx_traverse_finalize(
        total, ni, cap, log_cap, L.ptr(batch.level32), L.ptr(batch.leafpos32), ib,
        L.ptr(far_src32), L.ptr(near_nbr32), None, None, L.ptr(batch.node_base32),
        L.ptr(batch.leaf_base32), L.ptr(sources), L.ptr(targets), L.ptr(target_levels),
        L.ptr(neighbors), None, 0, L.ptr(ws), ws.numel(), st), "ygx_traverse_finalize")
    f = L.read_status(ws)
    if f & (L.FLAG_FAR_OVERFLOW | L.FLAG_NEAR_OVERFLOW | L.FLAG_QUEUE_OVERFLOW):
        raise L.YgxError(f"traversal fill disagreed with the walk (flags {f:#x})")
    return BatchedInteractions(
        node_offsets=node_offsets, far_counts=far_counts, sources=sources, targets=targets,
        target_levels=target_levels, near_offsets=near_offsets, near_counts=near_counts,
        neighbors=neighbors, stats=s)


def _lists_fixed(batch: BatchedTrees, geometry: BatchedGeometry, mac: int, theta: float,
                 scale: float, sizes: dict):
    """Batched lists with every size fixed in ``sizes`` (gens, wf, log, far,
    near capacities): one library call, no host synchronization.  Returns
    the full-capacity outputs and the workspace holding the statistics."""
    lib = L.lib()
    dev = batch.parent.device
    idt = INDEX_DTYPE
    total, Lt, S = batch.total_nodes, batch.total_leaves, batch.num_sets
    ws = L.workspace(lib.ygx_traverse_workspace_size(total, Lt, sizes["wf"], sizes["log"]), dev)
    e = lambda k, dt=idt: torch.empty(k, dtype=dt, device=dev)  # noqa: E731
    o = dict(node_offsets=e(total + 1), far_counts=e(total), near_offsets=e(Lt + 1),
             near_counts=e(Lt), far_src32=e(sizes["far"], torch.int32),
             near_nbr32=e(sizes["near"], torch.int32), sources=e(sizes["far"]),
             targets=e(sizes["far"]), target_levels=e(sizes["far"]), neighbors=e(sizes["near"]))
    L.check(lib.ygx_batch_traverse_lists(
        L.ptr(geometry.center), L.ptr(geometry.radius), L.ptr(geometry.max_extent),
        L.ptr(batch.left32), L.ptr(batch.right32), L.ptr(batch.leafpos32), L.ptr(batch.parent32),
        L.ptr(batch.nbl32), L.ptr(batch.level32), L.ptr(batch.node_base32),
        L.ptr(batch.leaf_base32), total, L.ptr(batch.leaf_off), S, L.ptr(batch.seg_flags), mac,
        float(theta), float(scale), int(sizes["gens"]), int(sizes["wf"]), int(sizes["log"]),
        int(sizes["far"]), int(sizes["near"]), INDEX_BITS,
        *[L.ptr(o[k]) for k in ("node_offsets", "far_counts", "near_offsets", "near_counts",
                                "far_src32", "near_nbr32", "sources", "targets",
                                "target_levels", "neighbors")],
        L.ptr(ws), ws.numel(), L.stream_handle(dev)), "ygx_batch_traverse_lists")
    return o, ws


class BatchedPipeline:
    """Build, geometry and exact lists of a batch with a FIXED layout (the
    same set sizes every call, new positions), captured once in a CUDA graph
    and replayed.

    The first call runs the ordinary batched functions and records what the
    walk needed (generations, wavefront / log capacities, list totals); it
    then allocates every buffer with ``margin`` head-room and captures the
    whole pipeline -- about 150 kernel launches, no host synchronization --
    in one graph.  Later calls copy the inputs into the graph's input
    buffers, replay it and read back one small status block (one host
    synchronization per call).  If a replay did not fit (the flags say which
    size), that call's result comes from the ordinary path and the graph is
    captured again with the new sizes, so results are always the exact
    lists.

    The returned objects are views of the graph's buffers: the next call
    overwrites them (copy what must be kept).  ``last_replayed`` tells
    whether the last call came from the graph."""

    def __init__(self, offsets, *, leaf_size: int = 16, theta: float = 0.5,
                 mac_type: str = "bh", dehnen_radius_scale: float = 1.0,
                 margin: float = 1.25, device=None):
        if mac_type not in _MAC_CODES:
            raise ValueError(f"Unknown mac_type '{mac_type}'")
        if float(dehnen_radius_scale) <= 0.0:
            raise ValueError("dehnen_radius_scale must be > 0")
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        off = np.asarray(offsets.cpu() if torch.is_tensor(offsets) else offsets, dtype=np.int64)
        self.layout = batch_layout(off, int(off[-1]), leaf_size, self.device)
        self.theta, self.mac_type = float(theta), mac_type
        self.scale, self.margin = float(dehnen_radius_scale), float(margin)
        self.graph = None
        self.sizes = None
        self.captures = 0
        self.last_replayed = False

    # -- the ordinary path, which also measures the sizes ---------------------
    def _eager(self, positions, masses):
        bt = _build_on_layout(positions, masses, self.layout)
        bg = compute_tree_geometry_batched(bt)
        bi = build_interactions_and_neighbors_batched(
            bt, bg, theta=self.theta, mac_type=self.mac_type,
            dehnen_radius_scale=self.scale)
        st = bi.stats
        if st:
            m = self.margin
            self.sizes = dict(
                gens=int(st["gens"]) + 4,
                wf=max(32 * bt.total_nodes + 65536, int(m * st["wf_need"])),
                log=max(8 * bt.total_nodes + 65536, int(m * st["log_need"])),
                far=max(1024, int(m * st["far_total"])),
                near=max(1024, int(m * st["near_total"])))
        return bt, bg, bi

    def _body(self):
        bt = _build_on_layout(self.pos, self.mass, self.layout)
        bg = compute_tree_geometry_batched(bt)
        o, ws = _lists_fixed(bt, bg, _MAC_CODES[self.mac_type], self.theta, self.scale,
                             self.sizes)
        return bt, bg, o, ws

    def _capture(self):
        lay = self.layout
        self.pos = torch.empty((lay.num_points, 3), dtype=torch.float32, device=self.device)
        self.mass = torch.empty(lay.num_points, dtype=torch.float32, device=self.device)
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):  # warm-up off the capture, as CUDA graphs require
            self._body()
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.out = self._body()
        self.graph = g
        self.captures += 1

    def _views(self, stats):
        bt, bg, o, ws = self.out
        P, Q = int(stats["far_total"]), int(stats["near_total"])
        bi = BatchedInteractions(
            node_offsets=o["node_offsets"], far_counts=o["far_counts"],
            sources=o["sources"][:P], targets=o["targets"][:P],
            target_levels=o["target_levels"][:P], near_offsets=o["near_offsets"],
            near_counts=o["near_counts"], neighbors=o["neighbors"][:Q], stats=stats)
        return bt, bg, bi

    def __call__(self, positions: torch.Tensor, masses: torch.Tensor):
        """(BatchedTrees, BatchedGeometry, BatchedInteractions) of this call."""
        lay = self.layout
        if tuple(positions.shape) != (lay.num_points, 3) or masses.shape[0] != lay.num_points:
            raise ValueError("positions / masses do not match the pipeline's layout")
        if self.graph is None:
            res = self._eager(positions, masses)
            self.last_replayed = False
            if self.sizes is not None:
                self._capture()
            return res
        self.pos.copy_(positions)
        self.mass.copy_(masses)
        self.graph.replay()
        bt = self.out[0]
        total, Lt = bt.total_nodes, bt.total_leaves
        stats = np.zeros(L.TSTAT_WORDS, np.uint64)
        flags = np.zeros(1, np.uint32)
        ws = self.out[3]
        L.check(L.lib().ygx_traverse_stats_read(
            total, Lt, self.sizes["wf"], self.sizes["log"], L.ptr(ws), ws.numel(),
            stats.ctypes.data, flags.ctypes.data, L.stream_handle(self.device)),
            "ygx_traverse_stats_read")
        s = {k: int(stats[v]) for k, v in L.TSTAT.items()}
        if int(flags[0]) & L.FLAG_BAD_INPUT:
            raise ValueError("MAC extents must be positive (geometry has zero or NaN extents)")
        if int(flags[0]):  # a size did not fit: the ordinary path, then re-capture
            self.graph, self.out = None, None
            res = self._eager(positions, masses)
            self._capture()
            self.last_replayed = False
            return res
        self.last_replayed = True
        return self._views(s)

"""Tree construction on the GPU, behind yggdrax's public tree API.

Mirrors ``yggdrax/tree.py`` (public wrappers, configs, registry) and
``yggdrax/_tree_impl.py`` (Morton/LBVH and fixed-depth builds): same
functions, keyword arguments, defaults, precedence rules, return-tuple
conventions and error messages.  Every stage runs as hand-written sm_100a
kernels from ``libygx.so`` on the positions' CUDA device; outputs are torch
CUDA tensors in the reference's layouts (index arrays in ``INDEX_DTYPE``).

Differences that are part of the contract:

* positions and masses must be float32 CUDA tensors; bounds are used in
  float32.
* the ``*_jit`` variants are the same builds (there is no tracing step); the
  fixed-depth ``*_jit`` variants skip local refinement exactly like the
  reference does under ``jax.jit`` (``_tree_impl.py:252``).
* ``workspace`` is accepted for signature compatibility; buffers come from
  torch's caching allocator, and ``return_workspace`` returns the buffers of
  the new tree.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, Literal, NamedTuple, Optional

import torch

from . import _lib as L
from .dtypes import INDEX_BITS, INDEX_DTYPE

MAX_TREE_LEVELS = 64
_MAX_MORTON_LEVEL = 21


# ---------------------------------------------------------------------------
# Topology containers (field order of _tree_impl.py:24-71, octree.py:73-110)


class _RadixFields(NamedTuple):
    parent: torch.Tensor
    left_child: torch.Tensor
    right_child: torch.Tensor
    left_is_leaf: torch.Tensor
    right_is_leaf: torch.Tensor
    particle_indices: torch.Tensor
    morton_codes: torch.Tensor
    node_ranges: torch.Tensor
    num_particles: int
    num_internal_nodes: int
    node_level: torch.Tensor
    level_offsets: torch.Tensor
    nodes_by_level: torch.Tensor
    num_levels: torch.Tensor
    bounds_min: torch.Tensor
    bounds_max: torch.Tensor
    leaf_codes: torch.Tensor
    leaf_depths: torch.Tensor
    use_morton_geometry: torch.Tensor
    leaf_size: Optional[int]


class RadixTreeTopology(_RadixFields):
    """Radix (LBVH) topology: parallel arrays over ``2L - 1`` nodes, internal
    nodes first, leaf ``j`` at node ``num_internal_nodes + j``."""


class _OctreeFields(NamedTuple):
    parent: torch.Tensor
    left_child: torch.Tensor
    right_child: torch.Tensor
    left_is_leaf: torch.Tensor
    right_is_leaf: torch.Tensor
    particle_indices: torch.Tensor
    morton_codes: torch.Tensor
    node_ranges: torch.Tensor
    num_particles: int
    num_internal_nodes: int
    node_level: torch.Tensor
    level_offsets: torch.Tensor
    nodes_by_level: torch.Tensor
    num_levels: torch.Tensor
    bounds_min: torch.Tensor
    bounds_max: torch.Tensor
    leaf_codes: torch.Tensor
    leaf_depths: torch.Tensor
    use_morton_geometry: torch.Tensor
    leaf_size: Optional[int]
    oct_parent: torch.Tensor
    oct_children: torch.Tensor
    oct_child_counts: torch.Tensor
    oct_child_mask: torch.Tensor
    oct_valid_mask: torch.Tensor
    oct_node_codes: torch.Tensor
    oct_node_depths: torch.Tensor
    oct_node_ranges: torch.Tensor
    oct_nodes_by_level: torch.Tensor
    oct_level_offsets: torch.Tensor
    oct_num_levels: torch.Tensor
    oct_leaf_mask: torch.Tensor
    oct_leaf_nodes: torch.Tensor
    radix_node_to_oct: torch.Tensor
    radix_leaf_to_oct: torch.Tensor


class OctreeTopology(_OctreeFields):
    """Radix topology plus the explicit octree tables."""


class RadixTreeWorkspace(NamedTuple):
    """Buffers of a radix build (``_tree_impl.py:74-82``)."""

    parent: torch.Tensor
    left_child: torch.Tensor
    right_child: torch.Tensor
    left_is_leaf: torch.Tensor
    right_is_leaf: torch.Tensor
    node_ranges: torch.Tensor


@dataclass
class DeviceTopology:
    """int32 copies of the topology used by the geometry/traversal kernels."""

    parent32: torch.Tensor
    left32: torch.Tensor   # all nodes, -1 on leaves
    right32: torch.Tensor  # all nodes, -1 on leaves
    level32: torch.Tensor
    nbl32: torch.Tensor
    tree_flags: torch.Tensor  # int32[1] device word; YGX_FLAG_MALFORMED
    bounds: torch.Tensor  # float32[6]


@dataclass(frozen=True)
class HostTopologyInfo:
    """Host copies of the few scalars the later stages branch on, read back
    once when the tree is built (so geometry and traversal need no sync)."""

    malformed: bool     # tied leaf codes produced a non-standard topology
    num_levels: int
    use_morton: bool    # geometry from Morton cells (fixed depth)


def _host_of(topology) -> HostTopologyInfo:
    """The host info of a topology (read back now if it was not recorded)."""
    h = getattr(topology, "_host", None)
    if h is not None:
        return h
    d = _dev_of(topology)
    um = topology.use_morton_geometry
    h = HostTopologyInfo(
        malformed=bool((d.tree_flags.cpu()[0] & L.FLAG_MALFORMED) != 0),
        num_levels=int(topology.num_levels),
        use_morton=bool(um.item()) if torch.is_tensor(um) else bool(um))
    try:
        object.__setattr__(topology, "_host", h)
    except Exception:
        pass
    return h


def _dev_of(topology) -> DeviceTopology:
    """The int32 device copies of a topology (rebuilt if absent)."""
    d = getattr(topology, "_dev", None)
    if d is not None:
        return d
    dev = topology.parent.device
    total = int(topology.parent.shape[0])
    ni = int(topology.left_child.shape[0])
    fill = torch.full((total - ni,), -1, dtype=torch.int32, device=dev)
    left32 = torch.cat([topology.left_child.to(torch.int32), fill])
    right32 = torch.cat([topology.right_child.to(torch.int32), fill])
    parent32 = topology.parent.to(torch.int32)
    flags = torch.zeros(1, dtype=torch.int32, device=dev)
    if ni > 0:
        idx = torch.arange(ni, device=dev, dtype=torch.int32)
        ok = (parent32[left32[:ni].long()] == idx) & (parent32[right32[:ni].long()] == idx)
        roots = int((parent32 < 0).sum().item())
        if not bool(ok.all().item()) or roots != 1 or int(parent32[0].item()) != -1:
            flags.fill_(L.FLAG_MALFORMED)
    d = DeviceTopology(
        parent32=parent32, left32=left32, right32=right32,
        level32=topology.node_level.to(torch.int32),
        nbl32=topology.nodes_by_level.to(torch.int32), tree_flags=flags,
        bounds=torch.cat([topology.bounds_min.float(), topology.bounds_max.float()]).to(dev))
    try:
        object.__setattr__(topology, "_dev", d)
    except (AttributeError, TypeError):
        pass
    return d


# ---------------------------------------------------------------------------
# Configs and requests (tree.py:28-130)


@dataclass(frozen=True)
class TreeBuildConfig:
    """Resolved options for standard LBVH tree construction."""

    leaf_size: int = 8
    return_reordered: bool = False
    workspace: Optional[RadixTreeWorkspace] = None
    return_workspace: bool = False


@dataclass(frozen=True)
class FixedDepthTreeBuildConfig:
    """Resolved options for fixed-depth tree construction."""

    target_leaf_particles: int = 32
    return_reordered: bool = False
    workspace: Optional[RadixTreeWorkspace] = None
    return_workspace: bool = False
    max_depth: Optional[int] = None
    refine_local: bool = True
    max_refine_levels: int = 2
    aspect_threshold: float = 8.0
    min_refined_leaf_particles: int = 2


TreeType = Literal["radix", "octree", "kdtree"]
TreeBuildMode = Literal["adaptive", "fixed_depth", "static_radix"]
_VALID_BUILD_MODES = ("adaptive", "fixed_depth", "static_radix")


@dataclass(frozen=True)
class TreeBuildRequest:
    """Normalized request passed to registered tree builders."""

    positions: torch.Tensor
    masses: torch.Tensor
    build_mode: str
    bounds: Optional[tuple]
    return_reordered: bool
    workspace: Optional[RadixTreeWorkspace]
    return_workspace: bool
    leaf_size: int
    target_leaf_particles: int
    max_depth: Optional[int]
    refine_local: bool
    max_refine_levels: int
    aspect_threshold: float
    min_refined_leaf_particles: int


TreeBuilder = Callable[[TreeBuildRequest], "Tree"]


# ---------------------------------------------------------------------------
# GPU build pipeline


def _check_inputs(positions: torch.Tensor, masses: torch.Tensor):
    L.require_cuda(positions, "positions")
    if positions.dim() != 2 or positions.shape[1] != 3:
        raise ValueError("positions must have shape (N, 3)")
    if positions.dtype != torch.float32:
        raise TypeError("positions must be float32")
    n = int(positions.shape[0])
    if n < 1:
        raise ValueError("Need at least one particle")
    if masses.shape[0] != n:
        raise ValueError("masses must have shape (N,)")
    return positions.contiguous(), masses.to(device=positions.device,
                                             dtype=torch.float32).contiguous(), n


def _bounds_tensor(bounds, device) -> Optional[torch.Tensor]:
    if bounds is None:
        return None
    lo = torch.as_tensor(bounds[0], dtype=torch.float32).reshape(3)
    hi = torch.as_tensor(bounds[1], dtype=torch.float32).reshape(3)
    return torch.cat([lo, hi]).to(device).contiguous()


def _resolve_fixed_depth_level(num_particles: int, target_leaf_particles: int, *,
                               max_allowed_depth: int) -> int:
    """``_tree_impl.py:1358-1370``."""
    target = max(1, int(target_leaf_particles))
    if num_particles <= target:
        return 0
    target_leaves = math.ceil(num_particles / target)
    depth = math.ceil(math.log(target_leaves, 8))
    return int(min(depth, max_allowed_depth))


def _ws(nbytes: int, device) -> torch.Tensor:
    return L.workspace(nbytes, device)


def _encode_sort(pos, n, bounds_in, dev, st):
    lib = L.lib()
    bounds_dev = torch.empty(6, dtype=torch.float32, device=dev)
    codes = torch.empty(n, dtype=torch.uint64, device=dev)
    order = torch.empty(n, dtype=torch.int32, device=dev)
    ws = _ws(lib.ygx_encode_sort_workspace_size(n), dev)
    L.check(lib.ygx_encode_sort(L.ptr(pos), n, L.ptr(bounds_in), L.ptr(bounds_dev), L.ptr(codes),
                                L.ptr(order), L.ptr(ws), ws.numel(), st), "ygx_encode_sort")
    return bounds_dev, codes, order, ws


def _build(positions, masses, bounds, *, build_mode: str, leaf_size: int = 8,
           target_leaf_particles: int = 32, max_depth: Optional[int] = None,
           refine_local: bool = True, max_refine_levels: int = 2,
           aspect_threshold: float = 8.0, min_refined_leaf_particles: int = 2,
           return_reordered: bool = False):
    """Morton encode -> stable sort -> leaf partitions -> Karras -> levels.

    Follows ``_tree_impl.build_tree`` (:354-420), ``build_fixed_depth_tree``
    (:423-519) and ``_build_tree_from_leaf_partitions`` (:1009-1355).
    Returns ``(topology, positions_sorted, masses_sorted, inverse)``."""
    pos, mass, n = _check_inputs(positions, masses)
    if build_mode == "adaptive" and leaf_size < 1:
        raise ValueError("leaf_size must be >= 1")
    if build_mode == "fixed_depth" and target_leaf_particles < 1:
        raise ValueError("target_leaf_particles must be >= 1")
    dev = pos.device
    lib = L.lib()
    st = L.stream_handle(dev)
    ib, idt = INDEX_BITS, INDEX_DTYPE
    bounds_dev, codes, order, ws0 = _encode_sort(pos, n, _bounds_tensor(bounds, dev), dev, st)

    pos_sorted = torch.empty((n, 3), dtype=torch.float32, device=dev)
    mass_sorted = torch.empty(n, dtype=torch.float32, device=dev)
    pidx = torch.empty(n, dtype=idt, device=dev)
    inv = torch.empty(n, dtype=idt, device=dev)
    # (x, y, z, mass) records: the Morton-order gather then reads one aligned
    # 16-byte record per particle
    packed = torch.empty((n, 4), dtype=torch.float32, device=dev)
    L.check(lib.ygx_pack_particles(L.ptr(pos), L.ptr(mass), n, L.ptr(packed), st),
            "ygx_pack_particles")
    L.check(lib.ygx_reorder_packed(L.ptr(packed), L.ptr(order), n, ib, L.ptr(pos_sorted),
                                   L.ptr(mass_sorted), L.ptr(pidx), L.ptr(inv), st),
            "ygx_reorder_packed")
    del packed

    use_morton = build_mode == "fixed_depth"
    tree_leaf_size: Optional[int] = None
    max_cell_depth = _MAX_MORTON_LEVEL
    if build_mode == "adaptive":
        Lf = (n + leaf_size - 1) // leaf_size
        starts = torch.empty(Lf, dtype=idt, device=dev)
        ends = torch.empty(Lf, dtype=idt, device=dev)
        lcodes = torch.empty(Lf, dtype=torch.uint64, device=dev)
        ldepths = torch.empty(Lf, dtype=idt, device=dev)
        L.check(lib.ygx_leaves_adaptive(L.ptr(codes), n, leaf_size, ib, L.ptr(starts),
                                        L.ptr(ends), L.ptr(lcodes), L.ptr(ldepths), st),
                "ygx_leaves_adaptive")
        tree_leaf_size = int(leaf_size)
    elif build_mode == "fixed_depth":
        max_allowed = min(MAX_TREE_LEVELS - 1, _MAX_MORTON_LEVEL)
        if max_depth is not None:
            max_allowed = min(max_allowed, int(max_depth))
        depth = _resolve_fixed_depth_level(n, target_leaf_particles,
                                           max_allowed_depth=max_allowed)
        if depth == 0:
            starts = torch.zeros(1, dtype=idt, device=dev)
            ends = torch.full((1,), n, dtype=idt, device=dev)
            lcodes = torch.zeros(1, dtype=torch.uint64, device=dev)
            ldepths = torch.zeros(1, dtype=idt, device=dev)
        else:
            if depth > 10:
                raise ValueError(f"fixed depth {depth} needs 8^{depth} dense buckets; "
                                 "the GPU build supports depth <= 10")
            Lf = 1 << (3 * depth)
            starts = torch.empty(Lf, dtype=idt, device=dev)
            ends = torch.empty(Lf, dtype=idt, device=dev)
            lcodes = torch.empty(Lf, dtype=torch.uint64, device=dev)
            ldepths = torch.empty(Lf, dtype=idt, device=dev)
            L.check(lib.ygx_leaves_fixed(L.ptr(codes), n, depth, ib, L.ptr(starts), L.ptr(ends),
                                         L.ptr(lcodes), L.ptr(ldepths), st), "ygx_leaves_fixed")
        max_cell_depth = depth
        if refine_local:
            Lb = int(starts.shape[0])
            wsr = _ws(lib.ygx_refine_workspace_size(Lb), dev)
            total_out = torch.empty(1, dtype=torch.int64, device=dev)
            args = (L.ptr(pos_sorted), L.ptr(codes), L.ptr(starts), L.ptr(ends), L.ptr(lcodes),
                    L.ptr(ldepths), Lb, depth, int(max_refine_levels), float(aspect_threshold),
                    int(min_refined_leaf_particles), ib)
            L.check(lib.ygx_refine_count(*args, L.ptr(total_out), L.ptr(wsr), wsr.numel(), st),
                    "ygx_refine_count")
            Lr = int(total_out.item())
            if L.read_status(wsr) & L.FLAG_QUEUE_OVERFLOW:
                raise RuntimeError("local refinement exceeded its per-bucket stack")
            r_starts = torch.empty(Lr, dtype=idt, device=dev)
            r_ends = torch.empty(Lr, dtype=idt, device=dev)
            r_codes = torch.empty(Lr, dtype=torch.uint64, device=dev)
            r_depths = torch.empty(Lr, dtype=idt, device=dev)
            L.check(lib.ygx_refine_emit(*args, L.ptr(r_starts), L.ptr(r_ends), L.ptr(r_codes),
                                        L.ptr(r_depths), L.ptr(wsr), wsr.numel(), st),
                    "ygx_refine_emit")
            starts, ends, lcodes, ldepths = r_starts, r_ends, r_codes, r_depths
            max_cell_depth = min(_MAX_MORTON_LEVEL, depth + max(0, int(max_refine_levels)))
    else:
        raise ValueError(f"Unsupported build_mode '{build_mode}'")

    Lf = int(starts.shape[0])
    bmin, bmax = bounds_dev[:3].clone(), bounds_dev[3:].clone()
    if Lf == 1:
        # _tree_impl.py:1052-1110
        level_offsets = torch.zeros(MAX_TREE_LEVELS + 1, dtype=idt, device=dev)
        level_offsets[1] = 1
        topo = RadixTreeTopology(
            parent=torch.full((1,), -1, dtype=idt, device=dev),
            left_child=torch.empty(0, dtype=idt, device=dev),
            right_child=torch.empty(0, dtype=idt, device=dev),
            left_is_leaf=torch.empty(0, dtype=torch.bool, device=dev),
            right_is_leaf=torch.empty(0, dtype=torch.bool, device=dev),
            particle_indices=pidx, morton_codes=codes,
            node_ranges=torch.tensor([[0, n - 1]], dtype=idt, device=dev),
            num_particles=n, num_internal_nodes=0,
            node_level=torch.zeros(1, dtype=idt, device=dev), level_offsets=level_offsets,
            nodes_by_level=torch.zeros(1, dtype=idt, device=dev),
            num_levels=torch.ones((), dtype=idt, device=dev), bounds_min=bmin, bounds_max=bmax,
            leaf_codes=lcodes, leaf_depths=ldepths,
            use_morton_geometry=torch.full((), use_morton, dtype=torch.bool, device=dev),
            leaf_size=tree_leaf_size)
        m1 = torch.full((1,), -1, dtype=torch.int32, device=dev)
        topo._dev = DeviceTopology(parent32=m1, left32=m1.clone(), right32=m1.clone(),
                                   level32=torch.zeros(1, dtype=torch.int32, device=dev),
                                   nbl32=torch.zeros(1, dtype=torch.int32, device=dev),
                                   tree_flags=torch.zeros(1, dtype=torch.int32, device=dev),
                                   bounds=bounds_dev)
    else:
        total, ni = 2 * Lf - 1, Lf - 1
        parent = torch.empty(total, dtype=idt, device=dev)
        left = torch.empty(ni, dtype=idt, device=dev)
        right = torch.empty(ni, dtype=idt, device=dev)
        lil = torch.empty(ni, dtype=torch.bool, device=dev)
        ril = torch.empty(ni, dtype=torch.bool, device=dev)
        ranges = torch.empty((total, 2), dtype=idt, device=dev)
        node_level = torch.empty(total, dtype=idt, device=dev)
        level_offsets = torch.empty(MAX_TREE_LEVELS + 1, dtype=idt, device=dev)
        nbl = torch.empty(total, dtype=idt, device=dev)
        num_levels = torch.empty((), dtype=idt, device=dev)
        i32 = dict(dtype=torch.int32, device=dev)
        parent32, left32, right32 = (torch.empty(total, **i32) for _ in range(3))
        level32, nbl32 = torch.empty(total, **i32), torch.empty(total, **i32)
        flags = torch.zeros(1, **i32)
        wst = _ws(lib.ygx_topology_workspace_size(Lf), dev)
        L.check(lib.ygx_build_topology(
            L.ptr(lcodes), L.ptr(starts), L.ptr(ends), Lf, ib, L.ptr(parent), L.ptr(left),
            L.ptr(right), L.ptr(lil), L.ptr(ril), L.ptr(ranges), L.ptr(node_level),
            L.ptr(level_offsets), L.ptr(nbl), L.ptr(num_levels), L.ptr(parent32), L.ptr(left32),
            L.ptr(right32), L.ptr(level32), L.ptr(nbl32), L.ptr(flags), L.ptr(wst), wst.numel(),
            st), "ygx_build_topology")
        topo = RadixTreeTopology(
            parent=parent, left_child=left, right_child=right, left_is_leaf=lil,
            right_is_leaf=ril, particle_indices=pidx, morton_codes=codes, node_ranges=ranges,
            num_particles=n, num_internal_nodes=ni, node_level=node_level,
            level_offsets=level_offsets, nodes_by_level=nbl, num_levels=num_levels,
            bounds_min=bmin, bounds_max=bmax, leaf_codes=lcodes, leaf_depths=ldepths,
            use_morton_geometry=torch.full((), use_morton, dtype=torch.bool, device=dev),
            leaf_size=tree_leaf_size)
        topo._dev = DeviceTopology(parent32=parent32, left32=left32, right32=right32,
                                   level32=level32, nbl32=nbl32, tree_flags=flags,
                                   bounds=bounds_dev)
    topo._max_cell_depth = max_cell_depth
    # one read-back for the flags and the level count
    hv = torch.cat([topo._dev.tree_flags.to(torch.int64).reshape(1),
                    topo.num_levels.to(torch.int64).reshape(1)]).cpu()
    topo._host = HostTopologyInfo(malformed=bool(int(hv[0]) & L.FLAG_MALFORMED),
                                  num_levels=int(hv[1]), use_morton=bool(use_morton))
    return topo, pos_sorted, mass_sorted, inv


def augment_radix_topology_with_octree(topology) -> OctreeTopology:
    """``octree.py:553-574``: radix fields plus explicit octree tables."""
    lib = L.lib()
    dev = topology.parent.device
    st = L.stream_handle(dev)
    ib, idt = INDEX_BITS, INDEX_DTYPE
    total = int(topology.node_ranges.shape[0])
    ni = (total - 1) // 2
    Lf = total - ni
    M = max(1, 2 * Lf - 1)
    e = lambda *shape, dt=idt: torch.empty(shape, dtype=dt, device=dev)  # noqa: E731
    o = dict(
        oct_parent=e(M), oct_children=e(M, 8), oct_child_counts=e(M),
        oct_child_mask=e(M, 8, dt=torch.bool), oct_valid_mask=e(M, dt=torch.bool),
        oct_node_codes=e(M, dt=torch.uint64), oct_node_depths=e(M), oct_node_ranges=e(M, 2),
        oct_nodes_by_level=e(M), oct_level_offsets=e(_MAX_MORTON_LEVEL + 2),
        oct_num_levels=e(), oct_leaf_mask=e(M, dt=torch.bool), oct_leaf_nodes=e(M),
        radix_node_to_oct=e(total), radix_leaf_to_oct=e(Lf))
    ws = _ws(lib.ygx_octree_workspace_size(Lf), dev)
    depth_hint = getattr(topology, "_max_cell_depth", _MAX_MORTON_LEVEL)
    L.check(lib.ygx_octree_tables(
        L.ptr(topology.node_ranges), total, L.ptr(topology.morton_codes),
        int(topology.morton_codes.shape[0]), L.ptr(topology.leaf_codes),
        L.ptr(topology.leaf_depths), int(depth_hint), ib,
        *[L.ptr(o[k]) for k in (
            "oct_parent", "oct_children", "oct_child_counts", "oct_child_mask", "oct_valid_mask",
            "oct_node_codes", "oct_node_depths", "oct_node_ranges", "oct_nodes_by_level",
            "oct_level_offsets", "oct_num_levels", "oct_leaf_mask", "oct_leaf_nodes",
            "radix_node_to_oct", "radix_leaf_to_oct")],
        L.ptr(ws), ws.numel(), st), "ygx_octree_tables")
    base = tuple(getattr(topology, name) for name in _RadixFields._fields)
    out = OctreeTopology(*base, *(o[k] for k in _OctreeFields._fields[len(_RadixFields._fields):]))
    out._dev = _dev_of(topology)
    out._host = _host_of(topology)
    out._max_cell_depth = depth_hint
    return out


def build_explicit_octree_metadata(topology) -> dict:
    """Octree tables of a radix topology as a dict (``octree.py:479-550``)."""
    aug = augment_radix_topology_with_octree(topology)
    return {k: getattr(aug, k) for k in _OctreeFields._fields[len(_RadixFields._fields):]}


# ---------------------------------------------------------------------------
# Public tree containers (tree.py:184-830)


@dataclass(frozen=True)
class Tree:
    """Public base class for concrete tree containers."""

    @property
    def num_nodes(self) -> int:
        return int(self.topology.parent.shape[0])

    @property
    def num_particles(self) -> int:
        return int(self.topology.num_particles)

    @property
    def num_leaves(self) -> int:
        t = self.topology
        return int(t.parent.shape[0]) - int(t.num_internal_nodes)

    def __getattr__(self, name):
        if name == "topology":
            raise AttributeError(name)
        return getattr(self.topology, name)

    @classmethod
    def from_particles(cls, positions, masses, *, tree_type: str = "radix",
                       build_mode: str = "adaptive", bounds=None, return_reordered: bool = True,
                       workspace=None, return_workspace: bool = False, leaf_size: int = 8,
                       target_leaf_particles: int = 32, max_depth: Optional[int] = None,
                       refine_local: bool = True, max_refine_levels: int = 2,
                       aspect_threshold: float = 8.0, min_refined_leaf_particles: int = 2):
        """Build a concrete tree, dispatching on ``tree_type`` (tree.py:243-341)."""
        request = TreeBuildRequest(
            positions=positions, masses=masses, build_mode=build_mode, bounds=bounds,
            return_reordered=return_reordered, workspace=workspace,
            return_workspace=return_workspace, leaf_size=leaf_size,
            target_leaf_particles=target_leaf_particles, max_depth=max_depth,
            refine_local=refine_local, max_refine_levels=max_refine_levels,
            aspect_threshold=aspect_threshold,
            min_refined_leaf_particles=min_refined_leaf_particles)
        builder = _TREE_BUILDERS.get(tree_type)
        if builder is None:
            supported = ", ".join(f"'{name}'" for name in sorted(_TREE_BUILDERS))
            raise ValueError(f"Unsupported tree_type '{tree_type}'. Supported: ({supported})")
        return builder(request)


def _workspace_of(topology) -> RadixTreeWorkspace:
    return RadixTreeWorkspace(topology.parent, topology.left_child, topology.right_child,
                              topology.left_is_leaf, topology.right_is_leaf,
                              topology.node_ranges)


@dataclass(frozen=True)
class RadixTree(Tree):
    """Concrete radix-tree container (tree.py:585-721)."""

    topology: RadixTreeTopology
    build_mode: TreeBuildMode = "adaptive"
    positions_sorted: Optional[torch.Tensor] = None
    masses_sorted: Optional[torch.Tensor] = None
    inverse_permutation: Optional[torch.Tensor] = None
    workspace: Optional[RadixTreeWorkspace] = None

    @property
    def tree_type(self) -> str:
        return "radix"

    @classmethod
    def from_particles(cls, positions, masses, *, build_mode: str = "adaptive", bounds=None,
                       return_reordered: bool = True, workspace=None,
                       return_workspace: bool = False, leaf_size: int = 8,
                       target_leaf_particles: int = 32, max_depth: Optional[int] = None,
                       refine_local: bool = True, max_refine_levels: int = 2,
                       aspect_threshold: float = 8.0, min_refined_leaf_particles: int = 2):
        if build_mode == "static_radix":
            raise NotImplementedError(
                "build_mode='static_radix' is outside the GPU tree pipeline")
        if build_mode not in ("adaptive", "fixed_depth"):
            raise ValueError(
                "Unsupported build_mode "
                f"'{build_mode}'. Supported: ('adaptive', 'fixed_depth', 'static_radix')")
        topo, ps, ms, inv = _build(
            positions, masses, bounds, build_mode=build_mode, leaf_size=leaf_size,
            target_leaf_particles=target_leaf_particles, max_depth=max_depth,
            refine_local=refine_local, max_refine_levels=max_refine_levels,
            aspect_threshold=aspect_threshold,
            min_refined_leaf_particles=min_refined_leaf_particles,
            return_reordered=return_reordered)
        return cls._make(topo, build_mode, return_reordered, return_workspace, ps, ms, inv)

    @classmethod
    def _make(cls, topo, build_mode, return_reordered, return_workspace, ps, ms, inv):
        return cls(topology=topo, build_mode=build_mode,
                   positions_sorted=ps if return_reordered else None,
                   masses_sorted=ms if return_reordered else None,
                   inverse_permutation=inv if return_reordered else None,
                   workspace=_workspace_of(topo) if return_workspace else None)


@dataclass(frozen=True)
class OctreeTree(RadixTree):
    """Oct-tree container (tree.py:724-830)."""

    @property
    def tree_type(self) -> str:
        return "octree"

    @property
    def oct_num_nodes(self) -> int:
        return int(self.topology.oct_valid_mask.sum().item())

    @property
    def oct_num_leaf_nodes(self) -> int:
        return int(self.topology.oct_leaf_mask.sum().item())

    @classmethod
    def from_particles(cls, positions, masses, *, build_mode: str = "adaptive", bounds=None,
                       return_reordered: bool = True, workspace=None,
                       return_workspace: bool = False, leaf_size: int = 8,
                       target_leaf_particles: int = 32, max_depth: Optional[int] = None,
                       refine_local: bool = True, max_refine_levels: int = 2,
                       aspect_threshold: float = 8.0, min_refined_leaf_particles: int = 2):
        if build_mode not in _VALID_BUILD_MODES:
            supported = ", ".join(f"'{name}'" for name in _VALID_BUILD_MODES)
            raise ValueError(f"Unsupported build_mode '{build_mode}'. Supported: ({supported})")
        if build_mode not in ("adaptive", "fixed_depth"):
            raise ValueError("Unsupported build_mode "
                             f"'{build_mode}'. Supported: ('adaptive', 'fixed_depth')")
        topo, ps, ms, inv = _build(
            positions, masses, bounds, build_mode=build_mode, leaf_size=leaf_size,
            target_leaf_particles=target_leaf_particles, max_depth=max_depth,
            refine_local=refine_local, max_refine_levels=max_refine_levels,
            aspect_threshold=aspect_threshold,
            min_refined_leaf_particles=min_refined_leaf_particles,
            return_reordered=return_reordered)
        return cls._make(augment_radix_topology_with_octree(topo), build_mode,
                         return_reordered, return_workspace, ps, ms, inv)


def _build_radix_tree_from_request(request: TreeBuildRequest) -> Tree:
    return RadixTree.from_particles(
        request.positions, request.masses, build_mode=request.build_mode,
        bounds=request.bounds, return_reordered=request.return_reordered,
        workspace=request.workspace, return_workspace=request.return_workspace,
        leaf_size=request.leaf_size, target_leaf_particles=request.target_leaf_particles,
        max_depth=request.max_depth, refine_local=request.refine_local,
        max_refine_levels=request.max_refine_levels, aspect_threshold=request.aspect_threshold,
        min_refined_leaf_particles=request.min_refined_leaf_particles)


def _build_octree_from_request(request: TreeBuildRequest) -> Tree:
    return OctreeTree.from_particles(
        request.positions, request.masses, build_mode=request.build_mode,
        bounds=request.bounds, return_reordered=request.return_reordered,
        workspace=request.workspace, return_workspace=request.return_workspace,
        leaf_size=request.leaf_size, target_leaf_particles=request.target_leaf_particles,
        max_depth=request.max_depth, refine_local=request.refine_local,
        max_refine_levels=request.max_refine_levels, aspect_threshold=request.aspect_threshold,
        min_refined_leaf_particles=request.min_refined_leaf_particles)


_TREE_BUILDERS: dict = {
    "radix": _build_radix_tree_from_request,
    "octree": _build_octree_from_request,
}


def available_tree_types() -> tuple:
    """Registered tree-type identifiers (tree.py:1303-1305)."""
    return tuple(sorted(_TREE_BUILDERS.keys()))


def register_tree_builder(tree_type: str, builder: TreeBuilder, *, overwrite: bool = False) -> None:
    """Register a builder for ``Tree.from_particles`` dispatch (tree.py:1308-1321)."""
    normalized = tree_type.strip()
    if not normalized:
        raise ValueError("tree_type must be a non-empty string")
    if (normalized in _TREE_BUILDERS) and (not overwrite):
        raise ValueError(f"tree_type '{normalized}' is already registered; "
                         "pass overwrite=True to replace it")
    _TREE_BUILDERS[normalized] = builder


# ---------------------------------------------------------------------------
# Public build functions (tree.py:1412-1879)


def _resolve(config, return_reordered, workspace, return_workspace):
    if config is None:
        return return_reordered, return_workspace
    return config.return_reordered, config.return_workspace


def _wrap(cls, topo, build_mode, rr, rw, ps, ms, inv):
    """Return conventions of _wrap_radix_public_result (tree.py:1324-1365)."""
    tree = cls._make(topo, build_mode, rr, rw, ps, ms, inv)
    if rr and rw:
        return tree, ps, ms, inv, tree.workspace
    if rr:
        return tree, ps, ms, inv
    if rw:
        return tree, tree.workspace
    return tree


def build_tree(positions, masses, bounds=None, *, return_reordered: bool = False,
               leaf_size: int = 8, workspace: Optional[RadixTreeWorkspace] = None,
               return_workspace: bool = False, config: Optional[TreeBuildConfig] = None):
    """Adaptive LBVH radix tree (tree.py:1412-1478)."""
    rr, rw = _resolve(config, return_reordered, workspace, return_workspace)
    ls = config.leaf_size if config is not None else leaf_size
    topo, ps, ms, inv = _build(positions, masses, bounds, build_mode="adaptive", leaf_size=ls,
                               return_reordered=rr)
    return _wrap(RadixTree, topo, "adaptive", rr, rw, ps, ms, inv)


def build_octree(positions, masses, bounds=None, *, return_reordered: bool = False,
                 leaf_size: int = 8, workspace: Optional[RadixTreeWorkspace] = None,
                 return_workspace: bool = False, config: Optional[TreeBuildConfig] = None):
    """Adaptive octree: radix build + explicit octree tables (tree.py:1481-1549)."""
    rr, rw = _resolve(config, return_reordered, workspace, return_workspace)
    ls = config.leaf_size if config is not None else leaf_size
    topo, ps, ms, inv = _build(positions, masses, bounds, build_mode="adaptive", leaf_size=ls,
                               return_reordered=rr)
    return _wrap(OctreeTree, augment_radix_topology_with_octree(topo), "adaptive", rr, rw, ps,
                 ms, inv)


def _fixed_kwargs(config, target_leaf_particles, max_depth, refine_local, max_refine_levels,
                  aspect_threshold, min_refined_leaf_particles):
    if config is not None:
        return dict(target_leaf_particles=config.target_leaf_particles,
                    max_depth=config.max_depth, refine_local=config.refine_local,
                    max_refine_levels=config.max_refine_levels,
                    aspect_threshold=config.aspect_threshold,
                    min_refined_leaf_particles=config.min_refined_leaf_particles)
    return dict(target_leaf_particles=target_leaf_particles, max_depth=max_depth,
                refine_local=refine_local, max_refine_levels=max_refine_levels,
                aspect_threshold=aspect_threshold,
                min_refined_leaf_particles=min_refined_leaf_particles)


def build_fixed_depth_tree(positions, masses, bounds=None, *, target_leaf_particles: int = 32,
                           return_reordered: bool = False, workspace=None,
                           return_workspace: bool = False, max_depth: Optional[int] = None,
                           refine_local: bool = True, max_refine_levels: int = 2,
                           aspect_threshold: float = 8.0, min_refined_leaf_particles: int = 2,
                           config: Optional[FixedDepthTreeBuildConfig] = None):
    """Fixed-depth Morton tree with local aspect refinement (tree.py:1628-1726)."""
    rr, rw = _resolve(config, return_reordered, workspace, return_workspace)
    kw = _fixed_kwargs(config, target_leaf_particles, max_depth, refine_local,
                       max_refine_levels, aspect_threshold, min_refined_leaf_particles)
    topo, ps, ms, inv = _build(positions, masses, bounds, build_mode="fixed_depth",
                               return_reordered=rr, **kw)
    return _wrap(RadixTree, topo, "fixed_depth", rr, rw, ps, ms, inv)


def build_fixed_depth_octree(positions, masses, bounds=None, *, target_leaf_particles: int = 32,
                             return_reordered: bool = False, workspace=None,
                             return_workspace: bool = False, max_depth: Optional[int] = None,
                             refine_local: bool = True, max_refine_levels: int = 2,
                             aspect_threshold: float = 8.0, min_refined_leaf_particles: int = 2,
                             config: Optional[FixedDepthTreeBuildConfig] = None):
    """Fixed-depth octree (tree.py:1821-1879)."""
    rr, rw = _resolve(config, return_reordered, workspace, return_workspace)
    kw = _fixed_kwargs(config, target_leaf_particles, max_depth, refine_local,
                       max_refine_levels, aspect_threshold, min_refined_leaf_particles)
    topo, ps, ms, inv = _build(positions, masses, bounds, build_mode="fixed_depth",
                               return_reordered=rr, **kw)
    return _wrap(OctreeTree, augment_radix_topology_with_octree(topo), "fixed_depth", rr, rw,
                 ps, ms, inv)


def build_tree_jit(*args, **kwargs):
    """Same build as :func:`build_tree` (no tracing step on this backend)."""
    return build_tree(*args, **kwargs)


def build_octree_jit(*args, **kwargs):
    """Same build as :func:`build_octree`."""
    return build_octree(*args, **kwargs)


def build_fixed_depth_tree_jit(*args, **kwargs):
    """:func:`build_fixed_depth_tree` without local refinement, as under jit."""
    cfg = kwargs.get("config")
    if cfg is not None:
        kwargs["config"] = FixedDepthTreeBuildConfig(**{**cfg.__dict__, "refine_local": False})
    kwargs["refine_local"] = False
    return build_fixed_depth_tree(*args, **kwargs)


def build_fixed_depth_octree_jit(*args, **kwargs):
    """:func:`build_fixed_depth_octree` without local refinement, as under jit."""
    cfg = kwargs.get("config")
    if cfg is not None:
        kwargs["config"] = FixedDepthTreeBuildConfig(**{**cfg.__dict__, "refine_local": False})
    kwargs["refine_local"] = False
    return build_fixed_depth_octree(*args, **kwargs)


# ---------------------------------------------------------------------------
# Topology helpers (tree.py:1055-1300)


def resolve_tree_topology(tree_or_topology):
    topology = getattr(tree_or_topology, "topology", None)
    return tree_or_topology if topology is None else topology


def get_num_internal_nodes(tree) -> int:
    t = resolve_tree_topology(tree)
    return int(t.left_child.shape[0])


def get_leaf_nodes(tree) -> torch.Tensor:
    t = resolve_tree_topology(tree)
    total = int(t.node_ranges.shape[0])
    return torch.arange(get_num_internal_nodes(t), total, dtype=INDEX_DTYPE,
                        device=t.node_ranges.device)


def get_node_levels(tree) -> torch.Tensor:
    return resolve_tree_topology(tree).node_level


def get_level_offsets(tree) -> torch.Tensor:
    return resolve_tree_topology(tree).level_offsets


def get_nodes_by_level(tree) -> torch.Tensor:
    return resolve_tree_topology(tree).nodes_by_level


def get_num_levels(tree) -> int:
    return _host_of(resolve_tree_topology(tree)).num_levels


__all__ = [
    "MAX_TREE_LEVELS", "RadixTreeTopology", "OctreeTopology", "RadixTreeWorkspace",
    "TreeBuildConfig", "FixedDepthTreeBuildConfig", "TreeBuildRequest", "TreeBuilder",
    "TreeType", "TreeBuildMode", "Tree", "RadixTree", "OctreeTree", "available_tree_types",
    "register_tree_builder", "build_tree", "build_octree", "build_fixed_depth_tree",
    "build_fixed_depth_octree", "build_tree_jit", "build_octree_jit",
    "build_fixed_depth_tree_jit", "build_fixed_depth_octree_jit",
    "augment_radix_topology_with_octree", "build_explicit_octree_metadata",
    "resolve_tree_topology", "get_num_internal_nodes", "get_leaf_nodes", "get_node_levels",
    "get_level_offsets", "get_nodes_by_level", "get_num_levels",
]

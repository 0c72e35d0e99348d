"""CPU oracle for the yggdrax tree pipeline -- TEST INFRASTRUCTURE ONLY.

A restatement of the reference algorithm used to check the CUDA product
(``yggdrax_b200``) bit for bit.  Only ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline legs of ``bench.py`` may import this module; the product
never does.

The heavy lifting lives in ``ygx_oracle.cpp`` (C++17 + OpenMP, compiled with
``-ffp-contract=off``); this module holds the thin orchestration that mirrors
the reference's public functions and returns numpy arrays:

* ``infer_bounds`` -- ``yggdrax/bounds.py:11-33``
* ``morton_encode`` -- ``yggdrax/morton.py:43-77``
* ``build_tree`` / ``build_fixed_depth_tree`` -- ``yggdrax/_tree_impl.py:354-519``
  and ``:1009-1401`` (Karras build, levels, fixed-depth buckets, refinement)
* ``octree_metadata`` -- ``yggdrax/octree.py:168-550``
* ``compute_tree_geometry`` -- ``yggdrax/_geometry_impl.py:176-338``
* ``build_interactions_and_neighbors`` -- ``yggdrax/_interactions_impl.py``
  (MAC 338-395, extents 993-1061, walk 1119-1905 / 2600-3558, result layouts
  3561-3837), with rows in canonical ascending order.

Parity status: the refinement helper is pinned against the reference's own
NumPy function (golden fixtures in ``tests/golden``); the remaining stages are
pinned against golden fixtures produced by running the reference's source in
this container over a NumPy stand-in for ``jax.numpy`` (see
``tests/golden/make_golden.py``).  Bit patterns that depend on XLA's own
lowering (fp32 reduction order of ``linalg.norm``/``sum``, FMA contraction)
follow IEEE evaluation in the written order and are documented as such.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "ygx_oracle.cpp")
_LIB_PATH = os.path.join(_HERE, "libygx_oracle.so")
_lib = None

MAX_TREE_LEVELS = 64
_MAX_MORTON_LEVEL = 21
_DEFAULT_MAX_NEIGHBORS = 2048


def build(force: bool = False) -> str:
    """Compile the C++ oracle into ``oracle/libygx_oracle.so``."""
    if (
        not force
        and os.path.exists(_LIB_PATH)
        and os.path.getmtime(_LIB_PATH) >= os.path.getmtime(_SRC)
    ):
        return _LIB_PATH
    cmd = [
        "g++", "-O3", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
        "-fPIC", "-shared", _SRC, "-o", _LIB_PATH,
    ]
    subprocess.run(cmd, check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    P = ctypes.c_void_p
    i64 = ctypes.c_int64
    lib.ygo_walk.restype = ctypes.c_void_p
    lib.ygo_walk.argtypes = [P, P, P, P, i64, i64, ctypes.c_float, ctypes.c_int, i64]
    lib.ygo_walk_sizes.argtypes = [P, P]
    lib.ygo_walk_lists.argtypes = [P, i64, P, P, i64, P, P, P, P, P, P, P]
    lib.ygo_walk_free.argtypes = [P]
    lib.ygo_refine.restype = i64
    lib.ygo_refine.argtypes = [P, P, P, P, P, P, i64, ctypes.c_int, ctypes.c_int,
                               ctypes.c_double, ctypes.c_int, i64, P, P, P, P]
    lib.ygo_octree_metadata.restype = i64
    lib.ygo_geometry.restype = ctypes.c_int
    lib.ygo_geometry.argtypes = [P, i64, P, P, P, P, i64, ctypes.c_int, P, P, P, P, i64,
                                 P, P, P, P]
    lib.ygo_num_threads.restype = ctypes.c_int
    _lib = lib
    return lib


def _p(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data) if a.size else ctypes.c_void_p(0)


def num_threads() -> int:
    return int(_load().ygo_num_threads())


def set_num_threads(t: int) -> None:
    _load().ygo_set_num_threads(ctypes.c_int(int(t)))


# ---------------------------------------------------------------------------
# L0 primitives


def infer_bounds(positions: np.ndarray):
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    mn = np.empty(3, np.float32)
    mx = np.empty(3, np.float32)
    _load().ygo_infer_bounds(_p(pos), ctypes.c_int64(pos.shape[0]), _p(mn), _p(mx))
    return mn, mx


def morton_encode(positions: np.ndarray, bounds) -> np.ndarray:
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    bmin = np.ascontiguousarray(bounds[0], dtype=np.float32)
    bmax = np.ascontiguousarray(bounds[1], dtype=np.float32)
    codes = np.empty(pos.shape[0], np.uint64)
    _load().ygo_morton_encode(_p(pos), ctypes.c_int64(pos.shape[0]), _p(bmin), _p(bmax),
                              _p(codes))
    return codes


def stable_argsort_u64(keys: np.ndarray, key_bits: int = 64) -> np.ndarray:
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    out = np.empty(keys.shape[0], np.int64)
    _load().ygo_stable_argsort_u64(_p(keys), ctypes.c_int64(keys.shape[0]),
                                   ctypes.c_int(key_bits), _p(out))
    return out


# ---------------------------------------------------------------------------
# L1 tree build


@dataclass
class OracleTree:
    """Field-for-field mirror of the reference ``RadixTree`` topology
    (``_tree_impl.py:24-71``), optionally extended with the ``oct_*`` fields
    of ``OctreeTopology`` (``octree.py:73-110``)."""

    parent: np.ndarray
    left_child: np.ndarray
    right_child: np.ndarray
    left_is_leaf: np.ndarray
    right_is_leaf: np.ndarray
    particle_indices: np.ndarray
    morton_codes: np.ndarray
    node_ranges: np.ndarray
    num_particles: int
    num_internal_nodes: int
    node_level: np.ndarray
    level_offsets: np.ndarray
    nodes_by_level: np.ndarray
    num_levels: int
    bounds_min: np.ndarray
    bounds_max: np.ndarray
    leaf_codes: np.ndarray
    leaf_depths: np.ndarray
    use_morton_geometry: bool
    leaf_size: Optional[int]
    octree: Optional[dict] = None
    positions_sorted: Optional[np.ndarray] = None
    masses_sorted: Optional[np.ndarray] = None
    inverse_permutation: Optional[np.ndarray] = None
    extras: dict = field(default_factory=dict)


def resolve_fixed_depth_level(num_particles: int, target: int, max_allowed_depth: int) -> int:
    """``_tree_impl.py:1358-1370``."""
    target = max(1, int(target))
    if num_particles <= target:
        return 0
    target_leaves = math.ceil(num_particles / target)
    depth = math.ceil(math.log(target_leaves, 8))
    return int(min(depth, max_allowed_depth))


def _tree_from_partitions(pos, mass, order, sorted_codes, starts, ends, bounds, *,
                          leaf_size, use_morton, leaf_codes=None, leaf_depths=None,
                          return_reordered=True) -> OracleTree:
    """``_tree_impl.py:1009-1355`` (_build_tree_from_leaf_partitions)."""
    lib = _load()
    n = pos.shape[0]
    L = int(starts.shape[0])
    starts = np.ascontiguousarray(starts, np.int64)
    ends = np.ascontiguousarray(ends, np.int64)
    if leaf_codes is None:
        leaf_codes = sorted_codes[np.clip(starts, 0, n - 1)]
    leaf_codes = np.ascontiguousarray(leaf_codes, np.uint64)
    if leaf_depths is None:
        leaf_depths = np.full(L, -1, np.int64)
    leaf_depths = np.ascontiguousarray(leaf_depths, np.int64)
    if L == 1:
        level_offsets = np.zeros(MAX_TREE_LEVELS + 1, np.int64)
        level_offsets[1] = 1
        t = OracleTree(
            parent=np.array([-1], np.int64), left_child=np.zeros(0, np.int64),
            right_child=np.zeros(0, np.int64), left_is_leaf=np.zeros(0, bool),
            right_is_leaf=np.zeros(0, bool), particle_indices=order,
            morton_codes=sorted_codes, node_ranges=np.array([[0, n - 1]], np.int64),
            num_particles=n, num_internal_nodes=0, node_level=np.zeros(1, np.int64),
            level_offsets=level_offsets, nodes_by_level=np.zeros(1, np.int64),
            num_levels=1, bounds_min=bounds[0], bounds_max=bounds[1],
            leaf_codes=leaf_codes, leaf_depths=leaf_depths,
            use_morton_geometry=use_morton, leaf_size=leaf_size)
    else:
        total = 2 * L - 1
        ni = L - 1
        parent = np.empty(total, np.int64)
        left = np.empty(ni, np.int64)
        right = np.empty(ni, np.int64)
        lil = np.empty(ni, np.uint8)
        ril = np.empty(ni, np.uint8)
        ranges = np.empty((total, 2), np.int64)
        lib.ygo_karras(_p(leaf_codes), _p(starts), _p(ends), ctypes.c_int64(L), _p(parent),
                       _p(left), _p(right), _p(lil), _p(ril), _p(ranges))
        node_level = np.empty(total, np.int64)
        level_offsets = np.empty(MAX_TREE_LEVELS + 1, np.int64)
        nbl = np.empty(total, np.int64)
        nl = np.zeros(1, np.int64)
        lib.ygo_levels(_p(parent), ctypes.c_int64(total), _p(node_level), _p(level_offsets),
                       _p(nbl), _p(nl))
        t = OracleTree(
            parent=parent, left_child=left, right_child=right,
            left_is_leaf=lil.astype(bool), right_is_leaf=ril.astype(bool),
            particle_indices=order, morton_codes=sorted_codes, node_ranges=ranges,
            num_particles=n, num_internal_nodes=ni, node_level=node_level,
            level_offsets=level_offsets, nodes_by_level=nbl, num_levels=int(nl[0]),
            bounds_min=bounds[0], bounds_max=bounds[1], leaf_codes=leaf_codes,
            leaf_depths=leaf_depths, use_morton_geometry=use_morton, leaf_size=leaf_size)
    if return_reordered:
        t.positions_sorted = pos[order]
        t.masses_sorted = mass[order]
        inv = np.empty(n, np.int64)
        inv[order] = np.arange(n, dtype=np.int64)
        t.inverse_permutation = inv
    return t


def _encode_and_sort(pos, bounds):
    codes = morton_encode(pos, bounds)
    order = stable_argsort_u64(codes, 63)
    return codes, order, codes[order]


def build_tree(positions, masses, bounds=None, *, leaf_size: int = 8,
               return_reordered: bool = True) -> OracleTree:
    """``tree.py:1412-1478`` -> ``_tree_impl.py:354-420``."""
    pos = np.ascontiguousarray(positions, np.float32)
    mass = np.ascontiguousarray(masses, np.float32)
    n = pos.shape[0]
    if n < 1:
        raise ValueError("Need at least one particle")
    if leaf_size < 1:
        raise ValueError("leaf_size must be >= 1")
    bounds = infer_bounds(pos) if bounds is None else (
        np.asarray(bounds[0], np.float32), np.asarray(bounds[1], np.float32))
    _, order, sc = _encode_and_sort(pos, bounds)
    starts = np.arange(0, n, leaf_size, dtype=np.int64)
    ends = np.minimum(starts + leaf_size, n)
    return _tree_from_partitions(pos, mass, order, sc, starts, ends, bounds,
                                 leaf_size=int(leaf_size), use_morton=False,
                                 return_reordered=return_reordered)


def fixed_depth_partitions(sorted_codes: np.ndarray, depth: int, n: int):
    """``_tree_impl.py:1373-1401``."""
    depth = max(0, int(depth))
    if depth == 0:
        return (np.array([0], np.int64), np.array([n], np.int64),
                np.array([0], np.uint64), np.array([0], np.int64))
    L = 1 << (3 * depth)
    starts = np.empty(L, np.int64)
    ends = np.empty(L, np.int64)
    codes = np.empty(L, np.uint64)
    depths = np.empty(L, np.int64)
    _load().ygo_fixed_depth_partitions(_p(sorted_codes), ctypes.c_int64(n), ctypes.c_int(depth),
                                       _p(starts), _p(ends), _p(codes), _p(depths))
    return starts, ends, codes, depths


def refine_partitions(pos_sorted, sorted_codes, starts, ends, codes, depths, current_depth,
                      max_refine_levels=2, aspect_threshold=8.0, min_leaf_particles=2):
    """``_tree_impl.py:96-227`` (_refine_leaf_partitions_by_aspect)."""
    lib = _load()
    pos_sorted = np.ascontiguousarray(pos_sorted, np.float32)
    sorted_codes = np.ascontiguousarray(sorted_codes, np.uint64)
    args = [np.ascontiguousarray(a, dt) for a, dt in
            ((starts, np.int64), (ends, np.int64), (codes, np.uint64), (depths, np.int64))]
    L = args[0].shape[0]
    cap = 4 * L + 64
    while True:
        o = [np.empty(cap, np.int64), np.empty(cap, np.int64), np.empty(cap, np.uint64),
             np.empty(cap, np.int64)]
        m = lib.ygo_refine(_p(pos_sorted), _p(sorted_codes), *[_p(a) for a in args],
                           ctypes.c_int64(L), ctypes.c_int(int(current_depth)),
                           ctypes.c_int(int(max_refine_levels)),
                           ctypes.c_double(float(aspect_threshold)),
                           ctypes.c_int(int(min_leaf_particles)), ctypes.c_int64(cap),
                           *[_p(a) for a in o])
        if m <= cap:
            return tuple(a[:m].copy() for a in o)
        cap = int(m)


def build_fixed_depth_tree(positions, masses, bounds=None, *, target_leaf_particles: int = 32,
                           max_depth: Optional[int] = None, refine_local: bool = True,
                           max_refine_levels: int = 2, aspect_threshold: float = 8.0,
                           min_refined_leaf_particles: int = 2,
                           return_reordered: bool = True) -> OracleTree:
    """``tree.py:1628-1726`` -> ``_tree_impl.py:423-519``."""
    pos = np.ascontiguousarray(positions, np.float32)
    mass = np.ascontiguousarray(masses, np.float32)
    n = pos.shape[0]
    if n < 1:
        raise ValueError("Need at least one particle")
    if target_leaf_particles < 1:
        raise ValueError("target_leaf_particles must be >= 1")
    bounds = infer_bounds(pos) if bounds is None else (
        np.asarray(bounds[0], np.float32), np.asarray(bounds[1], np.float32))
    _, order, sc = _encode_and_sort(pos, bounds)
    max_allowed = min(MAX_TREE_LEVELS - 1, _MAX_MORTON_LEVEL)
    if max_depth is not None:
        max_allowed = min(max_allowed, int(max_depth))
    depth = resolve_fixed_depth_level(n, target_leaf_particles, max_allowed)
    starts, ends, codes, depths = fixed_depth_partitions(sc, depth, n)
    if refine_local:
        starts, ends, codes, depths = refine_partitions(
            pos[order], sc, starts, ends, codes, depths, depth, max_refine_levels,
            aspect_threshold, min_refined_leaf_particles)
    t = _tree_from_partitions(pos, mass, order, sc, starts, ends, bounds, leaf_size=None,
                              use_morton=True, leaf_codes=codes, leaf_depths=depths,
                              return_reordered=return_reordered)
    t.extras["resolved_depth"] = depth
    return t


def octree_metadata(tree: OracleTree) -> dict:
    """``octree.py:479-550`` (build_explicit_octree_metadata)."""
    lib = _load()
    total = tree.node_ranges.shape[0]
    ni = (total - 1) // 2
    L = total - ni
    M = max(1, 2 * L - 1)
    o = dict(
        oct_parent=np.empty(M, np.int64), oct_children=np.empty((M, 8), np.int64),
        oct_child_counts=np.empty(M, np.int64), oct_child_mask=np.empty((M, 8), np.uint8),
        oct_valid_mask=np.empty(M, np.uint8), oct_node_codes=np.empty(M, np.uint64),
        oct_node_depths=np.empty(M, np.int64), oct_node_ranges=np.empty((M, 2), np.int64),
        oct_nodes_by_level=np.empty(M, np.int64), oct_level_offsets=np.empty(23, np.int64),
        oct_num_levels=np.empty(1, np.int64), oct_leaf_mask=np.empty(M, np.uint8),
        oct_leaf_nodes=np.empty(M, np.int64), radix_node_to_oct=np.empty(total, np.int64),
        radix_leaf_to_oct=np.empty(L, np.int64))
    ranges = np.ascontiguousarray(tree.node_ranges, np.int64)
    codes = np.ascontiguousarray(tree.morton_codes, np.uint64)
    lc = np.ascontiguousarray(tree.leaf_codes, np.uint64)
    ld = np.ascontiguousarray(tree.leaf_depths, np.int64)
    lib.ygo_octree_metadata(
        _p(ranges), ctypes.c_int64(total), _p(codes), ctypes.c_int64(codes.shape[0]), _p(lc),
        _p(ld), *[_p(o[k]) for k in (
            "oct_parent", "oct_children", "oct_child_counts", "oct_child_mask",
            "oct_valid_mask", "oct_node_codes", "oct_node_depths", "oct_node_ranges",
            "oct_nodes_by_level", "oct_level_offsets", "oct_num_levels", "oct_leaf_mask",
            "oct_leaf_nodes", "radix_node_to_oct", "radix_leaf_to_oct")])
    for k in ("oct_child_mask", "oct_valid_mask", "oct_leaf_mask"):
        o[k] = o[k].astype(bool)
    o["oct_num_levels"] = int(o["oct_num_levels"][0])
    return o


def build_octree(positions, masses, bounds=None, *, leaf_size: int = 8,
                 return_reordered: bool = True) -> OracleTree:
    """``tree.py:1481-1549``: adaptive partition + explicit octree tables."""
    t = build_tree(positions, masses, bounds, leaf_size=leaf_size,
                   return_reordered=return_reordered)
    t.octree = octree_metadata(t)
    return t


def build_fixed_depth_octree(positions, masses, bounds=None, **kw) -> OracleTree:
    """``tree.py:1821-1879``."""
    t = build_fixed_depth_tree(positions, masses, bounds, **kw)
    t.octree = octree_metadata(t)
    return t


# ---------------------------------------------------------------------------
# L2 geometry


@dataclass
class OracleGeometry:
    center: np.ndarray
    half_extent: np.ndarray
    radius: np.ndarray
    max_extent: np.ndarray


def compute_tree_geometry(tree: OracleTree, positions_sorted: np.ndarray,
                          max_leaf_size: Optional[int] = None) -> OracleGeometry:
    """``geometry.py:17-75`` -> ``_geometry_impl.py:176-338``."""
    lib = _load()
    total = tree.node_ranges.shape[0]
    if max_leaf_size is None and tree.leaf_size is not None:
        max_leaf_size = int(tree.leaf_size)
    cap = -1 if max_leaf_size is None else int(max_leaf_size)
    pos = np.ascontiguousarray(positions_sorted, np.float32)
    ranges = np.ascontiguousarray(tree.node_ranges, np.int64)
    left = np.ascontiguousarray(tree.left_child, np.int64)
    right = np.ascontiguousarray(tree.right_child, np.int64)
    parent = np.ascontiguousarray(tree.parent, np.int64)
    g = OracleGeometry(np.empty((total, 3), np.float32), np.empty((total, 3), np.float32),
                       np.empty(total, np.float32), np.empty(total, np.float32))
    rc = lib.ygo_geometry(_p(ranges), ctypes.c_int64(total), _p(left), _p(right), _p(parent),
                          _p(pos), ctypes.c_int64(pos.shape[0]),
                          ctypes.c_int(1 if tree.use_morton_geometry else 0),
                          _p(np.asarray(tree.bounds_min, np.float32)),
                          _p(np.asarray(tree.bounds_max, np.float32)),
                          _p(np.ascontiguousarray(tree.leaf_codes, np.uint64)),
                          _p(np.ascontiguousarray(tree.leaf_depths, np.int64)),
                          ctypes.c_int64(cap), _p(g.center), _p(g.half_extent), _p(g.radius),
                          _p(g.max_extent))
    if rc != 0:
        raise RuntimeError("geometry depth pass did not converge (cyclic parent array)")
    return g


# ---------------------------------------------------------------------------
# L3 traversal


def mac_extents(tree: OracleTree, geom: OracleGeometry, mac_type: str,
                dehnen_radius_scale: float = 1.0) -> np.ndarray:
    """``_interactions_impl.py:993-1061`` (_build_mac_extents).

    Propagation and leaf depth padding only touch extents <= 0; with
    ``half >= 1e-6`` every extent is positive, which this restatement
    requires (it raises otherwise)."""
    ext = np.asarray(geom.max_extent if mac_type == "bh" else geom.radius, np.float32)
    if not np.all(ext > 0):
        raise NotImplementedError("non-positive MAC extents are outside the restated path")
    if mac_type == "dehnen":
        ext = (np.float32(dehnen_radius_scale) * ext).astype(np.float32)
    return np.ascontiguousarray(ext, np.float32)


def leaf_ordering(tree: OracleTree):
    """``_interactions_impl.py:1071-1103`` (_resolve_leaf_ordering)."""
    total = tree.node_ranges.shape[0]
    ni = tree.num_internal_nodes
    L = total - ni
    po = np.arange(ni, total, dtype=np.int64)
    native = np.arange(L, dtype=np.int64)
    if tree.octree is not None:
        native = np.argsort(tree.octree["radix_leaf_to_oct"], kind="stable").astype(np.int64)
    leaf_indices = po[native]
    po_to_native = np.zeros(L, np.int64)
    po_to_native[native] = np.arange(L, dtype=np.int64)
    leaf_position = np.full(total, -1, np.int64)
    leaf_position[leaf_indices] = np.arange(L, dtype=np.int64)
    return leaf_indices, leaf_position, po, po_to_native


_MAC_CODES = {"bh": 0, "dehnen": 1, "engblom": 2}


def build_interactions_and_neighbors(tree: OracleTree, geom: OracleGeometry, theta: float = 0.5,
                                     mac_type: str = "bh",
                                     dehnen_radius_scale: float = 1.0) -> dict:
    """Exact far/near lists of ``build_interactions_and_neighbors``
    (``_interactions_impl.py:6031-6144``) with canonical row order."""
    lib = _load()
    total = tree.node_ranges.shape[0]
    ni = tree.num_internal_nodes
    L = total - ni
    leaf_indices, leaf_position, po, po_to_native = leaf_ordering(tree)
    out = dict(leaf_indices=leaf_indices, particle_order_leaf_indices=po,
               particle_order_to_native_leaf=po_to_native)
    theta_sq = np.float32(theta) * np.float32(theta)
    if ni == 0:
        out.update(far_counts=np.zeros(total, np.int64),
                   offsets=np.zeros(total + 1, np.int64), sources=np.zeros(0, np.int64),
                   targets=np.zeros(0, np.int64), near_counts=np.zeros(L, np.int64),
                   near_offsets=np.zeros(L + 1, np.int64), neighbors=np.zeros(0, np.int64),
                   accept_decisions=0, near_decisions=0, refine_decisions=0, max_wf=1,
                   generations=0)
        out["level_offsets"] = np.zeros(int(tree.num_levels) + 1, np.int64)
        out["target_levels"] = np.zeros(0, np.int64)
        return out
    ext = mac_extents(tree, geom, mac_type, dehnen_radius_scale)
    center = np.ascontiguousarray(geom.center, np.float32)
    left = np.concatenate([tree.left_child, np.full(L, -1, np.int64)]).astype(np.int64)
    right = np.concatenate([tree.right_child, np.full(L, -1, np.int64)]).astype(np.int64)
    root = int(np.argmin(tree.parent))
    h = lib.ygo_walk(_p(center), _p(ext), _p(left), _p(right), ctypes.c_int64(total),
                     ctypes.c_int64(ni), ctypes.c_float(theta_sq), ctypes.c_int(_MAC_CODES[mac_type]),
                     ctypes.c_int64(root))
    try:
        sizes = np.zeros(7, np.int64)
        lib.ygo_walk_sizes(h, _p(sizes))
        P, Q = int(sizes[0]), int(sizes[1])
        far_counts = np.empty(total, np.int64)
        offsets = np.empty(total + 1, np.int64)
        sources = np.empty(2 * P, np.int64)
        targets = np.empty(2 * P, np.int64)
        near_counts = np.empty(L, np.int64)
        near_offsets = np.empty(L + 1, np.int64)
        neighbors = np.empty(2 * Q, np.int64)
        nbl = np.ascontiguousarray(tree.nodes_by_level, np.int64)
        lib.ygo_walk_lists(h, ctypes.c_int64(total), _p(nbl), _p(leaf_position),
                           ctypes.c_int64(L), _p(far_counts), _p(offsets), _p(sources),
                           _p(targets), _p(near_counts), _p(near_offsets), _p(neighbors))
    finally:
        lib.ygo_walk_free(h)
    num_levels = int(tree.num_levels)
    lvl_idx = np.asarray(tree.level_offsets[: num_levels + 1], np.int64)
    counts_by_level = far_counts[nbl]
    offsets_by_level = np.concatenate([[0], np.cumsum(counts_by_level)]).astype(np.int64)
    out.update(
        far_counts=far_counts, offsets=offsets, sources=sources, targets=targets,
        level_offsets=offsets_by_level[lvl_idx] if P else np.zeros(num_levels + 1, np.int64),
        target_levels=np.asarray(tree.node_level, np.int64)[targets],
        near_counts=near_counts, near_offsets=near_offsets, neighbors=neighbors,
        accept_decisions=int(sizes[2]), near_decisions=int(sizes[3]),
        refine_decisions=int(sizes[4]), max_wf=int(sizes[5]), generations=int(sizes[6]))
    if P == 0:
        out["offsets"] = np.zeros(total + 1, np.int64)
    return out


def neighbor_leaf_positions(leaf_indices, near_offsets, near_counts, neighbors, total):
    """Dense helper of ``_result_to_neighbors`` (``_interactions_impl.py:3658-3688``)."""
    L = leaf_indices.shape[0]
    if L == 0:
        return np.zeros((0, 0), np.int64)
    max_nbr = int(near_counts.max()) if L else 0
    if max_nbr == 0:
        return np.zeros((L, 0), np.int64)
    lookup = np.full(total, -1, np.int64)
    lookup[leaf_indices] = np.arange(L, dtype=np.int64)
    k = np.arange(max_nbr, dtype=np.int64)
    idx = near_offsets[:-1, None] + k[None, :]
    valid = k[None, :] < near_counts[:, None]
    safe = np.where(valid, idx, 0)
    pos = lookup[neighbors[safe]] if neighbors.size else np.zeros_like(safe)
    return np.where(valid, pos, -1)


def dual_tree_walk_mutual(left_full, right_full, centers, radii, theta, root, *,
                          max_pair_queue: int, far_cap: int, near_cap: int) -> dict:
    """Restatement of ``dual_tree_walk_mutual`` (_interactions_impl.py:6357-6560)
    in NumPy, generation by generation: fp32 MAC ``theta^2 * d^2 > (r_a +
    r_b)^2`` with ``d`` = centers[b] - centers[a] summed in written order
    (:6480-6486), accept / near / refine (:6487-6494), ``_flat_append``
    (:6339-6354) for the far and near lists, split rule (:6503-6506),
    children in ``_count_refine_pairs_single`` order (:174-221) canonicalised
    and compacted in wavefront order (:6524-6545)."""
    left = np.asarray(left_full, np.int64)
    right = np.asarray(right_full, np.int64)
    c = np.asarray(centers, np.float32)
    r = np.asarray(radii, np.float32)
    theta_sq = np.float32(theta) * np.float32(theta)
    Q = int(max_pair_queue)
    cur_a = np.array([int(root)], np.int64)
    cur_b = np.array([int(root)], np.int64)
    far = [np.full(far_cap, -1, np.int64), np.full(far_cap, -1, np.int64)]
    near = [np.full(near_cap, -1, np.int64), np.full(near_cap, -1, np.int64)]
    far_n = near_n = 0
    fo = no = qo = False

    def append(buf, n, cap, mask, a, b):
        k = np.nonzero(mask)[0]
        slots = n + np.arange(k.shape[0])
        ok = slots < cap
        buf[0][slots[ok]] = a[k[ok]]
        buf[1][slots[ok]] = b[k[ok]]
        return n + k.shape[0], bool((~ok).any())

    while cur_a.shape[0] > 0 and not (fo or no or qo):
        sa, sb = cur_a, cur_b
        a_leaf, b_leaf = left[sa] < 0, left[sb] < 0
        same = sa == sb
        d = c[sb] - c[sa]
        d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        ra, rb = r[sa], r[sb]
        rs = ra + rb
        accept = ~same & (theta_sq * d2 > rs * rs)
        both_leaf = a_leaf & b_leaf
        is_near = ~accept & both_leaf & ~same
        refine = ~accept & ~both_leaf
        far_n, f1 = append(far, far_n, far_cap, accept, sa, sb)
        near_n, n1 = append(near, near_n, near_cap, is_near, sa, sb)
        fo, no = fo or f1, no or n1
        split_a = refine & ~a_leaf & (same | b_leaf | (ra >= rb))
        split_b = refine & ~b_leaf & (same | a_leaf | (rb > ra))
        both = split_a & split_b
        only_a = split_a & ~both
        only_b = split_b & ~both
        al, ar, bl, br = left[sa], right[sa], left[sb], right[sb]
        ca = np.full((sa.shape[0], 4), -1, np.int64)
        cb = np.full((sa.shape[0], 4), -1, np.int64)
        m = only_b
        ca[m, 0], cb[m, 0], ca[m, 1], cb[m, 1] = sa[m], bl[m], sa[m], br[m]
        m = only_a
        ca[m, 0], cb[m, 0], ca[m, 1], cb[m, 1] = al[m], sb[m], ar[m], sb[m]
        m = both & ~same
        ca[m, 0], cb[m, 0], ca[m, 1], cb[m, 1] = al[m], bl[m], al[m], br[m]
        ca[m, 2], cb[m, 2], ca[m, 3], cb[m, 3] = ar[m], bl[m], ar[m], br[m]
        m = both & same
        ca[m, 0], cb[m, 0], ca[m, 1], cb[m, 1] = al[m], al[m], al[m], ar[m]
        ca[m, 2], cb[m, 2] = ar[m], ar[m]
        pa, pb = ca.reshape(-1), cb.reshape(-1)
        valid = (pa >= 0) & (pb >= 0)
        pa, pb = pa[valid], pb[valid]
        if pa.shape[0] > Q:
            qo = True
            pa, pb = pa[:Q], pb[:Q]
        cur_a, cur_b = np.minimum(pa, pb), np.maximum(pa, pb)
    return dict(far_a=far[0], far_b=far[1], far_count=far_n, near_a=near[0], near_b=near[1],
                near_count=near_n, far_overflow=fo, near_overflow=no, queue_overflow=qo)


def level_major_geometry(nodes_by_level, level_offsets, num_levels: int, center, half_extent,
                         radius, max_extent) -> dict:
    """geometry_to_level_major (_geometry_impl.py:342-420): (num_levels,
    max_nodes) buffers, row l = level l's nodes in nodes_by_level order, zero
    (node index -1) past the level's count; max_nodes = max(counts, 1)."""
    lo = np.asarray(level_offsets, np.int64)
    nbl = np.asarray(nodes_by_level, np.int64)
    counts = (lo[1:] - lo[:-1])[:num_levels]
    M = int(np.maximum(counts, 1).max())
    idx = np.full((num_levels, M), -1, np.int64)
    for lv in range(num_levels):
        idx[lv, :counts[lv]] = nbl[lo[lv]:lo[lv] + counts[lv]]
    ok = idx >= 0
    safe = np.where(ok, idx, 0)

    def take(a, zero_shape):
        v = np.asarray(a)[safe]
        return np.where(ok.reshape(ok.shape + (1,) * (v.ndim - 2)), v, 0).astype(np.float32)

    return dict(centers=take(center, 3), half_extents=take(half_extent, 3),
                radii=take(radius, 0), max_extents=take(max_extent, 0), level_counts=counts,
                node_indices=idx)


def dense_m2l(node_indices, counts, offsets, sources, center) -> dict:
    """_dense_m2l_buffers (dense_interactions.py:34-146): slot (l, m) of node
    n gets its far row's sources (-1 past the count), the mask, the count and
    centre[n] - centre[source] in fp32 (zero where masked)."""
    idx = np.asarray(node_indices, np.int64)
    cnt = np.asarray(counts, np.int64)
    off = np.asarray(offsets, np.int64)
    srcs = np.asarray(sources, np.int64)
    if srcs.size == 0:
        srcs = np.zeros(1, np.int64)
    c = np.asarray(center, np.float32)
    K = max(1, int(cnt.max()) if cnt.size else 0)
    live = idx >= 0
    n = np.where(live, idx, 0)
    slot_cnt = np.where(live, cnt[n], 0)
    k = np.arange(K)[None, None, :]
    valid = k < slot_cnt[..., None]
    row = np.where(valid, srcs[np.where(valid, off[n][..., None] + k, 0)], -1)
    safe = np.clip(row, 0, c.shape[0] - 1)
    disp = c[n][:, :, None, :] - c[safe]
    disp = np.where(valid[..., None], disp, np.float32(0)).astype(np.float32)
    return dict(m2l_sources=row, m2l_mask=valid, m2l_counts=slot_cnt, m2l_displacements=disp)


def grouped_from_pairs(sources, targets, node_level, center, bounds_min, bounds_max) -> dict:
    """build_grouped_interactions_from_pairs (grouped_interactions.py:75-200):
    float64 displacement indices rint((c_t - c_s) / max(extent / max(2^lt, 1),
    1e-12)), keys (lt, ls, dx, dy, dz) ordered stably, classes = runs of equal
    keys, class displacement key * cell in float64 cast to float32; class
    ids as the reference's searchsorted gives them (see below)."""
    src = np.asarray(sources, np.int64)
    tgt = np.asarray(targets, np.int64)
    c = np.asarray(center, np.float64)
    lev = np.asarray(node_level, np.int32)
    ext = np.asarray(bounds_max, np.float64) - np.asarray(bounds_min, np.float64)

    def cell(level):
        denom = np.power(2.0, level.astype(np.float64))[:, None]
        return np.maximum(ext[None, :] / np.maximum(denom, 1.0), 1e-12)

    tl, sl = lev[tgt], lev[src]
    disp = np.rint((c[tgt] - c[src]) / cell(tl)).astype(np.int32)
    keys = np.stack([tl, sl, disp[:, 0], disp[:, 1], disp[:, 2]], 1).astype(np.int32)
    order = np.lexsort((keys[:, 4], keys[:, 3], keys[:, 2], keys[:, 1], keys[:, 0]))
    ks = keys[order]
    head = np.ones(ks.shape[0], bool)
    head[1:] = (ks[1:] != ks[:-1]).any(1)
    starts = np.nonzero(head)[0]
    # np.searchsorted(class_starts, arange(n)) with side="left" (:163): a pair
    # that is not the first of its class gets the NEXT class's id -- a quirk
    # of the reference, reproduced
    incl = np.cumsum(head)
    ids_sorted = np.where(head, incl - 1, incl)
    ids = np.empty_like(ids_sorted)
    ids[order] = ids_sorted
    ck = ks[starts]
    cdisp = (ck[:, 2:5].astype(np.float64) * cell(ck[:, 0])).astype(np.float32)
    return dict(class_keys=ck, class_displacements=cdisp,
                class_offsets=np.concatenate([starts, [ks.shape[0]]]).astype(np.int64),
                class_sources=src[order], class_targets=tgt[order], class_ids=ids.astype(np.int64))


def _combos(order: int):
    """multi_index_tuples(0..order) concatenated (multipole_utils.py)."""
    out = []
    for lv in range(order + 1):
        for i in range(lv + 1):
            for j in range(lv + 1 - i):
                out.append((i, j, lv - i - j))
    return out


def tree_mass_moments(node_ranges, positions_sorted, masses_sorted):
    """compute_tree_mass_moments (tree_moments.py:686-744): fp32 prefix sums
    of the masses and mass-weighted positions, differenced at each node's
    range; centre = weighted sum / mass (0 for a massless node)."""
    r = np.asarray(node_ranges, np.int64)
    st, en = r[:, 0], r[:, 1] + 1
    p = np.asarray(positions_sorted, np.float32)
    m = np.asarray(masses_sorted, np.float32)
    mp = np.concatenate([np.zeros(1, np.float32), np.cumsum(m)])
    wp = np.concatenate([np.zeros((1, 3), np.float32), np.cumsum(m[:, None] * p, axis=0)])
    tot = mp[en] - mp[st]
    mom = wp[en] - wp[st]
    safe = np.where(tot == 0, np.ones_like(tot), tot)
    ctr = np.where(tot[:, None] == 0, np.float32(0), mom / safe[:, None])
    return tot, ctr


def tree_multipole_moments(node_ranges, positions_sorted, masses_sorted, expansion_centers=None,
                           max_order: int = 2) -> dict:
    """compute_tree_multipole_moments (tree_moments.py:747-877) and the
    tensors of _moments_from_raw_packed (:312-395): fp32 cumprod powers,
    monomials x^a y^b z^c weighted by mass, prefix sums differenced at the
    node ranges, the binomial shift to the expansion centre (einsum over the
    stencil), then the symmetric second..fourth moments and their trace-free
    quadrupole / octupole / hexadecapole, zero for massless nodes."""
    tot, com = tree_mass_moments(node_ranges, positions_sorted, masses_sorted)
    center = com if expansion_centers is None else np.asarray(expansion_centers, np.float32)
    order = int(max_order)
    p = np.asarray(positions_sorted, np.float32)
    m = np.asarray(masses_sorted, np.float32)
    r = np.asarray(node_ranges, np.int64)
    st, en = r[:, 0], r[:, 1] + 1
    cb = np.asarray(_combos(order), np.int64)
    C = cb.shape[0]

    def axis_powers(v):
        base = np.asarray(v, np.float32)[:, None]
        ones = np.ones_like(base)
        if order == 0:
            return ones
        return np.cumprod(np.concatenate([ones, np.repeat(base, order, axis=1)], axis=1), axis=1)

    ax, ay, az = axis_powers(p[:, 0]), axis_powers(p[:, 1]), axis_powers(p[:, 2])
    mono = ax[:, cb[:, 0]] * ay[:, cb[:, 1]] * az[:, cb[:, 2]]
    w = m[:, None] * mono
    pre = np.concatenate([np.zeros((1, C), np.float32), np.cumsum(w, axis=0)], axis=0)
    raw = pre[en] - pre[st]
    neg = -center
    cx, cy, cz = axis_powers(neg[:, 0]), axis_powers(neg[:, 1]), axis_powers(neg[:, 2])
    full = np.asarray(_combos(4), np.int64)
    T = full.shape[0]
    gamma = np.zeros((T, T, 3), np.int64)
    mask = np.zeros((T, T), bool)
    binom = np.zeros((T, T), np.float64)
    for i in range(T):
        for j in range(T):
            if (full[i] >= full[j]).all():
                mask[i, j] = True
                gamma[i, j] = full[i] - full[j]
                binom[i, j] = (math.comb(*[int(x) for x in (full[i, 0], full[j, 0])])
                               * math.comb(int(full[i, 1]), int(full[j, 1]))
                               * math.comb(int(full[i, 2]), int(full[j, 2])))
    g = np.where(mask[:C, :C, None], gamma[:C, :C], 0)
    cf = (np.take(cx, g[..., 0], axis=1) * np.take(cy, g[..., 1], axis=1)
          * np.take(cz, g[..., 2], axis=1))
    transform = cf * mask[:C, :C].astype(np.float32)[None] * binom[:C, :C].astype(np.float32)[None]
    packed = np.einsum("nij,nj->ni", transform, raw)
    return _tensors_from_packed(packed, center, order)


def _tensors_from_packed(packed, center, order: int) -> dict:
    n = packed.shape[0]
    look = {c: k for k, c in enumerate(_combos(order))}
    mass = packed[:, 0]
    dt = packed.dtype
    dip = np.zeros((n, 3), dt)
    if order >= 1:
        dip[:, 0], dip[:, 1], dip[:, 2] = (packed[:, look[(1, 0, 0)]], packed[:, look[(0, 1, 0)]],
                                           packed[:, look[(0, 0, 1)]])
    sec = np.zeros((n, 3, 3), dt)
    thr = np.zeros((n, 3, 3, 3), dt)
    fou = np.zeros((n, 3, 3, 3, 3), dt)

    def combo_of(*axes):
        c = [0, 0, 0]
        for a in axes:
            c[a] += 1
        return tuple(c)

    import itertools as it
    if order >= 2:
        for i, j in it.product(range(3), repeat=2):
            sec[:, i, j] = packed[:, look[combo_of(i, j)]]
    if order >= 3:
        for i, j, k in it.product(range(3), repeat=3):
            thr[:, i, j, k] = packed[:, look[combo_of(i, j, k)]]
    if order >= 4:
        for i, j, k, l in it.product(range(3), repeat=4):
            fou[:, i, j, k, l] = packed[:, look[combo_of(i, j, k, l)]]
    trace = np.trace(sec, axis1=-2, axis2=-1)
    quad = dt.type(3.0) * sec - trace[:, None, None] * np.eye(3, dtype=dt)
    octu = np.zeros_like(thr)
    if order >= 3:
        r2rk = np.stack([thr[:, 0, 0, k] + thr[:, 1, 1, k] + thr[:, 2, 2, k] for k in range(3)], -1)
        for i, j, k in it.product(range(3), repeat=3):
            v = dt.type(5.0) * thr[:, i, j, k]
            if i == j:
                v = v - r2rk[:, k]
            if i == k:
                v = v - r2rk[:, j]
            if j == k:
                v = v - r2rk[:, i]
            octu[:, i, j, k] = v
    hexa = np.zeros_like(fou)
    if order >= 4:
        r2 = fou[:, 0, 0] + fou[:, 1, 1] + fou[:, 2, 2]
        r4 = (fou[:, 0, 0, 0, 0] + fou[:, 1, 1, 1, 1] + fou[:, 2, 2, 2, 2]
              + dt.type(2.0) * (fou[:, 0, 0, 1, 1] + fou[:, 0, 0, 2, 2] + fou[:, 1, 1, 2, 2]))
        for i, j, k, l in it.product(range(3), repeat=4):
            v = dt.type(35.0) * fou[:, i, j, k, l]
            term = np.zeros_like(v)
            for cond, (a, b) in ((i == j, (k, l)), (i == k, (j, l)), (i == l, (j, k)),
                                 (j == k, (i, l)), (j == l, (i, k)), (k == l, (i, j))):
                if cond:
                    term = term + r2[:, a, b]
            v = v - dt.type(5.0) * term
            df = int(i == j and k == l) + int(i == k and j == l) + int(i == l and j == k)
            if df:
                v = v + r4 * df
            hexa[:, i, j, k, l] = v
    z = mass == 0
    return dict(mass=mass, center=center, dipole=np.where(z[:, None], 0, dip).astype(dt),
                second_moment=np.where(z[:, None, None], 0, sec).astype(dt),
                quadrupole=np.where(z[:, None, None], 0, quad).astype(dt),
                third_moment=np.where(z[:, None, None, None], 0, thr).astype(dt),
                octupole=np.where(z[:, None, None, None], 0, octu).astype(dt),
                fourth_moment=np.where(z[:, None, None, None, None], 0, fou).astype(dt),
                hexadecapole=np.where(z[:, None, None, None, None], 0, hexa).astype(dt),
                raw_packed=packed)


# ---------------------------------------------------------------------------
# Native octree walk (octree node space)


def _compact3_np(x: np.ndarray) -> np.ndarray:
    """Every third bit of a uint64 (the inverse of the Morton spread,
    ``morton.py:32-39``), by the standard mask-and-shift compaction."""
    x = np.asarray(x, np.uint64) & np.uint64(0x1249249249249249)
    for sh, m in ((2, 0x10C30C30C30C30C3), (4, 0x100F00F00F00F00F), (8, 0x001F0000FF0000FF),
                  (16, 0x001F00000000FFFF), (32, 0x00000000001FFFFF)):
        x = (x ^ (x >> np.uint64(sh))) & np.uint64(m)
    return x


def octree_box_geometry(valid_mask, node_codes, node_depths, bounds_min, bounds_max) -> dict:
    """``octree.py:422-476`` (compute_explicit_octree_box_geometry) in fp32,
    each operation rounded: cell = domain / 2^depth, mins = bmin + cell *
    index, maxs = mins + cell, centres 0.5 (mins + maxs), half extents
    0.5 (maxs - mins), radius sqrt((h0^2 + h1^2) + h2^2), max extent max(h);
    zeros on invalid slots."""
    bmin = np.asarray(bounds_min, np.float32)
    dom = (np.asarray(bounds_max, np.float32) - bmin).astype(np.float32)
    d = np.clip(np.asarray(node_depths, np.int64), 0, 21)
    sh = (21 - d).astype(np.uint64)
    codes = np.asarray(node_codes, np.uint64)
    idx = np.stack([_compact3_np(codes) >> sh, _compact3_np(codes >> np.uint64(1)) >> sh,
                    _compact3_np(codes >> np.uint64(2)) >> sh], axis=1).astype(np.float32)
    cnt = np.maximum(np.left_shift(np.uint64(1), d.astype(np.uint64)), np.uint64(1))
    cell = (dom[None, :] / cnt.astype(np.float32)[:, None]).astype(np.float32)
    mins = (bmin[None, :] + (cell * idx).astype(np.float32)).astype(np.float32)
    maxs = (mins + cell).astype(np.float32)
    centers = (np.float32(0.5) * (mins + maxs)).astype(np.float32)
    half = (np.float32(0.5) * (maxs - mins)).astype(np.float32)
    s = (half[:, 0] * half[:, 0] + half[:, 1] * half[:, 1]).astype(np.float32)
    s = (s + half[:, 2] * half[:, 2]).astype(np.float32)
    radii = np.sqrt(s).astype(np.float32)
    maxe = np.max(half, axis=1).astype(np.float32)
    v = np.asarray(valid_mask, bool)
    centers[~v] = 0.0
    half[~v] = 0.0
    radii[~v] = 0.0
    maxe[~v] = 0.0
    return dict(centers=centers, half_extents=half, radii=radii, max_extents=maxe)


def octree_traversal_view(oct_fields: dict, num_internal: int, bounds_min, bounds_max) -> dict:
    """``octree.py:577-704`` (build_explicit_octree_traversal_view): the oct
    tables, the smallest radix node / leaf id carried by each oct cell
    (-1 where none, or where the cell is invalid / not a leaf), and the box
    geometry."""
    o = {k: np.asarray(v) for k, v in oct_fields.items()}
    valid = o["oct_valid_mask"].astype(bool)
    leaf = o["oct_leaf_mask"].astype(bool)
    M = valid.shape[0]
    r2o = o["radix_node_to_oct"].astype(np.int64)
    fill = r2o.shape[0]
    o2r = np.full(M, fill, np.int64)
    np.minimum.at(o2r, r2o, np.arange(fill, dtype=np.int64))
    o2r = np.where(valid & (o2r < fill), o2r, -1)
    l2o = o["radix_leaf_to_oct"].astype(np.int64)
    lfill = num_internal + l2o.shape[0]
    o2l = np.full(M, lfill, np.int64)
    np.minimum.at(o2l, l2o, np.arange(num_internal, lfill, dtype=np.int64))
    o2l = np.where(leaf & (o2l < lfill), o2l, -1)
    box = octree_box_geometry(valid, o["oct_node_codes"], o["oct_node_depths"], bounds_min,
                              bounds_max)
    return dict(o, oct_to_radix_node=o2r, oct_to_radix_leaf=o2l, box=box)


def octree_native_walk(view: dict, theta: float, mac_type: str = "bh", *,
                       dehnen_radius_scale: float = 1.0, collect_far: bool, collect_near: bool,
                       max_interactions_per_node: int, max_neighbors_per_leaf: int,
                       max_pair_queue: int) -> dict:
    """``_dual_tree_walk_octree_impl`` (_interactions_impl.py:1908-2597) with
    far rows in octree node space (the far-pairs entry point) and near rows
    in octree leaf space (the neighbour-list entry point, whose "leaves" are
    the cells that carry a radix leaf, ``:1958-1981``).

    Per generation: box-centre distance and MAC (:338-395) on the box radius
    (dehnen / engblom, dehnen scaled) or box max extent (bh); accept / near /
    refine (:713-728) with the leaf test of the node space in use; split
    rule (:2247-2257); children from ``_octree_refine_pairs_single`` (:106-
    165), which takes the first ``child_count`` of the eight octant slots
    (slots holding -1 are dropped at the push, :2432-2436), canonicalised
    and compacted in wavefront order.  Accepted pairs go to row t then row s
    (fwd block then bwd block of the generation, :2243-2300); the reference
    orders entries of one row within a block by an unstable argsort
    (:813-873), this restatement keeps wavefront order.  The walk stops after
    a generation whose pushes exceed the queue or whose row counts exceed a
    capacity (:2113-2131).  The effective-extent propagation (:876-990)
    leaves positive extents unchanged; valid cells always have positive
    boxes."""
    ch = np.asarray(view["oct_children"], np.int64)
    cc = np.asarray(view["oct_child_counts"], np.int64)
    parent = np.asarray(view["oct_parent"], np.int64)
    M = parent.shape[0]
    box = view["box"]
    c = box["centers"]
    use_sphere = mac_type in ("dehnen", "engblom")
    ext = (box["radii"] if use_sphere else box["max_extents"]).astype(np.float32)
    if mac_type == "dehnen":
        ext = (np.float32(dehnen_radius_scale) * ext).astype(np.float32)
    if collect_near:
        carrier = np.zeros(M, bool)
        carrier[np.asarray(view["radix_leaf_to_oct"], np.int64)] = True
        leaf_mask = carrier
        nz = np.nonzero(carrier)[0]
        L = np.asarray(view["radix_leaf_to_oct"]).shape[0]
        leaf_indices = np.full(L, -1, np.int64)
        leaf_indices[:nz.shape[0]] = nz
        leaf_pos = np.full(M, -1, np.int64)
        leaf_pos[nz] = np.arange(nz.shape[0])
    else:
        leaf_mask = np.asarray(view["oct_leaf_mask"], bool)
        leaf_indices = None
        leaf_pos = None
    theta_sq = np.float32(theta) * np.float32(theta)
    theta32 = np.sqrt(theta_sq).astype(np.float32)
    Q = max(int(max_pair_queue), 4)
    root = int(np.argmin(parent))
    wt = np.array([root], np.int64)
    ws = np.array([root], np.int64)
    far_rows = [[] for _ in range(M)] if collect_far else None
    n_rows = leaf_indices.shape[0] if collect_near else 0
    near_rows = [[] for _ in range(n_rows)] if collect_near else None
    far_cnt = np.zeros(M, np.int64)
    near_cnt = np.zeros(n_rows, np.int64)
    wo = fo = no = False
    acc = nea = ref = 0
    gens = 0
    slots = np.arange(8)
    while wt.shape[0] > 0 and not (wo or fo or no):
        gens += 1
        t, s = wt, ws
        d = (c[t] - c[s]).astype(np.float32)
        d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]).astype(np.float32)
        d2 = (d2 + d[:, 2] * d[:, 2]).astype(np.float32)
        et, es = ext[t], ext[s]
        diff = t != s
        if mac_type == "engblom":
            big, small = np.maximum(et, es), np.minimum(et, es)
            lhs = (big + theta32 * small).astype(np.float32)
            ok = (lhs * lhs).astype(np.float32) <= (theta_sq * d2).astype(np.float32)
        else:
            sm = (et + es).astype(np.float32)
            ok = (sm * sm).astype(np.float32) <= (theta_sq * d2).astype(np.float32)
        mac_ok = diff & (d2 > 0) & ok
        tl, sl = leaf_mask[t], leaf_mask[s]
        accept = mac_ok
        near = ~mac_ok & tl & sl & diff
        refine = ~accept & ~near
        acc += int(accept.sum())
        nea += int(near.sum())
        ref += int(refine.sum())
        same = ~diff
        split_t = refine & ~tl & (same | sl | (et >= es))
        split_s = refine & ~sl & (same | tl | (es > et))
        if collect_far:
            k = np.nonzero(accept)[0]
            for i in k:  # fwd block
                far_rows[t[i]].append(s[i])
            for i in k:  # bwd block
                far_rows[s[i]].append(t[i])
            np.add.at(far_cnt, t[k], 1)
            np.add.at(far_cnt, s[k], 1)
            if k.shape[0] and far_cnt.max() > max_interactions_per_node:
                fo = True
        if collect_near:
            k = np.nonzero(near)[0]
            pt, ps = leaf_pos[t[k]], leaf_pos[s[k]]
            for j, i in enumerate(k):
                near_rows[pt[j]].append(s[i])
            for j, i in enumerate(k):
                near_rows[ps[j]].append(t[i])
            np.add.at(near_cnt, pt, 1)
            np.add.at(near_cnt, ps, 1)
            if k.shape[0] and near_cnt.max() > max_neighbors_per_leaf:
                no = True
        pa, pb = [], []
        for i in np.nonzero(split_t | split_s)[0]:
            ti, si = t[i], s[i]
            if split_t[i] and split_s[i]:
                if same[i]:
                    for a in range(cc[ti]):
                        for b in range(a, cc[ti]):
                            pa.append(ch[ti, a]); pb.append(ch[ti, b])
                else:
                    for a in range(cc[ti]):
                        for b in range(cc[si]):
                            pa.append(ch[ti, a]); pb.append(ch[si, b])
            elif split_t[i]:
                for a in range(cc[ti]):
                    pa.append(ch[ti, a]); pb.append(si)
            else:
                for b in range(cc[si]):
                    pa.append(ti); pb.append(ch[si, b])
        pa = np.asarray(pa, np.int64)
        pb = np.asarray(pb, np.int64)
        keep = (pa >= 0) & (pb >= 0)
        pa, pb = pa[keep], pb[keep]
        if pa.shape[0] > Q:
            wo = True
            pa, pb = pa[:Q], pb[:Q]
        wt, ws = np.minimum(pa, pb), np.maximum(pa, pb)
    out = dict(queue_overflow=wo, far_overflow=fo, near_overflow=no, accept_decisions=acc,
               near_decisions=nea, refine_decisions=ref, generations=gens, root=root)
    if collect_far:
        nbl = np.asarray(view["oct_nodes_by_level"], np.int64)
        srcs = [np.asarray(far_rows[v], np.int64) for v in nbl]
        out["far_counts"] = far_cnt
        out["sources"] = np.concatenate(srcs) if srcs else np.zeros(0, np.int64)
        out["targets"] = np.repeat(nbl, far_cnt[nbl])
    if collect_near:
        out["near_counts"] = near_cnt
        out["neighbors"] = (np.concatenate([np.asarray(r, np.int64) for r in near_rows])
                            if n_rows else np.zeros(0, np.int64))
        out["leaf_indices"] = leaf_indices
    return out


def octree_native_neighbor_list(walk: dict, oct_node_ranges) -> dict:
    """``_raw_to_octree_native_neighbors`` (_interactions_impl.py:5411-5553)
    without target blocks: rows of the valid carrier cells, CSR offsets, the
    particle order of the carriers (stable by their first particle) and the
    dense (rows, max row) table of neighbour row positions (-1 padded)."""
    li = walk["leaf_indices"]
    keep = li >= 0
    leaf_indices = li[keep]
    counts = walk["near_counts"][keep]
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    ranges = np.asarray(oct_node_ranges, np.int64)
    order = np.argsort(ranges[np.clip(leaf_indices, 0, None), 0], kind="stable")
    po_to_native = np.zeros(leaf_indices.shape[0], np.int64)
    po_to_native[order] = np.arange(leaf_indices.shape[0])
    lookup = np.full(ranges.shape[0], -1, np.int64)
    lookup[leaf_indices] = np.arange(leaf_indices.shape[0])
    mx = int(counts.max()) if counts.shape[0] else 0
    pos = np.full((leaf_indices.shape[0], mx), -1, np.int64)
    nb = walk["neighbors"][: int(offsets[-1])]
    for r in range(leaf_indices.shape[0]):
        row = nb[offsets[r]:offsets[r + 1]]
        pos[r, :row.shape[0]] = lookup[row]
    return dict(offsets=offsets, neighbors=nb, leaf_indices=leaf_indices, counts=counts,
                particle_order_leaf_indices=leaf_indices[order],
                particle_order_to_native_leaf=po_to_native, neighbor_leaf_positions=pos)

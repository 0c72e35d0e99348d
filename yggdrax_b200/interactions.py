"""Dual-tree far/near interaction lists on the GPU.

Mirrors ``build_interactions_and_neighbors`` (yggdrax/interactions.py:338-448,
yggdrax/_interactions_impl.py:6031-6144) and its containers
(``_interactions_impl.py:235-242, 416-424, 566-644``).  The walk, the row
sizing and the level-major / CSR layouts run as sm_100a kernels
(``ygx_traverse_walk`` / ``_fill`` / ``_finalize``).

Output contract: the same pair sets and layouts as the reference; within
every row the entries are in ascending order (the reference's within-row
order comes from an unstable sort and is unspecified).  Capacity arguments
keep their meaning: with ``traversal_config`` / ``max_interactions_per_node``
/ ``max_pair_queue`` the reference's padded walk would fail on the same
inputs, so the same ``RuntimeError`` is raised; without them the exact
count-then-fill path is used, as in the reference.
"""

from __future__ import annotations

import logging
import os
from dataclasses import dataclass
from typing import Callable, Literal, NamedTuple, Optional

import numpy as np
import torch

from . import _lib as L
from .dtypes import INDEX_BITS, INDEX_DTYPE
from .tree import _dev_of, _host_of, resolve_tree_topology

logger = logging.getLogger(__name__)

_DEFAULT_MAX_INTERACTIONS = 512
_DEFAULT_MAX_NEIGHBORS = 2048
DEFAULT_PAIR_QUEUE_MULTIPLIER = 128
_DEFAULT_PAIR_BATCH = 32
_AUTO_INTERACTION_MIN = 2048
_AUTO_INTERACTION_MAX = 16384
_AUTO_INTERACTION_SCALE = 4
_INT32_MAX = (1 << 31) - 1

MACType = Literal["bh", "engblom", "dehnen"]
_MAC_CODES = {"bh": 0, "dehnen": 1, "engblom": 2}


@dataclass(frozen=True)
class DualTreeTraversalConfig:
    """Fixed traversal parameters for the dual-tree walk (:235-242)."""

    max_pair_queue: int
    process_block: int
    max_interactions_per_node: int
    max_neighbors_per_leaf: int = _DEFAULT_MAX_NEIGHBORS


_GLOBAL_DUAL_TREE_CONFIG: Optional[DualTreeTraversalConfig] = None


def set_default_dual_tree_config(config: Optional[DualTreeTraversalConfig]) -> None:
    """Module-level fallback configuration (:250-266)."""
    if config is not None:
        if config.max_pair_queue < 1:
            raise ValueError("max_pair_queue must be >= 1")
        if config.process_block < 1:
            raise ValueError("process_block must be >= 1")
        if config.max_interactions_per_node < 1:
            raise ValueError("max_interactions_per_node must be >= 1")
        if config.max_neighbors_per_leaf < 1:
            raise ValueError("max_neighbors_per_leaf must be >= 1")
    global _GLOBAL_DUAL_TREE_CONFIG
    _GLOBAL_DUAL_TREE_CONFIG = config


class DualTreeRetryEvent(NamedTuple):
    attempt: int
    queue_capacity: int
    interaction_capacity: int
    status: str
    far_pair_count: int
    near_pair_count: int


class NodeInteractionList(NamedTuple):
    """Far-field interactions in level-major order (:566-592)."""

    offsets: torch.Tensor
    sources: torch.Tensor
    targets: torch.Tensor
    counts: torch.Tensor
    level_offsets: torch.Tensor
    target_levels: torch.Tensor


class NodeNeighborList(NamedTuple):
    """Near-field neighbour CSR over leaves in native order (:595-609)."""

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


class DualTreeWalkResult(NamedTuple):
    """Raw walk payload (:612-631) in the exact count-then-fill layout."""

    interaction_offsets: torch.Tensor
    interaction_sources: torch.Tensor
    interaction_targets: torch.Tensor
    interaction_tags: torch.Tensor
    interaction_counts: torch.Tensor
    neighbor_offsets: torch.Tensor
    neighbor_indices: torch.Tensor
    neighbor_counts: torch.Tensor
    leaf_indices: torch.Tensor
    far_pair_count: torch.Tensor
    near_pair_count: torch.Tensor
    queue_overflow: torch.Tensor
    far_overflow: torch.Tensor
    near_overflow: torch.Tensor
    accept_decisions: torch.Tensor
    near_decisions: torch.Tensor
    refine_decisions: torch.Tensor


class CompactTaggedFarPairs(NamedTuple):
    sources: torch.Tensor
    targets: torch.Tensor
    tags: torch.Tensor
    far_pair_count: torch.Tensor


# ---------------------------------------------------------------------------
# Capacity ladders of the reference (used only to reproduce its errors)


def _next_power_of_two(value: int) -> int:
    value = max(1, int(value))
    return 1 << (value - 1).bit_length()


def _queue_candidates_bounded(*, max_capacity: int, process_block: int) -> list:
    """:296-316."""
    qmax = max(4, int(max_capacity))
    base = min(max(1024, int(process_block) * 16), qmax)
    cands = [base]
    while cands[-1] < qmax:
        nxt = min(qmax, cands[-1] * 2)
        if nxt == cands[-1]:
            break
        cands.append(nxt)
    return cands


def _auto_pair_queue_candidates(total_nodes: int, num_internal: int) -> list:
    """:450-485."""
    conservative = DEFAULT_PAIR_QUEUE_MULTIPLIER * max(4, total_nodes)
    start = min(max(4096, num_internal * 2), conservative)
    if start >= conservative:
        return [int(conservative)]
    cands = []
    cap = start
    while cap < conservative:
        cands.append(int(cap))
        cap = max(cap * 2, cap + 1024)
    cands.append(int(conservative))
    return list(dict.fromkeys(cands))


def _auto_interaction_capacity(total_nodes: int) -> int:
    """:516-537."""
    scaled = max(total_nodes // _AUTO_INTERACTION_SCALE, _AUTO_INTERACTION_MIN)
    scaled = min(scaled, _AUTO_INTERACTION_MAX)
    return int(min(_AUTO_INTERACTION_MAX, max(_AUTO_INTERACTION_MIN, _next_power_of_two(scaled))))


_REFERENCE_LIMITS = os.environ.get("YGGDRAX_B200_REFERENCE_LIMITS", "1").strip().lower() not in (
    "0", "false", "no", "off")


def set_reference_limits(enabled: bool) -> None:
    """Raise where the reference raises (default) or not.

    The reference sizes dense host/device buffers from the walk's counts and
    refuses to run when they would not fit: in count-then-fill mode it raises
    when the longest near row exceeds ``int32_max // num_leaves``
    (``_interactions_impl.py:4170-4187``), which every Plummer sphere above
    ~1.5M particles at leaf 32 triggers because its outermost halo leaf is near
    to every other leaf.  This implementation needs no dense buffers to
    produce the exact lists, so with ``enabled=False`` those checks are
    skipped and the lists are returned.  Environment:
    ``YGGDRAX_B200_REFERENCE_LIMITS=0``."""
    global _REFERENCE_LIMITS
    _REFERENCE_LIMITS = bool(enabled)


_DENSE_BUDGET: Optional[int] = None
_DENSE_WARNED: set = set()
LAST_WALK_STATS: dict = {}  # diagnostics of the most recent walk
# Capacity hints per (mac, theta): wavefront and pair-log entries per tree
# node that the last walk needed.  The next walk starts from them (with
# head-room) so a repeated workload sizes its buffers right the first time;
# a walk that overflows is re-run with the sizes it reports.
_CAPACITY_HINTS: dict = {}
# Generations of the last walk per (mac, theta): the walk checks its wavefront
# first after that many (one host sync instead of one per 16 generations).
_GENS_HINTS: dict = {}
# Largest wavefront a walk accepts (pair slots are 32-bit, with a block of
# head-room the kernels append into).
_WF_CAP_MAX = (1 << 32) - 4097


def _hint_key(mac_type: str, theta: float, total: int, kind: str = "tree") -> tuple:
    """Hints are kept per (mac, theta) and per octave of the tree size: the
    entries per node that a small tree needs say little about a large one
    (a few thousand nodes can need a hundred wavefront pairs per node)."""
    return (kind, mac_type, float(theta), int(total).bit_length())


def _grow_wf_cap(cap: int, stats) -> int:
    """Wavefront capacity for the re-run of a walk that overflowed it."""
    if cap >= _WF_CAP_MAX:
        raise L.YgxError("traversal wavefront exceeds 2^32 pairs")
    return min(_WF_CAP_MAX, max(cap * 4, 2 * int(stats[L.TSTAT["wf_need"]])))
_TIMING = os.environ.get("YGGDRAX_B200_TIMING", "0") == "1"  # per-pass CUDA-event times
TRAVERSAL_MODES = ("log", "two_pass", "learned", "target", "target_ordered")
_TRAVERSAL_MODE = os.environ.get("YGGDRAX_B200_TRAVERSAL_MODE", "learned")


def set_traversal_mode(mode: str) -> None:
    """How the exact lists are produced (all modes return identical lists):

    * ``"log"``: one walk that counts row entries and logs every accepted /
      near pair once, then a scatter of the log into the rows;
    * ``"two_pass"``: the reference's plain count-then-fill schedule, two
      walks (counts, then entries written at row cursors);
    * ``"learned"`` (default): the per-target walk below with every row given
      a slot sized by the learned capacity predictor
      (``yggdrax_b200.predictor``); the walk writes every chunk that fits in
      place, rows that outgrow their slot are completed from the rest (trees
      the per-target walk does not serve use the generation walk writing into
      predicted rows, completed from a log);
    * ``"target"``: one warp per target node walks that node's pairs
      (``ygx_target_walk``): the rows need no scatter, only a sort;
    * ``"target_ordered"``: the same walk in Morton order, so the rows come
      out in ascending order with no scatter and no row sort.

    Trees with tied leaf codes run the target modes as ``"log"``.

    Environment: ``YGGDRAX_B200_TRAVERSAL_MODE``."""
    global _TRAVERSAL_MODE
    if mode not in TRAVERSAL_MODES:
        raise ValueError(f"traversal mode must be one of {TRAVERSAL_MODES}, got {mode!r}")
    _TRAVERSAL_MODE = mode


def get_traversal_mode() -> str:
    """The schedule ``set_traversal_mode`` selected last."""
    return _TRAVERSAL_MODE


def set_dense_neighbor_budget(nbytes: Optional[int]) -> None:
    """Byte budget of the dense ``neighbor_leaf_positions`` helper table
    (``None``: a quarter of the device memory that is free at call time).
    The table is ``(num_leaves, max_neighbours)``; when one sparse leaf is
    near to nearly every other leaf it grows quadratically (terabytes for
    16M-particle Plummer spheres), so above the budget an empty ``(L, 0)``
    table is returned and the CSR ``offsets`` / ``neighbors`` stay exact."""
    global _DENSE_BUDGET
    _DENSE_BUDGET = None if nbytes is None else int(nbytes)


def _dense_neighbor_budget(dev) -> int:
    if _DENSE_BUDGET is not None:
        return _DENSE_BUDGET
    free, _ = torch.cuda.mem_get_info(dev)
    return int(free // 4)


_FAR_MSG = "Interaction list capacity exceeded; increase max_interactions_per_node and rebuild."
_NEAR_MSG = "Neighbor list capacity exceeded; increase max_neighbors_per_leaf and rebuild."


# ---------------------------------------------------------------------------


def _root_of(topology, d) -> int:
    """Node 0 unless tied leaf codes made the topology malformed (then the
    node without a parent, as the reference's walk starts there)."""
    if not _host_of(topology).malformed:
        return 0
    return int(torch.argmin(d.parent32).item())


def _leaf_ordering(topology, total: int, ni: int, dev):
    """_resolve_leaf_ordering (:1071-1103): native leaf order (stable order
    of radix_leaf_to_oct for octrees), leaf positions, inverse map."""
    nl = total - ni
    po = torch.arange(ni, total, dtype=INDEX_DTYPE, device=dev)
    if hasattr(topology, "radix_leaf_to_oct"):
        lib = L.lib()
        keys = topology.radix_leaf_to_oct.to(torch.int64).contiguous().view(torch.uint64)
        kout = torch.empty_like(keys)
        native = torch.empty(nl, dtype=torch.int32, device=dev)
        ws = L.workspace(lib.ygx_sort_pairs_workspace_size(nl), dev)
        L.check(lib.ygx_sort_pairs(L.ptr(keys), None, nl, 0, 32, L.ptr(kout), L.ptr(native),
                                   L.ptr(ws), ws.numel(), L.stream_handle(dev)),
                "ygx_sort_pairs")
        native = native.to(torch.int64)
    else:
        native = torch.arange(nl, dtype=torch.int64, device=dev)
    leaf_indices = po[native]
    po_to_native = torch.empty(nl, dtype=INDEX_DTYPE, device=dev)
    po_to_native[native] = torch.arange(nl, dtype=INDEX_DTYPE, device=dev)
    leafpos32 = torch.full((total,), -1, dtype=torch.int32, device=dev)
    leafpos32[leaf_indices.long()] = torch.arange(nl, dtype=torch.int32, device=dev)
    return leaf_indices, leafpos32, po, po_to_native


def _target_blocks(counts, offsets, nbr_leaf_pos, L_count, dev):
    """_build_target_blocks (:3690-3769); active only with
    YGGDRAX_NEARFIELD_TARGET_BLOCK_SIZE > 0."""
    raw = os.environ.get("YGGDRAX_NEARFIELD_TARGET_BLOCK_SIZE", "0")
    try:
        k = max(0, int(raw))
    except Exception:
        k = 0
    z = lambda *s, dt=INDEX_DTYPE: torch.zeros(s, dtype=dt, device=dev)  # noqa: E731
    if k <= 0 or L_count == 0:
        return z(0), z(0, 0), z(0, 0, dt=torch.bool), z(L_count + 1), 0
    max_nbr = int(nbr_leaf_pos.shape[1])
    if max_nbr == 0:
        return z(0), z(0, k), z(0, k, dt=torch.bool), z(L_count + 1), k
    blocks = (counts + (k - 1)) // k
    boff = torch.cat([z(1), torch.cumsum(blocks, 0).to(INDEX_DTYPE)])
    nb = int(boff[-1].item())
    if nb == 0:
        return z(0), z(0, k), z(0, k, dt=torch.bool), boff, k
    bid = torch.arange(nb, dtype=INDEX_DTYPE, device=dev)
    tl = torch.searchsorted(boff[1:], bid, right=True)
    local = bid - boff[tl]
    es = offsets[tl] + local * k
    stop = offsets[tl + 1]
    eo = torch.arange(k, dtype=INDEX_DTYPE, device=dev)
    eidx = es[:, None] + eo[None, :]
    ev = eidx < stop[:, None]
    lidx = local[:, None] * k + eo[None, :]
    lv = lidx < max_nbr
    safe = torch.where(ev & lv, lidx, torch.zeros_like(lidx))
    src = nbr_leaf_pos[tl[:, None], safe]
    sv = src >= 0
    valid = ev & lv & sv
    src = torch.where(valid, src, torch.zeros_like(src))
    return tl.to(INDEX_DTYPE), src.to(INDEX_DTYPE), valid, boff, k


@dataclass
class _WalkOut:
    far_counts: torch.Tensor
    node_offsets: torch.Tensor
    level_offsets: torch.Tensor
    sources: torch.Tensor
    targets: torch.Tensor
    target_levels: torch.Tensor
    near_counts: torch.Tensor
    near_offsets: torch.Tensor
    neighbors: torch.Tensor
    neighbor_leaf_positions: torch.Tensor
    leaf_indices: torch.Tensor
    particle_order_leaf_indices: torch.Tensor
    particle_order_to_native_leaf: torch.Tensor
    stats: dict
    num_levels: int


# Learned mode, per (mac, theta): the overflow log capacity and the far /
# near extension entries (per tree node) that the last predicted walk
# needed, to size the next walk's log and extension room.
_LEARNED_HINTS: dict = {}


def _learned_walk_fill(topology, d, total, ni, nl, num_levels, center, radius, max_extent,
                       leafpos32, theta, mac_type, mac, dehnen_radius_scale, root, wf_capacity,
                       timing, evs):
    """Predicted capacities -> padded offsets -> one walk into the padded rows
    -> offsets, overflowed rows completed.  Re-runs the walk with the sizes
    it reports when the wavefront, the overflow log or the extension room was
    too small."""
    from .predictor import default_predictor

    lib = L.lib()
    dev = topology.parent.device
    st = L.stream_handle(dev)
    ib, idt = INDEX_BITS, INDEX_DTYPE
    params, cal = default_predictor(dev)
    far_cap = torch.empty(total, dtype=torch.int32, device=dev)
    near_cap = torch.empty(nl, dtype=torch.int32, device=dev)
    L.check(lib.ygx_predict_caps(
        L.ptr(center), L.ptr(radius), L.ptr(max_extent), L.ptr(d.level32), L.ptr(d.parent32),
        L.ptr(leafpos32), total, ni, L.ptr(topology.node_ranges.contiguous()), ib, root,
        float(theta), mac, L.ptr(params), float(cal["slack_far"]), float(cal["slack_near"]),
        int(cal["add"]), L.ptr(far_cap), L.ptr(near_cap), st), "ygx_predict_caps")
    key = _hint_key(mac_type, theta, total)
    hint_wf, _ = _CAPACITY_HINTS.get(key, (0.0, 0.0))
    cap = int(wf_capacity) if wf_capacity else max(32 * total + 65536, int(1.25 * hint_wf * total))
    cap = min(cap, _WF_CAP_MAX)
    h_ovf, h_ext_far, h_ext_near = _LEARNED_HINTS.get(key, (0.0, 0.0, 0.0))
    log_cap = max(65536, int(1.25 * h_ovf * total))
    extra = [int(1.25 * h_ext_far * total), int(1.25 * h_ext_near * total)]
    runs = 0
    while True:
        runs += 1
        ws = L.workspace(lib.ygx_traverse_workspace_size(total, nl, cap, log_cap), dev)
        sums = np.zeros(2, np.uint64)
        L.check(lib.ygx_traverse_pad_offsets(total, ni, cap, log_cap, L.ptr(far_cap),
                                             L.ptr(near_cap), sums.ctypes.data, L.ptr(ws),
                                             ws.numel(), st), "ygx_traverse_pad_offsets")
        pf, pn = int(sums[0]), int(sums[1])
        fr = pf + max(extra[0], pf // 16 + 4096)
        nr = pn + max(extra[1], pn // 16 + 4096)
        far_raw = torch.empty(fr, dtype=torch.int32, device=dev)
        near_raw = torch.empty(nr, dtype=torch.int32, device=dev)
        stats = np.zeros(L.TSTAT_WORDS, np.uint64)
        flags = np.zeros(1, np.uint32)
        rc = lib.ygx_traverse_walk_predicted(
            L.ptr(center), L.ptr(radius), L.ptr(max_extent), L.ptr(d.left32), L.ptr(d.right32),
            L.ptr(leafpos32), total, ni, mac, float(theta), float(dehnen_radius_scale), root,
            _GENS_HINTS.get(key, 0), cap, log_cap, L.ptr(far_cap), L.ptr(near_cap),
            L.ptr(far_raw), L.ptr(near_raw),
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
            del ws, far_raw, near_raw
            continue
        L.check(rc, "ygx_traverse_walk_predicted")
        if f & L.FLAG_BAD_INPUT:
            raise ValueError("MAC extents must be positive (geometry has zero or NaN extents)")
        if f:
            raise L.YgxError(f"traversal walk reported flags {f:#x}")
        ef, en = int(stats[L.TSTAT["ext_far"]]), int(stats[L.TSTAT["ext_near"]])
        if pf + ef > fr or pn + en > nr:
            extra = [ef, en]  # the walk is deterministic: the re-run needs exactly this
            del ws, far_raw, near_raw
            continue
        break
    if not wf_capacity:
        # hints only grow: inputs that alternate between sizes then do not
        # re-run the walk
        pw, pl = _CAPACITY_HINTS.get(key, (0.0, 0.0))
        _CAPACITY_HINTS[key] = (max(pw, int(stats[L.TSTAT["wf_need"]]) / total), pl)
        po = _LEARNED_HINTS.get(key, (0.0, 0.0, 0.0))
        _LEARNED_HINTS[key] = (max(po[0], int(stats[L.TSTAT["log_need"]]) / total),
                               int(stats[L.TSTAT["ext_far"]]) / total,
                               int(stats[L.TSTAT["ext_near"]]) / total)
    _GENS_HINTS[key] = int(stats[L.TSTAT["gens"]])
    if timing:
        evs[1].record()
    s = {k: int(stats[v]) for k, v in L.TSTAT.items()}
    LAST_WALK_STATS.clear()
    entries = max(1, s["far_total"] + s["near_total"])
    LAST_WALK_STATS.update(
        s, wf_capacity=cap, log_capacity=log_cap, mode="learned", walk_runs=runs, padded_far=pf,
        padded_near=pn, over_allocation=(pf + pn) / entries,
        overflow_row_fraction=s["ovf_rows"] / max(1, total + nl),
        overflow_entry_fraction=s["ovf_entries"] / entries)
    node_offsets = torch.empty(total + 1, dtype=idt, device=dev)
    far_counts = torch.empty(total, dtype=idt, device=dev)
    level_offsets = torch.empty(num_levels + 1, dtype=idt, device=dev)
    near_offsets = torch.empty(nl + 1, dtype=idt, device=dev)
    near_counts = torch.empty(nl, dtype=idt, device=dev)
    far_raw_off = torch.empty(total, dtype=torch.int64, device=dev)
    near_raw_off = torch.empty(max(nl, 1), dtype=torch.int64, device=dev)
    L.check(lib.ygx_traverse_fill_predicted(
        total, ni, cap, log_cap, L.ptr(far_cap), L.ptr(near_cap), fr, nr, L.ptr(d.nbl32),
        L.ptr(topology.level_offsets), num_levels, ib, L.ptr(node_offsets), L.ptr(far_counts),
        L.ptr(level_offsets), L.ptr(near_offsets), L.ptr(near_counts), L.ptr(far_raw),
        L.ptr(near_raw), L.ptr(far_raw_off), L.ptr(near_raw_off), L.ptr(ws), ws.numel(), st),
        "ygx_traverse_fill_predicted")
    return (ws, cap, log_cap, s, far_raw, near_raw, far_raw_off, near_raw_off, node_offsets,
            far_counts, level_offsets, near_offsets, near_counts)


# Target mode, per (mac, theta, size octave): what each capacity needed per
# tree node in the last walk (far / near pools, split lists, spill area,
# far / near / split chunk records, continuation queue).
_TARGET_HINTS: dict = {}
_TARGET_FALLBACK_WARNED: set = set()
# Learned mode on the per-target walk, per (mac, theta, size octave): the far
# / near extension entries (per tree node) the last walk needed.
_LEARNED_TARGET_HINTS: dict = {}


def _target_caps(total: int, nl: int, hint) -> list:
    if hint is not None:
        return [max(1 << 16, int(1.15 * h * total) + 4096) for h in hint]
    far = max(1 << 20, 256 * total)
    near = max(1 << 20, 1024 * nl)
    split = max(1 << 20, 512 * total)
    return [far, near, split, max(1 << 20, 64 * total), 4 * total + far // 32 + 4096,
            4 * nl + near // 32 + 4096, 4 * total + split // 64 + 4096, 4 * total + 65536]


def _target_walk(topology, d, total, ni, nl, num_levels, center, radius, max_extent, leafpos32,
                 theta, mac_type, mac, dehnen_radius_scale, root, timing, evs, ordered,
                 learned=False):
    """ygx_target_walk + ygx_target_walk_lists: returns the output arrays and
    stats, or None when the walk cannot serve this tree (then the caller
    runs the log schedule).  ordered: rows ordered by the walk itself, else
    sorted after it.  learned (unordered): rows get the capacity predictor's
    slots and the walk writes every chunk that fits in place."""
    lib = L.lib()
    dev = topology.parent.device
    st = L.stream_handle(dev)
    ib, idt = INDEX_BITS, INDEX_DTYPE
    mode_name = "learned" if learned else ("target_ordered" if ordered else "target")
    key = _hint_key(mac_type, theta, total, mode_name)
    o = 1 if ordered else 0
    caps = _target_caps(total, nl, _TARGET_HINTS.get(key))
    far_raw = near_raw = None
    if learned:
        from .predictor import default_predictor

        params, cal = default_predictor(dev)
        far_rcap = torch.empty(total, dtype=torch.int32, device=dev)
        near_rcap = torch.empty(nl, dtype=torch.int32, device=dev)
        L.check(lib.ygx_predict_caps(
            L.ptr(center), L.ptr(radius), L.ptr(max_extent), L.ptr(d.level32),
            L.ptr(d.parent32), L.ptr(leafpos32), total, ni,
            L.ptr(topology.node_ranges.contiguous()), ib, root, float(theta), mac, L.ptr(params),
            float(cal["slack_far"]), float(cal["slack_near"]), int(cal["add"]), L.ptr(far_rcap),
            L.ptr(near_rcap), st), "ygx_predict_caps")
        pad_far = torch.empty(total + 1, dtype=torch.int64, device=dev)
        pad_near = torch.empty(nl + 1, dtype=torch.int64, device=dev)
        pws = L.workspace(lib.ygx_target_pad_workspace_size(total, nl), dev)
        sums = np.zeros(2, np.uint64)
        L.check(lib.ygx_target_pad(total, nl, L.ptr(far_rcap), L.ptr(near_rcap), L.ptr(pad_far),
                                   L.ptr(pad_near), sums.ctypes.data, L.ptr(pws), pws.numel(), st),
                "ygx_target_pad")
        del pws
        pf, pn = int(sums[0]), int(sums[1])
        h = _LEARNED_TARGET_HINTS.get(key, (0.0, 0.0))
        ext = [int(1.25 * h[0] * total), int(1.25 * h[1] * total)]
    runs = 0
    while True:
        runs += 1
        caps_np = np.asarray(caps, np.int64)
        pred = (None,) * 6
        if learned:
            fr = pf + max(ext[0], pf // 16 + 4096)
            nr = pn + max(ext[1], pn // 16 + 4096)
            far_raw = torch.empty(fr, dtype=torch.int32, device=dev)
            near_raw = torch.empty(nr, dtype=torch.int32, device=dev)
            pred = (L.ptr(far_rcap), L.ptr(near_rcap), L.ptr(pad_far), L.ptr(pad_near),
                    L.ptr(far_raw), L.ptr(near_raw))
        ws = L.workspace(lib.ygx_target_walk_workspace_size(total, nl, caps_np.ctypes.data, o),
                         dev)
        stats = np.zeros(L.TSTAT_WORDS, np.uint64)
        needs = np.zeros(14, np.uint64)
        flags = np.zeros(1, np.uint32)
        L.check(lib.ygx_target_walk(
            L.ptr(center), L.ptr(radius), L.ptr(max_extent), L.ptr(d.left32), L.ptr(d.right32),
            L.ptr(leafpos32), L.ptr(d.parent32), L.ptr(d.level32), L.ptr(d.nbl32), total, ni,
            root, mac, float(theta), float(dehnen_radius_scale), caps_np.ctypes.data, o, *pred,
            L.ptr(topology.level_offsets), num_levels, ib, stats.ctypes.data,
            needs.ctypes.data, flags.ctypes.data, L.ptr(ws), ws.numel(), st), "ygx_target_walk")
        f = int(flags[0])
        if f & L.FLAG_BAD_INPUT:
            raise ValueError("MAC extents must be positive (geometry has zero or NaN extents)")
        if f & (L.FLAG_TIMEOUT | L.FLAG_MALFORMED):
            if key not in _TARGET_FALLBACK_WARNED:
                _TARGET_FALLBACK_WARNED.add(key)
                logger.warning("target walk could not serve this tree (flags %#x); using the "
                               "log schedule", f)
            return None
        if f & L.FLAG_LOG_OVERFLOW:
            # A walk cut short by one capacity reports only the needs of the
            # work it did: grow what overflowed by 2x its need and re-run.
            grown = [c if int(n) <= c else 2 * int(n) + 4096 for c, n in zip(caps, needs[:8])]
            if grown == caps or runs > 12:
                raise L.YgxError(f"target walk capacities did not converge (flags {f:#x})")
            caps = grown
            ws = far_raw = near_raw = None
            continue
        if f:
            raise L.YgxError(f"target walk reported flags {f:#x}")
        if learned:
            ef = int(stats[L.TSTAT["ext_far"]])
            en = int(stats[L.TSTAT["ext_near"]])
            if pf + ef > far_raw.numel() or pn + en > near_raw.numel():
                ext = [ef, en]  # the row counts are deterministic: the re-run fits
                ws = far_raw = near_raw = None
                continue
        break
    prev = _TARGET_HINTS.get(key)
    cur = [int(n) / total for n in needs[:8]]
    _TARGET_HINTS[key] = cur if prev is None else [max(a, b) for a, b in zip(prev, cur)]
    if learned:
        _LEARNED_TARGET_HINTS[key] = (int(stats[L.TSTAT["ext_far"]]) / total,
                                      int(stats[L.TSTAT["ext_near"]]) / total)
    if timing:
        evs[1].record()
    s = {k: int(stats[v]) for k, v in L.TSTAT.items()}
    P, Q = s["far_total"], s["near_total"]
    node_offsets = torch.empty(total + 1, dtype=idt, device=dev)
    far_counts = torch.empty(total, dtype=idt, device=dev)
    level_offsets = torch.empty(num_levels + 1, dtype=idt, device=dev)
    near_offsets = torch.empty(nl + 1, dtype=idt, device=dev)
    near_counts = torch.empty(nl, dtype=idt, device=dev)
    sources = torch.empty(P, dtype=idt, device=dev)
    targets = torch.empty(P, dtype=idt, device=dev)
    target_levels = torch.empty(P, dtype=idt, device=dev)
    neighbors = torch.empty(Q, dtype=idt, device=dev)
    max_nbr = _dense_table_width(s["max_near"], nl, ib, dev)
    nlp = torch.empty((nl, max_nbr), dtype=idt, device=dev)
    if timing:
        evs[2].record()
    if not ordered and not learned:
        far_raw = torch.empty(max(P, 1), dtype=torch.int32, device=dev)
        near_raw = torch.empty(max(Q, 1), dtype=torch.int32, device=dev)
    raw = (None, 0, None, 0) if ordered else (L.ptr(far_raw), far_raw.numel(), L.ptr(near_raw),
                                              near_raw.numel())
    L.check(lib.ygx_target_walk_lists(
        total, ni, caps_np.ctypes.data, o, *pred[:4], *raw, L.ptr(d.nbl32), L.ptr(d.level32),
        L.ptr(topology.level_offsets), num_levels, ib, P, Q, int(needs[4]), int(needs[5]),
        L.ptr(node_offsets), L.ptr(far_counts), L.ptr(level_offsets), L.ptr(sources),
        L.ptr(targets), L.ptr(target_levels), L.ptr(near_offsets), L.ptr(near_counts),
        L.ptr(neighbors), L.ptr(leafpos32), max_nbr, L.ptr(nlp) if max_nbr > 0 else None,
        L.ptr(ws), ws.numel(), st), "ygx_target_walk_lists")
    f = L.read_status(ws)
    if f:
        raise L.YgxError(f"target walk lists reported flags {f:#x}")
    far_raw = near_raw = None
    LAST_WALK_STATS.clear()
    if learned:
        entries = max(1, P + Q)
        LAST_WALK_STATS.update(padded_far=pf, padded_near=pn, over_allocation=(pf + pn) / entries,
                               overflow_row_fraction=s["ovf_rows"] / max(1, total + nl),
                               overflow_entry_fraction=s["ovf_entries"] / entries)
    LAST_WALK_STATS.update(s, mode=mode_name, walk_runs=runs,
                           split_list_max_chunks=int(needs[8]),
                           continuation_pieces=int(needs[7]), pieces_run=int(needs[11]),
                           busy_fraction=int(needs[9]) / max(1, int(needs[9]) + int(needs[10])),
                           steps=int(needs[12]), far_records=int(needs[4]),
                           near_records=int(needs[5]),
                           lane_fill=int(needs[13]) / max(1, 32 * int(needs[12])))
    if P == 0:
        node_offsets.zero_()
        level_offsets.zero_()
    return s, node_offsets, far_counts, level_offsets, sources, targets, target_levels, \
        near_offsets, near_counts, neighbors, nlp


_DEVICE_BYTES: dict = {}


def _dense_table_width(max_near: int, nl: int, ib: int, dev) -> int:
    """Width of the dense neighbour_leaf_positions table, or 0 when it would
    not fit the budget (warned once per table shape).  The free-memory query
    behind the default budget can take milliseconds, so it is skipped when
    the table exceeds a quarter of the whole device (then it exceeds a
    quarter of the free memory too)."""
    dense_bytes = nl * max_near * (4 if ib == 32 else 8)
    too_big = False
    if _DENSE_BUDGET is None:
        key = (dev.type, dev.index)
        if key not in _DEVICE_BYTES:
            _DEVICE_BYTES[key] = torch.cuda.get_device_properties(dev).total_memory
        too_big = dense_bytes > _DEVICE_BYTES[key] // 4
    if too_big or dense_bytes > _dense_neighbor_budget(dev):
        if (nl, max_near) not in _DENSE_WARNED:  # once per table shape
            _DENSE_WARNED.add((nl, max_near))
            logger.warning(
                "neighbor_leaf_positions would need %.1f GiB (%d leaves x %d neighbours); "
                "returning an empty (L, 0) table -- raise the budget with "
                "set_dense_neighbor_budget() to build it", dense_bytes / 2**30, nl, max_near)
        return 0
    return max_near


def _run_walk(topology, geometry, theta: float, mac_type: str, dehnen_radius_scale: float,
              wf_capacity: Optional[int] = None) -> _WalkOut:
    """Walk (counts + pair log) -> scan -> fill (scatter) -> finalize on the GPU."""
    lib = L.lib()
    total = int(topology.parent.shape[0])
    ni = int(topology.left_child.shape[0])
    nl = total - ni
    dev = topology.parent.device
    st = L.stream_handle(dev)
    ib, idt = INDEX_BITS, INDEX_DTYPE
    leaf_indices, leafpos32, po, po_to_native = _leaf_ordering(topology, total, ni, dev)
    num_levels = _host_of(topology).num_levels
    z = lambda *s: torch.zeros(s, dtype=idt, device=dev)  # noqa: E731
    if ni == 0:
        return _WalkOut(
            far_counts=z(total), node_offsets=z(total + 1), level_offsets=z(num_levels + 1),
            sources=z(0), targets=z(0), target_levels=z(0), near_counts=z(nl),
            near_offsets=z(nl + 1), neighbors=z(0), neighbor_leaf_positions=z(nl, 0),
            leaf_indices=leaf_indices, particle_order_leaf_indices=po,
            particle_order_to_native_leaf=po_to_native,
            stats=dict(far_total=0, near_total=0, max_far=0, max_near=0, accept=0, near=0,
                       refine=0, max_wf=1, gens=0), num_levels=num_levels)
    d = _dev_of(topology)
    timing = _TIMING
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(4)] if timing else None
    if timing:
        evs[0].record()
    center = geometry.center.contiguous().float()
    radius = geometry.radius.contiguous().float()
    max_extent = geometry.max_extent.contiguous().float()
    mode = _TRAVERSAL_MODE
    if mode not in TRAVERSAL_MODES:
        raise ValueError(f"traversal mode must be one of {TRAVERSAL_MODES}, got {mode!r}")
    mac = _MAC_CODES[mac_type]
    root = _root_of(topology, d)
    far_raw_off = near_raw_off = None
    if mode in ("target", "target_ordered", "learned") and not _host_of(topology).malformed and \
            num_levels >= 2 and not wf_capacity:
        out = _target_walk(topology, d, total, ni, nl, num_levels, center, radius, max_extent,
                           leafpos32, theta, mac_type, mac, dehnen_radius_scale, root, timing,
                           evs, mode == "target_ordered", learned=mode == "learned")
        if out is not None:
            (s, node_offsets, far_counts, level_offsets, sources, targets, target_levels,
             near_offsets, near_counts, neighbors, nlp) = out
            if timing:
                evs[3].record()
                torch.cuda.synchronize(dev)
                LAST_WALK_STATS.update(walk_ms=evs[0].elapsed_time(evs[1]),
                                       fill_ms=evs[1].elapsed_time(evs[2]),
                                       finalize_ms=evs[2].elapsed_time(evs[3]))
            return _WalkOut(far_counts=far_counts, node_offsets=node_offsets,
                            level_offsets=level_offsets, sources=sources, targets=targets,
                            target_levels=target_levels, near_counts=near_counts,
                            near_offsets=near_offsets, neighbors=neighbors,
                            neighbor_leaf_positions=nlp, leaf_indices=leaf_indices,
                            particle_order_leaf_indices=po,
                            particle_order_to_native_leaf=po_to_native, stats=s,
                            num_levels=num_levels)
        mode = "log"
    if mode == "learned":
        (ws, cap, log_cap, s, far_src32, near_nbr32, far_raw_off, near_raw_off, node_offsets,
         far_counts, level_offsets, near_offsets, near_counts) = _learned_walk_fill(
            topology, d, total, ni, nl, num_levels, center, radius, max_extent, leafpos32,
            theta, mac_type, mac, dehnen_radius_scale, root, wf_capacity, timing, evs)
        P, Q = s["far_total"], s["near_total"]
    else:
        walk_mode = L.WALK_LOG if mode == "log" else L.WALK_COUNT
        key = _hint_key(mac_type, theta, total)
        hint_wf, hint_log = _CAPACITY_HINTS.get(key, (0.0, 0.0))
        cap = int(wf_capacity) if wf_capacity else max(32 * total + 65536,
                                                       int(1.25 * hint_wf * total))
        log_cap = (max(8 * total + 65536, int(1.1 * hint_log * total))
                   if walk_mode == L.WALK_LOG else 1)
        cap = min(cap, _WF_CAP_MAX)
        runs = 0
        while True:
            runs += 1
            ws = L.workspace(lib.ygx_traverse_workspace_size(total, nl, cap, log_cap), dev)
            stats = np.zeros(L.TSTAT_WORDS, np.uint64)
            flags = np.zeros(1, np.uint32)
            rc = lib.ygx_traverse_walk(
                L.ptr(center), L.ptr(radius), L.ptr(max_extent), L.ptr(d.left32),
                L.ptr(d.right32), L.ptr(leafpos32), total, ni, mac, float(theta),
                float(dehnen_radius_scale), root, walk_mode,
                _GENS_HINTS.get(key, 0), cap, log_cap, stats.ctypes.data,
                flags.ctypes.data, L.ptr(ws), ws.numel(), st)
            f = int(flags[0])
            if f & (L.FLAG_QUEUE_OVERFLOW | L.FLAG_LOG_OVERFLOW) and rc == 0:
                if f & L.FLAG_QUEUE_OVERFLOW:
                    # the needs a truncated walk reports are lower bounds only
                    cap = _grow_wf_cap(cap, stats)
                    log_cap = max(log_cap, int(stats[L.TSTAT["log_need"]]))
                else:
                    # the reported need fits the re-run; head-room spares another
                    # re-run when the next inputs need a little more
                    log_cap = max(int(1.15 * int(stats[L.TSTAT["log_need"]])),
                                  log_cap + log_cap // 4)
                del ws
                continue
            L.check(rc, "ygx_traverse_walk")
            if f & L.FLAG_BAD_INPUT:
                raise ValueError("MAC extents must be positive (geometry has zero or NaN extents)")
            if f:
                raise L.YgxError(f"traversal walk reported flags {f:#x}")
            break
        if not wf_capacity:
            # hints only grow (inputs that alternate do not re-run the walk)
            prev = _CAPACITY_HINTS.get(key, (0.0, 0.0))
            log_need = (max(prev[1], int(stats[L.TSTAT["log_need"]]) / total)
                        if walk_mode == L.WALK_LOG else prev[1])
            _CAPACITY_HINTS[key] = (
                max(prev[0], int(stats[L.TSTAT["wf_need"]]) / total), log_need)
        _GENS_HINTS[key] = int(stats[L.TSTAT["gens"]])
        if timing:
            evs[1].record()
        s = {k: int(stats[v]) for k, v in L.TSTAT.items()}
        LAST_WALK_STATS.clear()
        LAST_WALK_STATS.update(s, wf_capacity=cap, log_capacity=log_cap, mode=mode,
                               walk_runs=runs)
        P, Q = s["far_total"], s["near_total"]
        node_offsets = torch.empty(total + 1, dtype=idt, device=dev)
        far_counts = torch.empty(total, dtype=idt, device=dev)
        level_offsets = torch.empty(num_levels + 1, dtype=idt, device=dev)
        near_offsets = torch.empty(nl + 1, dtype=idt, device=dev)
        near_counts = torch.empty(nl, dtype=idt, device=dev)
        far_src32 = torch.empty(max(P, 1), dtype=torch.int32, device=dev)
        near_nbr32 = torch.empty(max(Q, 1), dtype=torch.int32, device=dev)
        if walk_mode == L.WALK_LOG:
            L.check(lib.ygx_traverse_fill(
                total, ni, cap, log_cap, P, Q, L.ptr(d.nbl32), L.ptr(leafpos32),
                L.ptr(topology.level_offsets), num_levels, ib, L.ptr(node_offsets),
                L.ptr(far_counts), L.ptr(level_offsets), L.ptr(near_offsets), L.ptr(near_counts),
                L.ptr(far_src32), L.ptr(near_nbr32), L.ptr(ws), ws.numel(), st),
                "ygx_traverse_fill")
        else:
            L.check(lib.ygx_traverse_fill_walk(
                total, ni, mac, float(theta), root, cap, log_cap, s["gens"], P, Q,
                L.ptr(d.nbl32),
                L.ptr(topology.level_offsets), num_levels, ib, L.ptr(node_offsets),
                L.ptr(far_counts), L.ptr(level_offsets), L.ptr(near_offsets), L.ptr(near_counts),
                L.ptr(far_src32), L.ptr(near_nbr32), L.ptr(ws), ws.numel(), st),
                "ygx_traverse_fill_walk")
    if timing:
        evs[2].record()
    sources = torch.empty(P, dtype=idt, device=dev)
    targets = torch.empty(P, dtype=idt, device=dev)
    target_levels = torch.empty(P, dtype=idt, device=dev)
    neighbors = torch.empty(Q, dtype=idt, device=dev)
    max_nbr = _dense_table_width(s["max_near"], nl, ib, dev)
    nlp = torch.empty((nl, max_nbr), dtype=idt, device=dev)
    L.check(lib.ygx_traverse_finalize(
        total, ni, cap, log_cap, L.ptr(d.level32), L.ptr(leafpos32), ib, L.ptr(far_src32),
        L.ptr(near_nbr32), L.ptr(far_raw_off) if far_raw_off is not None else None,
        L.ptr(near_raw_off) if near_raw_off is not None else None, None, None,
        L.ptr(sources), L.ptr(targets),
        L.ptr(target_levels),
        L.ptr(neighbors), L.ptr(nlp) if max_nbr > 0 else None, max_nbr, L.ptr(ws), ws.numel(),
        st), "ygx_traverse_finalize")
    if timing:
        evs[3].record()
        torch.cuda.synchronize(dev)
        LAST_WALK_STATS.update(walk_ms=evs[0].elapsed_time(evs[1]),
                               fill_ms=evs[1].elapsed_time(evs[2]),
                               finalize_ms=evs[2].elapsed_time(evs[3]))
    f = L.read_status(ws)
    if f & (L.FLAG_FAR_OVERFLOW | L.FLAG_NEAR_OVERFLOW | L.FLAG_QUEUE_OVERFLOW):
        raise L.YgxError(f"traversal fill pass disagreed with the count pass (flags {f:#x})")
    if P == 0:
        node_offsets = z(total + 1)
        level_offsets = z(num_levels + 1)
    return _WalkOut(far_counts=far_counts, node_offsets=node_offsets,
                    level_offsets=level_offsets, sources=sources, targets=targets,
                    target_levels=target_levels, near_counts=near_counts,
                    near_offsets=near_offsets, neighbors=neighbors,
                    neighbor_leaf_positions=nlp, leaf_indices=leaf_indices,
                    particle_order_leaf_indices=po, particle_order_to_native_leaf=po_to_native,
                    stats=s, num_levels=num_levels)


def _node_order_far_pairs(w, total: int, dev):
    """The far lists in the count-then-fill layout: rows in node order
    (``interaction_offsets``), each row's sources ascending; targets are the
    row's node; tags -1 (no pair policy).  (_raw_to_compact_far_pairs,
    :5340-5390, reads the same arrays.)  One CUDA re-layout of the level-major
    rows (ygx_node_order_far_rows)."""
    idt = INDEX_DTYPE
    lib = L.lib()
    P = int(w.sources.shape[0])
    no = torch.empty(total + 1, dtype=idt, device=dev)
    raw_src = torch.empty(P, dtype=idt, device=dev)
    raw_tgt = torch.empty(P, dtype=idt, device=dev)
    ws = L.workspace(lib.ygx_layout_workspace_size(total), dev)
    L.check(lib.ygx_node_order_far_rows(
        total, L.ptr(w.far_counts), L.ptr(w.node_offsets), L.ptr(w.sources) if P else None,
        INDEX_BITS, L.ptr(no), L.ptr(raw_src) if P else None, L.ptr(raw_tgt) if P else None,
        L.ptr(ws), ws.numel(), L.stream_handle(dev)), "ygx_node_order_far_rows")
    tags = torch.full((P,), -1, dtype=idt, device=dev)
    fpc = torch.tensor(P, dtype=idt, device=dev)
    return no, raw_src, raw_tgt, tags, fpc


def _check_capacities(w: _WalkOut, total: int, ni: int, **kw) -> None:
    """Raise where the reference's runner (_run_dual_tree_walk_raw,
    :3840-4440) would raise on the same pair sets (a far-only or near-only
    run checks only the lists it collects)."""
    v = _capacity_violations(w, total, ni, **kw)
    if v:
        raise RuntimeError(v[0][1])


def _overflow_flags(w: _WalkOut, total: int, ni: int, **kw) -> tuple:
    """``(queue_overflow, far_overflow, near_overflow)`` of the reference's
    padded walk (_dual_tree_walk_impl, :1119-1905) with the capacities the
    caller gave, evaluated on the exact walk's maxima: the flags its
    ``DualTreeWalkResult`` would carry where it returns them instead of
    raising (:4417-4421).  The count-then-fill schedule (no capacities)
    never overflows its exact-size buffers: all False there."""
    kinds = {k for k, _ in _capacity_violations(w, total, ni, **kw)}
    return ("queue" in kinds, "far" in kinds, "near" in kinds)


def _capacity_violations(w: _WalkOut, total: int, ni: int, *, max_interactions_per_node,
                         max_neighbors_per_leaf, max_pair_queue, process_block,
                         traversal_config, collect_far: bool = True,
                         collect_near: bool = True) -> list:
    """Every check of the reference's runner that the walk's maxima fail, as
    ``(kind, message)`` in the order the runner tests them; kind is
    ``queue`` / ``far`` / ``near`` for the padded walk's overflow flags and
    ``count`` for the count-then-fill schedule's own errors."""
    out = []
    s = dict(w.stats)
    if not collect_far:
        s["max_far"] = s["far_total"] = 0
    if not collect_near:
        s["max_near"] = s["near_total"] = 0
    nl = total - ni
    use_count_pass = (max_interactions_per_node is None and max_pair_queue is None
                      and traversal_config is None)
    if use_count_pass:
        conservative = max(total * DEFAULT_PAIR_QUEUE_MULTIPLIER,
                           _auto_pair_queue_candidates(total, ni)[-1])
        if s["max_wf"] > conservative:
            out.append(("count",
                        "Count-pass traversal wavefront overflowed its conservative buffer."))
        if max(1, s["max_near"]) > max(1, _INT32_MAX // max(1, nl)):
            out.append(("count",
                "Suggested per-leaf neighbor capacity is too large to safely allocate on the "
                "host (would overflow int32). Enable local refinement or pass explicit "
                "capacities (max_neighbors_per_leaf / max_interactions_per_node)."))
        if s["far_total"] > _INT32_MAX or s["near_total"] > _INT32_MAX:
            out.append(("count",
                "Dual-tree traversal pair totals exceed signed int32 capacity; refine the tree "
                "or use a lower-memory traversal strategy."))
        return out
    config = traversal_config if traversal_config is not None else _GLOBAL_DUAL_TREE_CONFIG
    auto = _auto_pair_queue_candidates(total, ni)
    if config is not None:
        K = int(config.max_interactions_per_node)
        nbr_limit = int(config.max_neighbors_per_leaf)
        queue = _queue_candidates_bounded(max_capacity=max(4, int(config.max_pair_queue)),
                                          process_block=int(config.process_block))
        queue += [c for c in auto if c > queue[-1]]
        qmsg = "Pair queue capacity exceeded; increase max_pair_queue and rebuild."
    else:
        K = (int(max_interactions_per_node) if max_interactions_per_node is not None
             else _auto_interaction_capacity(total))
        if max_interactions_per_node is not None and max_interactions_per_node < 1:
            raise ValueError("max_interactions_per_node must be >= 1")
        nbr_limit = int(max_neighbors_per_leaf)
        if max_pair_queue is not None:
            queue = [max(4, int(max_pair_queue))]
            qmsg = "Pair queue capacity exceeded; increase max_pair_queue and rebuild."
        else:
            queue = auto
            qmsg = ("Pair queue capacity exceeded; pass a larger max_pair_queue value to "
                    "override auto-scaling.")
    if s["max_wf"] > queue[-1]:
        out.append(("queue", qmsg))
    if s["max_far"] > K:
        out.append(("far", _FAR_MSG))
    hard_cap = max(1, _INT32_MAX // max(1, nl))
    if s["max_near"] > max(min(max(1, nbr_limit), hard_cap), hard_cap):
        out.append(("near", _NEAR_MSG))
    return out


def build_interactions_and_neighbors(
    tree,
    geometry,
    theta: float = 0.5,
    max_interactions_per_node: Optional[int] = None,
    max_neighbors_per_leaf: int = _DEFAULT_MAX_NEIGHBORS,
    max_pair_queue: Optional[int] = None,
    process_block: Optional[int] = None,
    traversal_config: Optional[DualTreeTraversalConfig] = None,
    retry_logger: Optional[Callable[[DualTreeRetryEvent], object]] = None,
    mac_type: MACType = "bh",
    dehnen_radius_scale: float = 1.0,
    pair_policy=None,
    policy_state: object = None,
    *,
    return_result: bool = False,
    return_compact_far_pairs: bool = False,
    return_interactions: bool = True,
    return_grouped: bool = False,
):
    """Far-field interactions and near-field neighbour lists in one walk.

    Same arguments, defaults and return conventions as the reference
    (``(interactions, neighbors)`` plus, in this order, the raw result, the
    compact far pairs and the grouped buffers when requested).  ``pair_policy``
    is outside the GPU pipeline and raises."""
    topology = resolve_tree_topology(tree)
    if mac_type not in _MAC_CODES:
        raise ValueError(f"Unknown mac_type: {mac_type}")
    if float(dehnen_radius_scale) <= 0.0:
        raise ValueError("dehnen_radius_scale must be > 0")
    if pair_policy is not None:
        raise NotImplementedError("pair_policy is outside the GPU traversal (default MAC only)")
    if return_grouped and not return_interactions:
        raise ValueError("grouped interaction return requires return_interactions=True")
    if process_block is not None and process_block < 1:
        raise ValueError("process_block must be >= 1")
    del retry_logger, policy_state  # no retries happen on this path
    total = int(topology.parent.shape[0])
    ni = int(topology.left_child.shape[0])
    w = _run_walk(topology, geometry, theta, mac_type, dehnen_radius_scale)
    caps = dict(max_interactions_per_node=max_interactions_per_node,
                max_neighbors_per_leaf=max_neighbors_per_leaf, max_pair_queue=max_pair_queue,
                process_block=process_block, traversal_config=traversal_config)
    if _REFERENCE_LIMITS:
        _check_capacities(w, total, ni, **caps)
    dev = topology.parent.device
    interactions = None
    if return_interactions:
        interactions = NodeInteractionList(
            offsets=w.node_offsets, sources=w.sources, targets=w.targets, counts=w.far_counts,
            level_offsets=w.level_offsets, target_levels=w.target_levels)
    nl = total - ni
    tb = _target_blocks(w.near_counts, w.near_offsets, w.neighbor_leaf_positions, nl, dev)
    neighbors = NodeNeighborList(
        offsets=w.near_offsets, neighbors=w.neighbors, leaf_indices=w.leaf_indices,
        counts=w.near_counts, particle_order_leaf_indices=w.particle_order_leaf_indices,
        particle_order_to_native_leaf=w.particle_order_to_native_leaf,
        neighbor_leaf_positions=w.neighbor_leaf_positions, target_block_leaf_ids=tb[0],
        target_block_source_leaf_ids=tb[1], target_block_valid_mask=tb[2],
        target_block_offsets=tb[3], target_block_size=int(tb[4]))
    out = [interactions, neighbors]
    if return_result or return_compact_far_pairs:
        no, raw_src, raw_tgt, tags, fpc = _node_order_far_pairs(w, total, dev)
        idt = INDEX_DTYPE
        if return_result:
            s = w.stats
            # with the reference limits on, a failing check raised above, so
            # these are all False; with them off they say what the padded
            # walk would have flagged (the lists themselves stay exact)
            q_ovf, f_ovf, n_ovf = _overflow_flags(w, total, ni, **caps)
            out.append(DualTreeWalkResult(
                interaction_offsets=no, interaction_sources=raw_src,
                interaction_targets=raw_tgt, interaction_tags=tags,
                interaction_counts=w.far_counts, neighbor_offsets=w.near_offsets,
                neighbor_indices=w.neighbors, neighbor_counts=w.near_counts,
                leaf_indices=w.leaf_indices, far_pair_count=fpc,
                near_pair_count=torch.tensor(int(w.neighbors.shape[0]), dtype=idt, device=dev),
                queue_overflow=torch.tensor(q_ovf, device=dev),
                far_overflow=torch.tensor(f_ovf, device=dev),
                near_overflow=torch.tensor(n_ovf, device=dev),
                accept_decisions=torch.tensor(s["accept"], dtype=idt, device=dev),
                near_decisions=torch.tensor(s["near"], dtype=idt, device=dev),
                refine_decisions=torch.tensor(s["refine"], dtype=idt, device=dev)))
        if return_compact_far_pairs:
            out.append(CompactTaggedFarPairs(sources=raw_src, targets=raw_tgt, tags=tags,
                                             far_pair_count=fpc))
    if return_grouped:
        # (:6113-6123) the raw far pairs (node-order rows) grouped by class
        from .grouped_interactions import build_grouped_interactions_from_pairs

        _, g_src, g_tgt, _, _ = _node_order_far_pairs(w, total, dev)
        out.append(build_grouped_interactions_from_pairs(
            topology, geometry, g_src, g_tgt,
            level_offsets=interactions.level_offsets if interactions is not None else None))
    return tuple(out)


def _walk_checked(tree, geometry, theta, mac_type, dehnen_radius_scale, pair_policy,
                  process_block, checks: dict, collect_far: bool, collect_near: bool):
    topology = resolve_tree_topology(tree)
    if mac_type not in _MAC_CODES:
        raise ValueError(f"Unknown mac_type: {mac_type}")
    if float(dehnen_radius_scale) <= 0.0:
        raise ValueError("dehnen_radius_scale must be > 0")
    if pair_policy is not None:
        raise NotImplementedError("pair_policy is outside the GPU traversal (default MAC only)")
    if process_block is not None and process_block < 1:
        raise ValueError("process_block must be >= 1")
    total = int(topology.parent.shape[0])
    ni = int(topology.left_child.shape[0])
    w = _run_walk(topology, geometry, theta, mac_type, dehnen_radius_scale)
    if _REFERENCE_LIMITS:
        _check_capacities(w, total, ni, process_block=process_block, collect_far=collect_far,
                          collect_near=collect_near, **checks)
    return topology, w, total, ni


def _neighbor_list(w, total: int, ni: int, dev) -> NodeNeighborList:
    nl = total - ni
    tb = _target_blocks(w.near_counts, w.near_offsets, w.neighbor_leaf_positions, nl, dev)
    return NodeNeighborList(
        offsets=w.near_offsets, neighbors=w.neighbors, leaf_indices=w.leaf_indices,
        counts=w.near_counts, particle_order_leaf_indices=w.particle_order_leaf_indices,
        particle_order_to_native_leaf=w.particle_order_to_native_leaf,
        neighbor_leaf_positions=w.neighbor_leaf_positions, target_block_leaf_ids=tb[0],
        target_block_source_leaf_ids=tb[1], target_block_valid_mask=tb[2],
        target_block_offsets=tb[3], target_block_size=int(tb[4]))


def build_compact_far_pairs(tree, geometry, theta: float = 0.5,
                            max_interactions_per_node: Optional[int] = None,
                            mac_type: MACType = "bh", *, pair_policy=None,
                            policy_state: object = None, max_pair_queue: Optional[int] = None,
                            process_block: Optional[int] = None,
                            traversal_config: Optional[DualTreeTraversalConfig] = None,
                            retry_logger=None,
                            dehnen_radius_scale: float = 1.0) -> CompactTaggedFarPairs:
    """Exact-length far pairs (build_compact_far_pairs,
    _interactions_impl.py:5765-5816; public wrapper interactions.py:110-175):
    ``sources`` / ``targets`` / ``tags`` of every directed far entry, rows in
    node order with ascending sources, tags -1, ``far_pair_count`` their
    number.  Same walk as build_interactions_and_neighbors."""
    del retry_logger, policy_state
    topology, w, total, ni = _walk_checked(
        tree, geometry, theta, mac_type, dehnen_radius_scale, pair_policy, process_block,
        dict(max_interactions_per_node=max_interactions_per_node,
             max_neighbors_per_leaf=_DEFAULT_MAX_NEIGHBORS, max_pair_queue=max_pair_queue,
             traversal_config=traversal_config), True, False)
    _, src, tgt, tags, fpc = _node_order_far_pairs(w, total, topology.parent.device)
    return CompactTaggedFarPairs(sources=src, targets=tgt, tags=tags, far_pair_count=fpc)


def build_leaf_neighbor_lists(tree, geometry, theta: float = 0.5,
                              max_neighbors_per_leaf: int = _DEFAULT_MAX_NEIGHBORS,
                              max_interactions_per_node: Optional[int] = None,
                              mac_type: MACType = "bh", *, pair_policy=None,
                              policy_state: object = None,
                              max_pair_queue: Optional[int] = None,
                              process_block: Optional[int] = None,
                              traversal_config: Optional[DualTreeTraversalConfig] = None,
                              retry_logger=None,
                              dehnen_radius_scale: float = 1.0) -> NodeNeighborList:
    """Near-field neighbour lists of the leaves alone (build_leaf_neighbor_lists,
    _interactions_impl.py:5917-5990): the NodeNeighborList that
    build_interactions_and_neighbors returns."""
    del retry_logger, policy_state
    topology, w, total, ni = _walk_checked(
        tree, geometry, theta, mac_type, dehnen_radius_scale, pair_policy, process_block,
        dict(max_interactions_per_node=max_interactions_per_node,
             max_neighbors_per_leaf=max_neighbors_per_leaf, max_pair_queue=max_pair_queue,
             traversal_config=traversal_config), False, True)
    return _neighbor_list(w, total, ni, topology.parent.device)


def build_compact_far_pairs_and_leaf_neighbor_lists(
        tree, geometry, theta: float = 0.5,
        max_neighbors_per_leaf: int = _DEFAULT_MAX_NEIGHBORS,
        max_interactions_per_node: Optional[int] = None, mac_type: MACType = "bh", *,
        pair_policy=None, policy_state: object = None, max_pair_queue: Optional[int] = None,
        process_block: Optional[int] = None,
        traversal_config: Optional[DualTreeTraversalConfig] = None, retry_logger=None,
        dehnen_radius_scale: float = 1.0, timing_callback=None,
        compact_far_pair_capacity: Optional[int] = None):
    """``(CompactTaggedFarPairs, NodeNeighborList)`` from one walk
    (_interactions_impl.py:5819-5914; public wrapper interactions.py:180-260).
    With ``compact_far_pair_capacity`` the far arrays are padded with -1 to
    that length, and a larger pair count raises the reference's RuntimeError
    (_raw_to_compact_far_pairs, :5340-5360).  ``timing_callback(stage,
    seconds)`` receives the wall time of the whole call."""
    import time

    del retry_logger, policy_state
    t0 = time.perf_counter()
    topology, w, total, ni = _walk_checked(
        tree, geometry, theta, mac_type, dehnen_radius_scale, pair_policy, process_block,
        dict(max_interactions_per_node=max_interactions_per_node,
             max_neighbors_per_leaf=max_neighbors_per_leaf, max_pair_queue=max_pair_queue,
             traversal_config=traversal_config), True, True)
    dev = topology.parent.device
    _, src, tgt, tags, fpc = _node_order_far_pairs(w, total, dev)
    if compact_far_pair_capacity is not None:
        cap = int(compact_far_pair_capacity)
        P = int(src.shape[0])
        if P > cap:
            raise RuntimeError(
                "strict fused compact far-pair cap exceeded: "
                f"cap={cap}. Increase JACCPOT_STATIC_STRICT_FUSED_COMPACT_FAR_PAIR_CAP.")

        def pad(x):
            out = torch.full((cap,), -1, dtype=x.dtype, device=dev)
            out[:P] = x
            return out

        src, tgt, tags = pad(src), pad(tgt), pad(tags)
    far = CompactTaggedFarPairs(sources=src, targets=tgt, tags=tags, far_pair_count=fpc)
    near = _neighbor_list(w, total, ni, dev)
    if timing_callback is not None:
        torch.cuda.synchronize(dev)
        timing_callback("compact_far_pairs_and_leaf_neighbors", time.perf_counter() - t0)
    return far, near


__all__ = [
    "MACType", "DualTreeTraversalConfig", "DualTreeRetryEvent", "DualTreeWalkResult",
    "NodeInteractionList", "NodeNeighborList", "CompactTaggedFarPairs",
    "build_interactions_and_neighbors", "set_default_dual_tree_config",
    "build_compact_far_pairs", "build_leaf_neighbor_lists",
    "build_compact_far_pairs_and_leaf_neighbor_lists",
    "set_dense_neighbor_budget", "set_reference_limits",
]

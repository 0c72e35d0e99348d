"""Per-node mass and multipole moments on the GPU.

Mirrors ``TreeMassMoments`` / ``TreeMultipoleMoments`` /
``compute_tree_mass_moments`` / ``compute_tree_multipole_moments`` /
``pack_multipole_expansions`` (yggdrax/tree_moments.py:33-48, 183-197,
686-940).  The kernels (``csrc/moments.cu``) follow the reference's
algorithm -- fp32 prefix sums of mass-weighted monomials over the
Morton-sorted particles, differenced at each node's particle range, shifted
to the expansion centre with the binomial stencil -- and its fp32 operation
order, except that the prefix sums are a parallel scan: results agree with
the reference to the rounding of those sums, not bit for bit.
"""

from __future__ import annotations

from typing import NamedTuple, Optional

import torch

from . import _lib as L
from .dtypes import INDEX_BITS, INDEX_DTYPE
from .tree import resolve_tree_topology

MAX_MULTIPOLE_ORDER = 4


def total_coefficients(max_order: int) -> int:
    """Packed length for orders 0..max_order (multipole_utils.py)."""
    o = int(max_order)
    return (o + 1) * (o + 2) * (o + 3) // 6


def level_offset(level: int) -> int:
    lv = int(level)
    return lv * (lv + 1) * (lv + 2) // 6


def multi_index_tuples(level: int):
    lv = int(level)
    return tuple((i, j, lv - i - j) for i in range(lv + 1) for j in range(lv + 1 - i))


class TreeMassMoments(NamedTuple):
    """Total mass and centre of mass of every node (tree_moments.py:33-37)."""

    mass: torch.Tensor
    center_of_mass: torch.Tensor


class TreeMultipoleMoments(NamedTuple):
    """Multipole summaries through the hexadecapole (tree_moments.py:183-197)."""

    max_order: int
    mass: torch.Tensor
    center: torch.Tensor
    dipole: torch.Tensor
    second_moment: torch.Tensor
    quadrupole: torch.Tensor
    third_moment: torch.Tensor
    octupole: torch.Tensor
    fourth_moment: torch.Tensor
    hexadecapole: torch.Tensor
    raw_packed: torch.Tensor


def _validate(topology, positions_sorted, masses_sorted):
    n = int(topology.num_particles)
    if topology.node_ranges.shape[0] != topology.parent.shape[0]:
        raise ValueError("tree.node_ranges must align with tree.parent shape")
    if positions_sorted.shape[0] != n:
        raise ValueError("positions_sorted must match tree.num_particles")
    if masses_sorted.shape[0] != n:
        raise ValueError("masses_sorted must match tree.num_particles")
    if positions_sorted.ndim != 2 or positions_sorted.shape[1] != 3:
        raise ValueError("positions must have shape (N, 3)")


def _run(topology, positions_sorted, masses_sorted, order: int, centers, packed: bool):
    lib = L.lib()
    dev = topology.parent.device
    pos = positions_sorted.contiguous().float()
    mass = masses_sorted.contiguous().float()
    n, nodes = int(pos.shape[0]), int(topology.parent.shape[0])
    ranges = topology.node_ranges.to(INDEX_DTYPE).contiguous()
    f = lambda *s: torch.empty(s, dtype=torch.float32, device=dev)  # noqa: E731
    out = dict(mass=f(nodes), com=f(nodes, 3))
    if packed:
        C = total_coefficients(order)
        out.update(center=f(nodes, 3), packed=f(nodes, C), dipole=f(nodes, 3),
                   second=f(nodes, 3, 3), quad=f(nodes, 3, 3), third=f(nodes, 3, 3, 3),
                   oct=f(nodes, 3, 3, 3), fourth=f(nodes, 3, 3, 3, 3),
                   hexa=f(nodes, 3, 3, 3, 3))
    ws = L.workspace(lib.ygx_moments_workspace_size(n, order), dev)
    P = lambda k: L.ptr(out[k]) if k in out else None  # noqa: E731
    ctr = centers.contiguous().float() if centers is not None else None
    L.check(lib.ygx_tree_moments(
        L.ptr(pos), L.ptr(mass), n, L.ptr(ranges), INDEX_BITS, nodes, order,
        L.ptr(ctr) if ctr is not None else None, P("mass"), P("com"), P("center"), P("packed"),
        P("dipole"), P("second"), P("quad"), P("third"), P("oct"), P("fourth"), P("hexa"),
        L.ptr(ws), ws.numel(), L.stream_handle(dev)), "ygx_tree_moments")
    return out


def compute_tree_mass_moments(tree, positions_sorted: torch.Tensor,
                              masses_sorted: torch.Tensor) -> TreeMassMoments:
    """Total mass and centre of mass of every node (tree_moments.py:686-744)."""
    topology = resolve_tree_topology(tree)
    _validate(topology, positions_sorted, masses_sorted)
    o = _run(topology, positions_sorted, masses_sorted, 1, None, False)
    return TreeMassMoments(mass=o["mass"], center_of_mass=o["com"])


def compute_tree_multipole_moments(tree, positions_sorted: torch.Tensor,
                                   masses_sorted: torch.Tensor,
                                   expansion_centers: Optional[torch.Tensor] = None,
                                   max_order: int = 2) -> TreeMultipoleMoments:
    """Multipole moments through ``max_order`` about ``expansion_centers``
    (default: the centres of mass) for every node (tree_moments.py:747-877)."""
    topology = resolve_tree_topology(tree)
    _validate(topology, positions_sorted, masses_sorted)
    order = int(max_order)
    if order < 0 or order > MAX_MULTIPOLE_ORDER:
        raise ValueError(f"max_order must be between 0 and {MAX_MULTIPOLE_ORDER} inclusive")
    nodes = int(topology.parent.shape[0])
    if expansion_centers is not None and tuple(expansion_centers.shape) != (nodes, 3):
        raise ValueError("expansion_centers must have shape (num_nodes, 3)")
    o = _run(topology, positions_sorted, masses_sorted, order, expansion_centers, True)
    return TreeMultipoleMoments(
        max_order=order, mass=o["mass"], center=o["center"], dipole=o["dipole"],
        second_moment=o["second"], quadrupole=o["quad"], third_moment=o["third"],
        octupole=o["oct"], fourth_moment=o["fourth"], hexadecapole=o["hexa"],
        raw_packed=o["packed"])


def pack_multipole_expansions(moments: TreeMultipoleMoments, max_order: int) -> torch.Tensor:
    """Packed triangular coefficients through ``max_order`` read off the
    trace-free tensors (tree_moments.py:878-930)."""
    order = int(max_order)
    if order < 0 or order > MAX_MULTIPOLE_ORDER:
        raise ValueError(f"max_order must be between 0 and {MAX_MULTIPOLE_ORDER} inclusive")
    if order > moments.max_order:
        raise ValueError("cannot pack coefficients beyond stored max_order")
    n = int(moments.mass.shape[0])
    out = torch.zeros((n, total_coefficients(order)), dtype=moments.mass.dtype,
                      device=moments.mass.device)
    out[:, 0] = moments.mass
    tensors = {1: moments.dipole, 2: moments.quadrupole, 3: moments.octupole,
               4: moments.hexadecapole}
    for lv in range(1, order + 1):
        t = tensors[lv]
        for k, (a, b, c) in enumerate(multi_index_tuples(lv)):
            idx = (0,) * a + (1,) * b + (2,) * c
            out[:, level_offset(lv) + k] = t[(slice(None),) + idx]
    return out


__all__ = ["TreeMassMoments", "TreeMultipoleMoments", "compute_tree_mass_moments",
           "compute_tree_multipole_moments", "pack_multipole_expansions"]

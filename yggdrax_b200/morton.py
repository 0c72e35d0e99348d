"""Bounds and Morton codes on the GPU (mirrors yggdrax/bounds.py:11-33 and
yggdrax/morton.py:43-156)."""

from __future__ import annotations

import torch

from . import _lib as L
from .tree import _bounds_tensor, _encode_sort


def infer_bounds(positions: torch.Tensor):
    """Padded bounding box ``(min - pad, max + pad)`` with
    ``pad = max(0.05 * span, 1e-6)`` per axis (float32)."""
    L.require_cuda(positions, "positions")
    pos = positions.contiguous()
    if pos.dtype != torch.float32 or pos.dim() != 2 or pos.shape[1] != 3:
        raise ValueError("positions must be a float32 (N, 3) tensor")
    lib = L.lib()
    out = torch.empty(6, dtype=torch.float32, device=pos.device)
    ws = L.workspace(lib.ygx_encode_sort_workspace_size(0), pos.device)
    L.check(lib.ygx_bounds(L.ptr(pos), int(pos.shape[0]), L.ptr(out), L.ptr(ws), ws.numel(),
                           L.stream_handle(pos.device)), "ygx_bounds")
    return out[:3], out[3:]


def morton_encode(positions: torch.Tensor, bounds) -> torch.Tensor:
    """63-bit Morton codes (uint64) of float32 positions in ``bounds``."""
    L.require_cuda(positions, "positions")
    pos = positions.contiguous()
    lib = L.lib()
    b = _bounds_tensor(bounds, pos.device)
    codes = torch.empty(int(pos.shape[0]), dtype=torch.uint64, device=pos.device)
    L.check(lib.ygx_morton_encode(L.ptr(pos), int(pos.shape[0]), L.ptr(b), L.ptr(codes),
                                  L.stream_handle(pos.device)), "ygx_morton_encode")
    return codes


def sort_by_morton(codes: torch.Tensor) -> torch.Tensor:
    """Indices that stably sort ``codes`` ascending (ties by index)."""
    L.require_cuda(codes, "codes")
    lib = L.lib()
    n = int(codes.shape[0])
    keys = codes.contiguous()
    kout = torch.empty_like(keys)
    vals = torch.empty(n, dtype=torch.int32, device=codes.device)
    ws = L.workspace(lib.ygx_sort_pairs_workspace_size(n), codes.device)
    L.check(lib.ygx_sort_pairs(L.ptr(keys), None, n, 0, 64, L.ptr(kout), L.ptr(vals), L.ptr(ws),
                               ws.numel(), L.stream_handle(codes.device)), "ygx_sort_pairs")
    return vals.to(torch.int64)


def encode_and_sort(positions: torch.Tensor, bounds=None):
    """Fused bounds + encode + stable sort: ``(bounds6, sorted_codes, order)``."""
    L.require_cuda(positions, "positions")
    pos = positions.contiguous()
    b, codes, order, _ = _encode_sort(pos, int(pos.shape[0]), _bounds_tensor(bounds, pos.device),
                                      pos.device, L.stream_handle(pos.device))
    return b, codes, order


def get_common_prefix_length(code1, code2) -> int:
    """Shared leading bits of two codes (64 when equal), morton.py:118-139."""
    c1, c2 = int(code1), int(code2)
    if c1 == c2:
        return 64
    return 64 - (c1 ^ c2).bit_length()


__all__ = ["infer_bounds", "morton_encode", "sort_by_morton", "encode_and_sort",
           "get_common_prefix_length"]

"""ctypes binding of ``libygx.so`` (declared in ``include/ygx.h``).

The library is built in-tree by :mod:`yggdrax_b200.build_ext`.  There is no
CPU fallback: if the shared object is missing or no CUDA device is present,
every entry point raises.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
# YGGDRAX_B200_LIBRARY names another build of the same library (same ABI).
LIB_PATH = os.environ.get("YGGDRAX_B200_LIBRARY") or os.path.join(_HERE, "libygx.so")

YGX_OK = 0
ERROR_NAMES = {
    1: "YGX_ERR_ARG",
    2: "YGX_ERR_CUDA",
    3: "YGX_ERR_TIMEOUT",
    4: "YGX_ERR_QUEUE_OVERFLOW",
    5: "YGX_ERR_FAR_OVERFLOW",
    6: "YGX_ERR_NEAR_OVERFLOW",
    7: "YGX_ERR_INT32_TOTAL",
    8: "YGX_ERR_MALFORMED",
    9: "YGX_ERR_TOO_LARGE",
}
FLAG_TIMEOUT = 1 << 0
FLAG_QUEUE_OVERFLOW = 1 << 1
FLAG_FAR_OVERFLOW = 1 << 2
FLAG_NEAR_OVERFLOW = 1 << 3
FLAG_MALFORMED = 1 << 4
FLAG_BAD_INPUT = 1 << 5
FLAG_LOG_OVERFLOW = 1 << 6
WALK_LOG = 0
TUNE = dict(sort_rank=0, sort_skew=1, walk_blocks=2, refit_warps=3, row_grid=4, sort_tile=5,
            spin_limit=6, target_budget=7, sort_bits=8)
WALK_COUNT = 1

TSTAT_WORDS = 16
TSTAT = dict(far_total=0, near_total=1, max_far=2, max_near=3, accept=4, near=5, refine=6,
             max_wf=7, gens=8, wf_need=9, log_need=10, ovf_rows=11, ovf_entries=12,
             ext_far=13, ext_near=14)

P = ctypes.c_void_p
I64 = ctypes.c_int64
I32 = ctypes.c_int
SZ = ctypes.c_size_t
F32 = ctypes.c_float
F64 = ctypes.c_double

# name -> (restype, argtypes)
_SIGS = {
    "ygx_workspace_init": (I32, [P, SZ, P]),
    "ygx_status_read": (I32, [P, P, P]),
    "ygx_launch_counter": (ctypes.c_uint64, []),
    "ygx_tune_set": (I32, [I32, I32]),
    "ygx_tune_get": (I32, [I32, P]),
    "ygx_bounds": (I32, [P, I64, P, P, SZ, P]),
    "ygx_morton_encode": (I32, [P, I64, P, P, P]),
    "ygx_encode_sort_workspace_size": (SZ, [I64]),
    "ygx_encode_sort": (I32, [P, I64, P, P, P, P, P, SZ, P]),
    "ygx_octree_box_geometry": (I32, [P, P, P, I32, I64, P, P, P, P, P, P, P]),
    "ygx_octree_walk_workspace_size": (SZ, [I64, I64]),
    "ygx_octree_walk": (I32, [P, P, I32, I64, P, P, P, P, P, P, I64, I64, I32, F32, F32, I64,
                              I64, I64, I64, I64, P, P, P, P, P, P, P, P, P, SZ, P]),
    "ygx_sort_pairs_workspace_size": (SZ, [I64]),
    "ygx_sort_pairs": (I32, [P, P, I64, I32, I32, P, P, P, SZ, P]),
    "ygx_sort_pairs_noalloc": (I32, [P, P, I64, I32, I32, P, P, P]),
    "ygx_sort_pairs_noalloc_status": (I32, [P, P]),
    "ygx_reorder": (I32, [P, P, P, I64, I32, P, P, P, P, P]),
    "ygx_pack_particles": (I32, [P, P, I64, P, P]),
    "ygx_reorder_packed": (I32, [P, P, I64, I32, P, P, P, P, P]),
    "ygx_leaves_adaptive": (I32, [P, I64, I64, I32, P, P, P, P, P]),
    "ygx_leaves_fixed": (I32, [P, I64, I32, I32, P, P, P, P, P]),
    "ygx_refine_workspace_size": (SZ, [I64]),
    "ygx_refine_count": (I32, [P, P, P, P, P, P, I64, I32, I32, F64, I32, I32, P, P, SZ, P]),
    "ygx_refine_emit": (I32, [P, P, P, P, P, P, I64, I32, I32, F64, I32, I32, P, P, P, P, P,
                              SZ, P]),
    "ygx_topology_workspace_size": (SZ, [I64]),
    "ygx_build_topology": (I32, [P, P, P, I64, I32] + [P] * 16 + [P, SZ, P]),
    "ygx_octree_workspace_size": (SZ, [I64]),
    "ygx_octree_tables": (I32, [P, I64, P, I64, P, P, I32, I32] + [P] * 15 + [P, SZ, P]),
    "ygx_geometry_workspace_size": (SZ, [I64]),
    "ygx_tree_geometry": (I32, [P, I64, I32, P, P, P, P, P, P, I64, I32, P, P, P, I64, P, P,
                                P, P, P, SZ, P]),
    "ygx_traverse_workspace_size": (SZ, [I64, I64, I64, I64]),
    "ygx_traverse_walk": (I32, [P, P, P, P, P, P, I64, I64, I32, F32, F32, I32, I32, I32, I64,
                                I64, P, P, P, SZ, P]),
    "ygx_traverse_fill_walk": (I32, [I64, I64, I32, F32, I32, I64, I64, I32, I64, I64, P, P, I32,
                                     I32, P, P, P, P, P, P, P, P, SZ, P]),
    "ygx_traverse_fill": (I32, [I64, I64, I64, I64, I64, I64, P, P, P, I32, I32, P, P, P, P, P,
                                P, P, P, SZ, P]),
    "ygx_traverse_pad_offsets": (I32, [I64, I64, I64, I64, P, P, P, P, SZ, P]),
    "ygx_traverse_walk_predicted": (I32, [P, P, P, P, P, P, I64, I64, I32, F32, F32, I32, I32,
                                          I64, I64, P, P, P, P, P, P, P, SZ, P]),
    "ygx_traverse_fill_predicted": (I32, [I64, I64, I64, I64, P, P, I64, I64, P, P, I32, I32, P,
                                          P, P, P, P, P, P, P, P, P, SZ, P]),
    "ygx_mlp_param_count": (I32, []),
    "ygx_mlp_workspace_size": (SZ, [I64]),
    "ygx_node_features": (I32, [P, P, P, P, P, I64, I64, P, I32, I32, F32, I32, P, P]),
    "ygx_mlp_forward": (I32, [P, P, I64, P, P]),
    "ygx_mlp_gradients": (I32, [P, P, P, P, I64, P, P, P, SZ, P]),
    "ygx_mlp_train_step": (I32, [P, P, P, I32, F32, P, P, P, I64, P, P, SZ, P]),
    "ygx_predict_caps": (I32, [P, P, P, P, P, P, I64, I64, P, I32, I32, F32, I32, P, F32, F32,
                               I32, P, P, P]),
    "ygx_layout_workspace_size": (SZ, [I64]),
    "ygx_counts_to_offsets": (I32, [P, I64, I32, P, P, SZ, P]),
    "ygx_node_order_far_rows": (I32, [I64, P, P, P, I32, P, P, P, P, SZ, P]),
    "ygx_flag_compact": (I32, [P, I64, I64, I32, P, P, P, P, SZ, P]),
    "ygx_dense_row_table": (I32, [P, P, I64, P, P, I64, I32, I64, P, P]),
    "ygx_gather_index": (I32, [P, I64, P, I64, I32, P, P, SZ, P]),
    "ygx_scatter_positions": (I32, [P, I32, I64, I64, P, I32, P, SZ, P]),
    "ygx_target_walk_workspace_size": (SZ, [I64, I64, P, I32]),
    "ygx_target_walk": (I32, [P, P, P, P, P, P, P, P, P, I64, I64, I32, I32, F32, F32, P, I32,
                              P, P, P, P, P, P, P, I32, I32, P, P, P, P, SZ, P]),
    "ygx_target_pad_workspace_size": (SZ, [I64, I64]),
    "ygx_target_pad": (I32, [I64, I64, P, P, P, P, P, P, SZ, P]),
    "ygx_target_walk_lists": (I32, [I64, I64, P, I32, P, P, P, P, P, I64, P, I64, P, P, P, I32, I32,
                                    I64, I64, ctypes.c_uint64,
                                    ctypes.c_uint64, P, P, P, P, P, P, P, P, P, P, I64, P, P,
                                    SZ, P]),
    "ygx_traverse_finalize": (I32, [I64, I64, I64, I64, P, P, I32, P, P, P, P, P, P, P, P, P, P,
                                    P, I64, P, SZ, P]),
    "ygx_batch_encode_sort_workspace_size": (SZ, [I64]),
    "ygx_batch_encode_sort": (I32, [P, I64, P, I64, P, P, P, P, P, SZ, P]),
    "ygx_batch_reorder": (I32, [P, P, P, P, P, I64, I32, P, P, P, P, P]),
    "ygx_batch_leaf_offsets_workspace_size": (SZ, [I64]),
    "ygx_batch_leaf_offsets": (I32, [P, I64, I64, P, P, P, SZ, P]),
    "ygx_batch_leaves": (I32, [P, P, P, I64, I64, I64, I32, P, P, P, P, P, P]),
    "ygx_batch_topology_workspace_size": (SZ, [I64, I64]),
    "ygx_batch_build_topology": (I32, [P, P, P, P, P, I64, I64, I32] + [P] * 22 + [SZ, P]),
    "ygx_batch_tree_geometry": (I32, [P, I64, I64, P, P, I64, P, I32, P, P, P, P, P, P, I64, P, P,
                                      P, P, P, SZ, P]),
    "ygx_level_major_geometry": (I32, [P, P, I32, I32, I64, P, P, P, P, P, P, P, P, P, P]),
    "ygx_dense_m2l": (I32, [P, I32, I64, I64, P, P, P, P, I64, P, P, P, P, P]),
    "ygx_grouped_workspace_size": (SZ, [I64]),
    "ygx_grouped_classes": (I32, [P, P, I32, I64, P, P, P, P, P, SZ, P]),
    "ygx_grouped_emit": (I32, [P, P, I32, I64, P, P, P, P, P, P, P, P, SZ, P]),
    "ygx_moments_workspace_size": (SZ, [I64, I32]),
    "ygx_tree_moments": (I32, [P, P, I64, P, I32, I64, I32] + [P] * 13 + [SZ, P]),
    "ygx_mutual_walk_workspace_size": (SZ, [I64, I64]),
    "ygx_mutual_walk": (I32, [P, P, I32, P, P, I64, F32, I64, I64, I64, I64, P, P, P, P, P, P, P,
                              P, SZ, P]),
    "ygx_batch_traverse_lists": (I32, [P] * 11 + [I64, P, I64, P, I32, F32, F32, I32, I64, I64,
                                               I64, I64, I32] + [P] * 11 + [SZ, P]),
    "ygx_traverse_stats_read": (I32, [I64, I64, I64, I64, P, SZ, P, P, P]),
    "ygx_batch_traverse_walk": (I32, [P, P, P, P, P, P, P, I64, P, I64, P, I32, F32, F32, I32,
                                      I64, I64, P, P, P, SZ, P]),
}

_lib: Optional[ctypes.CDLL] = None


class YgxError(RuntimeError):
    """A libygx entry point returned an error code."""


def lib() -> ctypes.CDLL:
    """Load ``libygx.so`` (raises if it is missing -- no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libygx.so not found at {LIB_PATH}; build it with "
            "`python -m yggdrax_b200.build_ext` (the CUDA path has no CPU fallback)")
    h = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(h, name)
        fn.restype = res
        fn.argtypes = args
    _lib = h
    return h


def exported_symbols() -> list:
    return sorted(_SIGS)


def ptr(t: Optional[torch.Tensor]):
    """Device pointer of a tensor (None -> NULL)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream_handle(device: torch.device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def check(rc: int, what: str) -> None:
    if rc != YGX_OK:
        raise YgxError(f"{what} failed: {ERROR_NAMES.get(rc, rc)}")


def require_cuda(t: torch.Tensor, what: str = "input") -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("yggdrax_b200 requires a CUDA device (no CPU fallback)")
    if not t.is_cuda:
        raise ValueError(f"{what} must be a CUDA tensor")
    return t.device


def workspace(nbytes: int, device: torch.device) -> torch.Tensor:
    """Device workspace with a zeroed status header."""
    ws = torch.empty(max(int(nbytes), 512), dtype=torch.uint8, device=device)
    ws[:512].zero_()
    return ws


def read_status(ws: torch.Tensor) -> int:
    """Synchronously read the device status word at the start of ``ws``."""
    return int(ws[:4].view(torch.int32).item()) & 0xFFFFFFFF

"""Index dtype policy (mirrors yggdrax/dtypes.py:12-35).

``YGGDRAX_INDEX_PRECISION`` (falling back to ``JACCPOT_INDEX_PRECISION``)
selects int32 or int64 index outputs; int64 is the default.
"""

from __future__ import annotations

import os

import torch


def _resolve_index_dtype() -> torch.dtype:
    raw = os.environ.get("YGGDRAX_INDEX_PRECISION")
    if raw is None:
        raw = os.environ.get("JACCPOT_INDEX_PRECISION", "int64")
    raw_norm = str(raw).strip().lower()
    if raw_norm in ("int32", "i32", "32"):
        return torch.int32
    return torch.int64


INDEX_DTYPE: torch.dtype = _resolve_index_dtype()
INDEX_BITS: int = 32 if INDEX_DTYPE == torch.int32 else 64


def as_index(x, device=None) -> torch.Tensor:
    """Convert a scalar/array to the index dtype."""
    return torch.as_tensor(x, dtype=INDEX_DTYPE, device=device)


__all__ = ["INDEX_DTYPE", "INDEX_BITS", "as_index"]

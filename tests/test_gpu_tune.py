"""Launch-shape knobs change speed, never results: the full pipeline (sort,
build, geometry, walk, finalize) gives bit-identical outputs under every
legal setting of each knob, the single-set and the batched path alike, and
illegal values are rejected."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SETTINGS = [
    ("sort_rank", 1), ("sort_rank", 2), ("sort_skew", 1), ("sort_skew", 256),
    ("walk_blocks", 2), ("walk_blocks", 5), ("refit_warps", 2), ("refit_warps", 4),
    ("row_grid", 4), ("row_grid", 32), ("sort_tile", 1), ("sort_tile", 2), ("sort_tile", 3),
    ("sort_bits", 11),
]


def _run(P, M):
    import yggdrax_b200 as yb

    t, ps, ms, inv = yb.build_tree(P, M, leaf_size=16, return_reordered=True)[:4]
    g = yb.compute_tree_geometry(t, ps)
    fi, ni = yb.build_interactions_and_neighbors(t, g, theta=0.6, mac_type="dehnen")
    out = [t.particle_indices, t.morton_codes, t.parent, t.node_ranges, t.nodes_by_level,
           inv, g.center, g.radius, g.max_extent, fi.offsets, fi.sources, fi.targets,
           fi.target_levels, ni.offsets, ni.neighbors]
    return [o.detach().cpu().numpy().copy() for o in out]


def _same(a, b):
    return all(x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8))
               for x, y in zip(a, b))


def test_knobs_do_not_change_results(cuda_device):
    import torch

    from yggdrax_b200 import _lib as L
    from yggdrax_b200 import autotune, inputs

    lib = L.lib()
    pos, mass = inputs.plummer(150_000, 17)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)
    defaults = autotune.current()
    try:
        ref = _run(P, M)
        for knob, v in SETTINGS:
            autotune.apply(dict(defaults, **{knob: v}))
            assert _same(_run(P, M), ref), (knob, v)
            autotune.apply(defaults)
    finally:
        autotune.apply(defaults)
    assert lib.ygx_tune_set(L.TUNE["walk_blocks"], 7) == 1  # YGX_ERR_ARG
    assert lib.ygx_tune_set(99, 1) == 1
    assert autotune.current() == defaults


def test_batched_path_under_knobs(cuda_device):
    import torch

    from yggdrax_b200 import autotune, inputs
    from yggdrax_b200 import batch as B

    pos, mass, off = inputs.batched_sets(40, 9, lo=16, hi=6000)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)

    def run():
        bt = B.build_trees_batched(P, M, off, leaf_size=16)
        bg = B.compute_tree_geometry_batched(bt)
        bi = B.build_interactions_and_neighbors_batched(bt, bg, theta=0.6, mac_type="dehnen")
        return [x.cpu().numpy().copy() for x in (bt.particle_indices, bt.parent, bg.radius,
                                                  bi.node_offsets, bi.sources, bi.neighbors)]

    defaults = autotune.current()
    try:
        ref = run()
        for knob, v in (("walk_blocks", 2), ("sort_rank", 1), ("refit_warps", 2),
                        ("sort_tile", 3), ("sort_bits", 11)):
            autotune.apply(dict(defaults, **{knob: v}))
            assert _same(run(), ref), (knob, v)
            autotune.apply(defaults)
    finally:
        autotune.apply(defaults)

"""The padded single-pass configuration (``traversal_config``) on the GPU.

The reference runs one padded walk when a ``DualTreeTraversalConfig`` is
given (_dual_tree_walk_impl, _interactions_impl.py:1119-1905; runner
:4306-4440).  Its lists are the same pair sets as the count-then-fill
schedule, and its ``DualTreeWalkResult`` carries queue / far / near overflow
flags that eager calls turn into RuntimeErrors and traced calls return
(:4417-4421).  Checked here:

* the lists equal the fixtures made by the reference's own padded walk
  (``padded_dehnen_*`` in tests/golden, DualTreeTraversalConfig(4096, 64,
  256, 256)), bit for bit, with every overflow flag False;
* the 65,536-particle uniform configuration with
  DualTreeTraversalConfig(65536, 256, 2048, 2048) equals the oracle, lists and
  decision counts;
* with the reference limits off, capacities the walk outgrows set exactly the
  matching flags while the lists stay exact.
"""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _np(t):
    return t.detach().cpu().numpy()


def _flags(res):
    return bool(res.queue_overflow), bool(res.far_overflow), bool(res.near_overflow)


@pytest.mark.parametrize("fname,leaf", [("adaptive_uniform300_leaf4.npz", 4),
                                        ("adaptive_plummer400_leaf8.npz", 8)])
def test_padded_walk_matches_reference_fixture(cuda_device, fname, leaf):
    import torch

    import yggdrax_b200 as yb
    from test_gpu_parity import _assert_eq

    g = dict(np.load(os.path.join(GOLD, fname)))
    P = torch.from_numpy(g["pos"]).to(cuda_device)
    M = torch.from_numpy(g["mass"]).to(cuda_device)
    gt, ps = yb.build_tree(P, M, leaf_size=leaf, return_reordered=True)[:2]
    gg = yb.compute_tree_geometry(gt, ps)
    cfg = yb.DualTreeTraversalConfig(max_pair_queue=4096, process_block=64,
                                     max_interactions_per_node=256, max_neighbors_per_leaf=256)
    gi, gn, res = yb.build_interactions_and_neighbors(gt, gg, theta=0.6, mac_type="dehnen",
                                                      traversal_config=cfg, return_result=True)
    p = "padded_dehnen_"
    _assert_eq("far_counts", _np(gi.counts), g[p + "far_counts"])
    _assert_eq("far_offsets", _np(gi.offsets), g[p + "far_offsets"])
    _assert_eq("far_sources", _np(gi.sources), g[p + "far_sources"])
    _assert_eq("far_targets", _np(gi.targets), g[p + "far_targets"])
    _assert_eq("far_level_offsets", _np(gi.level_offsets), g[p + "far_level_offsets"])
    _assert_eq("far_target_levels", _np(gi.target_levels), g[p + "far_target_levels"])
    _assert_eq("near_counts", _np(gn.counts), g[p + "near_counts"])
    _assert_eq("near_offsets", _np(gn.offsets), g[p + "near_offsets"])
    _assert_eq("near_neighbors", _np(gn.neighbors), g[p + "near_neighbors"])
    _assert_eq("near_leaf_indices", _np(gn.leaf_indices), g[p + "near_leaf_indices"])
    _assert_eq("near_po_to_native", _np(gn.particle_order_to_native_leaf),
               g[p + "near_po_to_native"])
    assert _flags(res) == (False, False, False)


def test_uniform_65k_traversal_config_matches_oracle(cuda_device, oracle):
    """N=65,536 uniform in [-1,1]^3, masses U[0.5,1.5], seed 0; radix leaf 16;
    dehnen theta 0.6 with DualTreeTraversalConfig(65536, 256, 2048, 2048)."""
    import torch

    import yggdrax_b200 as yb
    from test_gpu_parity import _compare_lists
    from yggdrax_b200 import inputs

    pos, mass = inputs.uniform_cube(65536, 0)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)
    gt, ps = yb.build_tree(P, M, leaf_size=16, return_reordered=True)[:2]
    gg = yb.compute_tree_geometry(gt, ps)
    cfg = yb.DualTreeTraversalConfig(65536, 256, 2048, 2048)
    gi, gn, res = yb.build_interactions_and_neighbors(gt, gg, theta=0.6, mac_type="dehnen",
                                                      traversal_config=cfg, return_result=True)
    ot = oracle.build_tree(pos, mass, leaf_size=16)
    og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
    r = oracle.build_interactions_and_neighbors(ot, og, theta=0.6, mac_type="dehnen")
    _compare_lists(gi, gn, r)
    assert int(res.accept_decisions) == r["accept_decisions"]
    assert int(res.near_decisions) == r["near_decisions"]
    assert int(res.refine_decisions) == r["refine_decisions"]
    assert _flags(res) == (False, False, False)
    # the raw payload: node-order rows with ascending sources, -1 tags
    counts = r["far_counts"]
    no = np.concatenate([[0], np.cumsum(counts)])
    _assert = np.testing.assert_array_equal
    _assert(_np(res.interaction_offsets), no)
    _assert(_np(res.interaction_targets), np.repeat(np.arange(counts.shape[0]), counts))
    assert int(res.far_pair_count) == int(counts.sum())
    assert int(res.near_pair_count) == int(r["near_counts"].sum())


def test_overflow_flags_with_reference_limits_off(cuda_device, oracle):
    """Capacities below what the walk needs: the reference raises in eager
    mode (checked elsewhere); with the limits off the result carries the
    flags its padded walk would set, and the lists stay exact."""
    import torch

    import yggdrax_b200 as yb
    from test_gpu_parity import _compare_lists
    from yggdrax_b200 import inputs

    pos, mass = inputs.uniform_cube(20000, 5)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)
    gt, ps = yb.build_tree(P, M, leaf_size=16, return_reordered=True)[:2]
    gg = yb.compute_tree_geometry(gt, ps)
    ot = oracle.build_tree(pos, mass, leaf_size=16)
    og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
    r = oracle.build_interactions_and_neighbors(ot, og, theta=0.6, mac_type="dehnen")
    max_far = int(r["far_counts"].max())
    cases = [
        (yb.DualTreeTraversalConfig(1 << 20, 256, max_far, 2048), (False, False, False)),
        (yb.DualTreeTraversalConfig(1 << 20, 256, max_far - 1, 2048), (False, True, False)),
        (yb.DualTreeTraversalConfig(4, 1, 1 << 20, 2048), None),  # queue: depends on ladder
    ]
    yb.set_reference_limits(False)
    try:
        for cfg, want in cases:
            gi, gn, res = yb.build_interactions_and_neighbors(
                gt, gg, theta=0.6, mac_type="dehnen", traversal_config=cfg, return_result=True)
            _compare_lists(gi, gn, r)
            got = _flags(res)
            if want is not None:
                assert got == want, (cfg, got)
            else:
                # the queue ladder grows to the automatic candidates of the
                # tree size (:296-316, :450-485); flagged only past them
                assert got[1:] == (False, False)
    finally:
        yb.set_reference_limits(True)
    with pytest.raises(RuntimeError, match="Interaction list capacity exceeded"):
        yb.build_interactions_and_neighbors(gt, gg, theta=0.6, mac_type="dehnen",
                                            traversal_config=cases[1][0])

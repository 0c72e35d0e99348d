"""The per-target walk (traversal modes "target" and "target_ordered")
against the oracle.

One warp per target node walks that node's pairs of the reference's
symmetric walk (ygx_target_walk): in Morton order ("target_ordered", rows
ascending straight from the walk) or emitting every resolved pair at once
("target", rows sorted afterwards).  Its rows must equal the oracle's bit for
bit -- offsets, counts, level-major far rows, leaf-order near rows -- and its
decision counts, largest wavefront and generation count must equal what the
generation-by-generation walk reports.  The hand-off of long expansions to
other warps is exercised by a budget of one step per piece, and the capacity
re-run by starting from capacities far too small.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _build(yb, kind, P, M, leaf):
    if kind == "radix":
        return yb.build_tree(P, M, leaf_size=leaf, return_reordered=True)[:2]
    if kind == "octree":
        return yb.build_octree(P, M, leaf_size=leaf, return_reordered=True)[:2]
    return yb.build_fixed_depth_octree(P, M, target_leaf_particles=leaf, return_reordered=True)[:2]


def _obuild(oracle, kind, pos, mass, leaf):
    if kind == "radix":
        return oracle.build_tree(pos, mass, leaf_size=leaf)
    if kind == "octree":
        return oracle.build_octree(pos, mass, leaf_size=leaf)
    return oracle.build_fixed_depth_octree(pos, mass, target_leaf_particles=leaf)


MODES = ("target", "target_ordered")


def _run(yb, gt, gg, theta, mac, budget=None, mode="target"):
    from yggdrax_b200 import _lib as L
    from yggdrax_b200.interactions import LAST_WALK_STATS

    lib = L.lib()
    old = np.zeros(1, np.int32)
    L.check(lib.ygx_tune_get(L.TUNE["target_budget"], old.ctypes.data), "ygx_tune_get")
    if budget is not None:
        L.check(lib.ygx_tune_set(L.TUNE["target_budget"], budget), "ygx_tune_set")
    prev = yb.get_traversal_mode()
    yb.set_traversal_mode(mode)
    try:
        gi, gn, res = yb.build_interactions_and_neighbors(gt, gg, theta=theta, mac_type=mac,
                                                          return_result=True)
        stats = dict(LAST_WALK_STATS)
    finally:
        yb.set_traversal_mode(prev)
        L.check(lib.ygx_tune_set(L.TUNE["target_budget"], int(old[0])), "ygx_tune_set")
    return gi, gn, res, stats


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("case,kind,leaf,mac,theta,budget", [
    ("uniform65k", "radix", 16, "dehnen", 0.6, None),
    ("uniform65k", "radix", 16, "bh", 0.5, None),
    ("uniform65k", "radix", 16, "dehnen", 0.6, 1),
    ("plummer40k", "octree", 32, "dehnen", 0.6, None),
    ("plummer40k", "octree", 32, "engblom", 0.5, 2),
    ("clumps30k", "fixed_octree", 16, "dehnen", 0.6, None),
    ("small17", "radix", 4, "bh", 0.5, None),
    ("collinear128", "radix", 4, "dehnen", 0.6, None),
    ("dup64", "radix", 4, "dehnen", 0.6, None),  # tied codes: served by the log walk
])
def test_target_walk_matches_oracle(cuda_device, oracle, case, kind, leaf, mac, theta, budget,
                                    mode):
    import yggdrax_b200 as yb
    from test_gpu_parity import BOUNDS, CASES, _assert_eq, _compare_lists, _to_dev

    pos, mass = CASES[case]
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    del BOUNDS
    gt, ps = _build(yb, kind, P, M, leaf)
    gg = yb.compute_tree_geometry(gt, ps)
    gi, gn, res, st = _run(yb, gt, gg, theta, mac, budget, mode)
    ot = _obuild(oracle, kind, pos, mass, leaf)
    og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
    r = oracle.build_interactions_and_neighbors(ot, og, theta=theta, mac_type=mac)
    _compare_lists(gi, gn, r)
    assert int(res.accept_decisions) == r["accept_decisions"]
    assert int(res.near_decisions) == r["near_decisions"]
    assert int(res.refine_decisions) == r["refine_decisions"]
    assert st["max_wf"] == r["max_wf"] and st["gens"] == r["generations"], (st, r["max_wf"])
    nlp = oracle.neighbor_leaf_positions(r["leaf_indices"], r["near_offsets"],
                                         r["near_counts"], r["neighbors"],
                                         ot.node_ranges.shape[0])
    _assert_eq("neighbor_leaf_positions", _np(gn.neighbor_leaf_positions), nlp)
    if case != "dup64" and budget == 1:
        assert st["continuation_pieces"] > 0


@pytest.mark.parametrize("mode", MODES)
def test_target_walk_capacities_grow_on_overflow(cuda_device, mode):
    """Capacities far too small: the walk reports what it needed and the
    re-run returns the same lists as a walk sized right."""
    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs
    from yggdrax_b200 import interactions as I
    from test_gpu_parity import _to_dev

    pos, mass = inputs.plummer(300_000, 13)
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    gt, ps = yb.build_tree(P, M, leaf_size=16, return_reordered=True)[:2]
    gg = yb.compute_tree_geometry(gt, ps)
    total = int(gt.parent.shape[0])
    key = I._hint_key("dehnen", 0.6, total, mode)
    I._TARGET_HINTS[key] = [1e-6] * 8  # next walk starts from tiny capacities
    a, an, _, st = _run(yb, gt, gg, 0.6, "dehnen", mode=mode)
    assert st["walk_runs"] > 1
    b, bn, _, st2 = _run(yb, gt, gg, 0.6, "dehnen", mode=mode)
    assert st2["walk_runs"] == 1
    for f in ("offsets", "counts", "sources", "targets", "level_offsets", "target_levels"):
        np.testing.assert_array_equal(_np(getattr(a, f)), _np(getattr(b, f)), err_msg=f)
    for f in ("offsets", "counts", "neighbors"):
        np.testing.assert_array_equal(_np(getattr(an, f)), _np(getattr(bn, f)), err_msg=f)


@pytest.mark.parametrize("mode", MODES)
def test_target_walk_4m_plummer_matches_log_walk(cuda_device, mode):
    """4M Plummer sphere (the heavy halo leaves are split over many warps):
    the target walk and the log walk return identical lists."""
    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs
    from test_gpu_parity import _to_dev

    pos, mass = inputs.plummer(1 << 22, 1)
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    gt, ps = yb.build_tree(P, M, leaf_size=32, return_reordered=True)[:2]
    gg = yb.compute_tree_geometry(gt, ps)
    yb.set_reference_limits(False)
    try:
        a, an, ares, _ = _run(yb, gt, gg, 0.6, "dehnen", mode=mode)
        b, bn, bres, st = _run(yb, gt, gg, 0.6, "dehnen", mode="log")
        assert st["mode"] == "log"
    finally:
        yb.set_reference_limits(True)
    for f in ("offsets", "counts", "sources", "targets", "level_offsets", "target_levels"):
        assert np.array_equal(_np(getattr(a, f)), _np(getattr(b, f))), f
    for f in ("offsets", "counts", "neighbors"):
        assert np.array_equal(_np(getattr(an, f)), _np(getattr(bn, f))), f
    assert int(ares.refine_decisions) == int(bres.refine_decisions)

"""The reference's hot-path test properties (tests/test_tree.py,
test_tree_geometry.py, test_tree_interactions.py, test_octree_topology.py,
test_morton.py of yggdrax), re-expressed against the CPU oracle: sorted codes, stable ties, parent/child consistency,
DFS leaf order, node counts, fixed-depth shape, geometry clamps, MAC
consistency and symmetry of the lists."""

import numpy as np
import pytest


def _uniform(n, seed=0):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, (n, 3)).astype(np.float32), np.ones(n, np.float32)


def test_sorted_codes_and_node_counts(oracle):
    pos, m = _uniform(1000)
    for leaf in (1, 7, 32):
        t = oracle.build_tree(pos, m, leaf_size=leaf)
        assert np.all(np.diff(t.morton_codes.astype(np.float64)) >= 0)
        L = -(-1000 // leaf)
        assert t.num_internal_nodes == L - 1
        assert t.parent.shape[0] == 2 * L - 1


def test_identical_points_keep_identity_order(oracle):
    pos = np.zeros((8, 3), np.float32)
    t = oracle.build_tree(pos, np.ones(8, np.float32), leaf_size=1)
    np.testing.assert_array_equal(t.particle_indices, np.arange(8))


def test_parent_child_consistency_and_dfs_order(oracle):
    pos, m = _uniform(777, 3)
    t = oracle.build_tree(pos, m, leaf_size=1)
    ni = t.num_internal_nodes
    for i in range(ni):
        assert t.parent[t.left_child[i]] == i and t.parent[t.right_child[i]] == i
        assert bool(t.left_is_leaf[i]) == (t.left_child[i] >= ni)
    assert (t.parent < 0).sum() == 1 and t.parent[0] == -1
    stack, leaves = [0], []
    while stack:
        v = stack.pop()
        if v >= ni:
            leaves.append(v - ni)
        else:
            stack += [t.right_child[v], t.left_child[v]]
    assert leaves == list(range(777))


def test_fixed_depth_shape_and_morton_cells_contain_particles(oracle):
    pos, m = _uniform(4096, 5)
    t = oracle.build_fixed_depth_tree(pos, m, target_leaf_particles=8, refine_local=False)
    d = t.extras["resolved_depth"]
    assert t.leaf_depths.shape[0] == 8 ** d and np.all(t.leaf_depths == d)
    g = oracle.compute_tree_geometry(t, t.positions_sorted)
    ni = t.num_internal_nodes
    for j in range(0, 8 ** d, 37):
        s, e = t.node_ranges[ni + j]
        if e < s:
            continue
        pts = t.positions_sorted[s: e + 1]
        lo = g.center[ni + j] - g.half_extent[ni + j]
        hi = g.center[ni + j] + g.half_extent[ni + j]
        assert np.all(pts >= lo - 1e-5) and np.all(pts <= hi + 1e-5)


def test_refinement_only_deepens(oracle):
    rng = np.random.default_rng(9)
    pos = np.concatenate([rng.normal(0, [1, 0.01, 0.01], (500, 3))]).astype(np.float32)
    a = oracle.build_fixed_depth_tree(pos, np.ones(500, np.float32), target_leaf_particles=8,
                                      refine_local=False)
    b = oracle.build_fixed_depth_tree(pos, np.ones(500, np.float32), target_leaf_particles=8,
                                      refine_local=True)
    assert b.leaf_depths.min() >= a.leaf_depths.min()
    assert b.leaf_depths.shape[0] >= a.leaf_depths.shape[0]


def test_geometry_clamp_and_root_span(oracle):
    pos = np.zeros((5, 3), np.float32)
    t = oracle.build_tree(pos, np.ones(5, np.float32), leaf_size=8)
    g = oracle.compute_tree_geometry(t, t.positions_sorted)
    np.testing.assert_array_equal(g.half_extent, np.full((1, 3), np.float32(1e-6)))
    pos, m = _uniform(300, 1)
    t = oracle.build_tree(pos, m, leaf_size=4)
    g = oracle.compute_tree_geometry(t, t.positions_sorted)
    assert np.all(g.center[0] - g.half_extent[0] <= pos.min(0) + 1e-6)
    assert np.all(g.center[0] + g.half_extent[0] >= pos.max(0) - 1e-6)


@pytest.mark.parametrize("mac,theta", [("bh", 0.5), ("dehnen", 0.6), ("engblom", 0.5)])
def test_lists_symmetric_and_mac_consistent(oracle, mac, theta):
    pos, m = _uniform(3000, 2)
    t = oracle.build_tree(pos, m, leaf_size=8)
    g = oracle.compute_tree_geometry(t, t.positions_sorted)
    r = oracle.build_interactions_and_neighbors(t, g, theta=theta, mac_type=mac)
    src, tgt = r["sources"], r["targets"]
    pairs = set(zip(tgt.tolist(), src.tolist()))
    assert all((s, t_) in pairs for t_, s in pairs)  # symmetry
    ext = oracle.mac_extents(t, g, mac)
    th2 = np.float32(theta) * np.float32(theta)
    d = (g.center[tgt] - g.center[src]).astype(np.float32)
    d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    if mac == "engblom":
        big = np.maximum(ext[tgt], ext[src])
        small = np.minimum(ext[tgt], ext[src])
        lhs = big + np.sqrt(th2) * small
        assert np.all(lhs * lhs <= th2 * d2)
    else:
        s_ = ext[tgt] + ext[src]
        assert np.all(s_ * s_ <= th2 * d2)
    # level-major order of targets
    assert np.all(np.diff(r["target_levels"]) >= 0)
    # no node interacts with itself or an ancestor
    ni = t.num_internal_nodes
    for v, w in zip(tgt[:2000], src[:2000]):
        x = v
        while x >= 0:
            assert x != w
            x = t.parent[x]
    # near lists: leaves only, every leaf pair not accepted
    nb = r["neighbors"]
    assert np.all(nb >= ni)

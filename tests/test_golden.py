"""Pin the CPU oracle to the reference: golden fixtures in tests/golden were
produced by running the reference yggdrax source (over a NumPy stand-in for
jax, see tests/golden/make_golden.py).  Every output must match exactly;
list rows are compared in ascending order (the reference's within-row order
is unspecified)."""

import glob
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

TREE_FIELDS = ["parent", "left_child", "right_child", "left_is_leaf", "right_is_leaf",
               "particle_indices", "morton_codes", "node_ranges", "node_level", "level_offsets",
               "nodes_by_level", "bounds_min", "bounds_max", "leaf_codes", "leaf_depths"]
OCT_FIELDS = ["oct_parent", "oct_children", "oct_child_counts", "oct_child_mask",
              "oct_valid_mask", "oct_node_codes", "oct_node_depths", "oct_node_ranges",
              "oct_nodes_by_level", "oct_level_offsets", "oct_leaf_mask", "oct_leaf_nodes",
              "radix_node_to_oct", "radix_leaf_to_oct"]


def _eq(name, got, want):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape, f"{name}: shape {got.shape} vs {want.shape}"
    if want.dtype.kind == "f":
        assert np.array_equal(got.astype(want.dtype).view(np.uint32 if want.dtype == np.float32
                                                           else np.uint64),
                              want.view(np.uint32 if want.dtype == np.float32 else np.uint64)), name
    else:
        assert np.array_equal(got.astype(want.dtype), want), name


def _load(name):
    return dict(np.load(os.path.join(GOLD, name)))


def test_fixtures_present():
    assert len(glob.glob(os.path.join(GOLD, "*.npz"))) >= 14


def test_morton_and_order_match_reference(oracle):
    g = _load("morton.npz")
    for name in ("uniform300", "plummer400", "clumps600"):
        pos = g[f"{name}_pos"]
        bmin, bmax = oracle.infer_bounds(pos)
        _eq(f"{name}.bmin", bmin, g[f"{name}_bmin"])
        _eq(f"{name}.bmax", bmax, g[f"{name}_bmax"])
        codes = oracle.morton_encode(pos, (bmin, bmax))
        _eq(f"{name}.codes", codes, g[f"{name}_codes"])
        _eq(f"{name}.order", oracle.stable_argsort_u64(codes, 63), g[f"{name}_order"])
    pos = g["collinear128_pos"]
    codes = oracle.morton_encode(pos, (np.array([-10, -1, -1], np.float32),
                                       np.array([10, 1, 1], np.float32)))
    _eq("collinear.codes", codes, g["collinear128_codes"])


def _check_tree(t, g):
    for f in TREE_FIELDS:
        _eq(f, getattr(t, f), g[f])
    assert int(t.num_levels) == int(g["num_levels"])
    assert t.num_internal_nodes == int(g["num_internal_nodes"])
    _eq("positions_sorted", t.positions_sorted, g["positions_sorted"])
    _eq("masses_sorted", t.masses_sorted, g["masses_sorted"])
    _eq("inverse", t.inverse_permutation, g["inverse"])


def _check_geometry(geo, g):
    for f in ("center", "half_extent", "radius", "max_extent"):
        _eq(f"geom.{f}", getattr(geo, f), g[f"geom_{f}"])


def _check_octree(t, g, oracle):
    meta = oracle.octree_metadata(t)
    for f in OCT_FIELDS:
        _eq(f, meta[f], g[f])
    assert meta["oct_num_levels"] == int(g["oct_num_levels"])
    return meta


def _check_walk(prefix, t, geo, g, oracle, theta, mac):
    r = oracle.build_interactions_and_neighbors(t, geo, theta=theta, mac_type=mac)
    _eq(prefix + "far_counts", r["far_counts"], g[prefix + "far_counts"])
    _eq(prefix + "far_offsets", r["offsets"], g[prefix + "far_offsets"])
    _eq(prefix + "far_sources", r["sources"], g[prefix + "far_sources"])
    _eq(prefix + "far_targets", r["targets"], g[prefix + "far_targets"])
    _eq(prefix + "far_level_offsets", r["level_offsets"], g[prefix + "far_level_offsets"])
    _eq(prefix + "far_target_levels", r["target_levels"], g[prefix + "far_target_levels"])
    _eq(prefix + "near_counts", r["near_counts"], g[prefix + "near_counts"])
    _eq(prefix + "near_offsets", r["near_offsets"], g[prefix + "near_offsets"])
    _eq(prefix + "near_neighbors", r["neighbors"], g[prefix + "near_neighbors"])
    _eq(prefix + "near_leaf_indices", r["leaf_indices"], g[prefix + "near_leaf_indices"])
    _eq(prefix + "near_po_to_native", r["particle_order_to_native_leaf"],
        g[prefix + "near_po_to_native"])


@pytest.mark.parametrize("fname,leaf", [("adaptive_uniform300_leaf4.npz", 4),
                                        ("adaptive_uniform300_leaf1.npz", 1),
                                        ("adaptive_plummer400_leaf8.npz", 8),
                                        ("adaptive_dup16_leaf1.npz", 1),
                                        ("adaptive_dup16_leaf4.npz", 4)])
def test_adaptive_pipeline_matches_reference(oracle, fname, leaf):
    g = _load(fname)
    t = oracle.build_tree(g["pos"], g["mass"], leaf_size=leaf)
    _check_tree(t, g)
    geo = oracle.compute_tree_geometry(t, t.positions_sorted, max_leaf_size=leaf)
    _check_geometry(geo, g)
    _check_octree(t, g, oracle)
    if "walk_dehnen_far_counts" in g:
        for theta, mac in ((0.6, "dehnen"), (0.5, "bh"), (0.5, "engblom")):
            _check_walk(f"walk_{mac}_", t, geo, g, oracle, theta, mac)
        # padded (traversal_config) walk: same pair sets
        _check_walk("padded_dehnen_", t, geo, g, oracle, 0.6, "dehnen")
        tt = oracle.build_octree(g["pos"], g["mass"], leaf_size=leaf)
        _check_walk("walkoct_dehnen_", tt, geo, g, oracle, 0.6, "dehnen")


@pytest.mark.parametrize("fname", sorted(os.path.basename(p) for p in
                                         glob.glob(os.path.join(GOLD, "fixed_*.npz"))))
def test_fixed_depth_pipeline_matches_reference(oracle, fname):
    g = _load(fname)
    refine = "_refine" in fname
    target = int(fname.split("_t")[1].split("_")[0])
    bounds = (g["bmin_in"], g["bmax_in"])
    t = oracle.build_fixed_depth_tree(g["pos"], g["mass"], bounds, target_leaf_particles=target,
                                      refine_local=refine)
    _check_tree(t, g)
    geo = oracle.compute_tree_geometry(t, t.positions_sorted)
    _check_geometry(geo, g)
    meta = _check_octree(t, g, oracle)
    if "walkoct_dehnen_far_counts" in g:
        t.octree = meta
        _check_walk("walkoct_dehnen_", t, geo, g, oracle, 0.6, "dehnen")


@pytest.mark.parametrize("depth", [1, 2])
def test_refinement_matches_reference_numpy(oracle, depth):
    g = _load(f"refine_d{depth}.npz")
    out = oracle.refine_partitions(g["pos_sorted"], g["sorted_codes"], g["starts"], g["ends"],
                                   g["codes"], g["depths"], depth)
    for got, key in zip(out, ("out_starts", "out_ends", "out_codes", "out_depths")):
        _eq(key, got, g[key])

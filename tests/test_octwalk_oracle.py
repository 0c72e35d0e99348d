"""The native octree walk oracle against golden fixtures made by running the
reference's own build_explicit_octree_traversal_view,
build_octree_native_far_pairs and build_octree_native_neighbor_lists
(tests/golden/make_golden.py --octwalk-only) on adaptive and fixed-depth
octrees: box geometry and cell maps equal; far targets, near offsets /
counts / leaf tables equal; rows equal as sets (the reference orders the
entries of one row within a generation block by an unstable argsort); and
the same RuntimeError where a far row, a near row or the queue overflows."""

import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "octwalk_*.npz")))
OCT_FIELDS = ["oct_parent", "oct_children", "oct_child_counts", "oct_child_mask",
              "oct_valid_mask", "oct_node_codes", "oct_node_depths", "oct_node_ranges",
              "oct_nodes_by_level", "oct_level_offsets", "oct_num_levels", "oct_leaf_mask",
              "oct_leaf_nodes", "radix_node_to_oct", "radix_leaf_to_oct"]
RUNS = ("dehnen06", "bh05", "far_over", "near_over", "queue_over")
NEAR_FIELDS = ("offsets", "leaf_indices", "counts", "particle_order_leaf_indices",
               "particle_order_to_native_leaf")


def view_of(oracle, z):
    return oracle.octree_traversal_view({f: z[f] for f in OCT_FIELDS}, int(z["num_internal"]),
                                        z["bounds_min"], z["bounds_max"])


def rows_sorted(offsets, vals):
    out = np.array(vals, copy=True)
    for a, b in zip(offsets[:-1], offsets[1:]):
        out[a:b] = np.sort(out[a:b])
    return out


def far_row_offsets(targets):
    """Rows of the far output are runs of one target (level order)."""
    if targets.shape[0] == 0:
        return np.zeros(1, np.int64)
    cut = np.nonzero(np.diff(targets))[0] + 1
    return np.concatenate([[0], cut, [targets.shape[0]]]).astype(np.int64)


def far_error(w):
    if w["far_overflow"]:
        return "Native octree interaction list capacity exceeded"
    if w["queue_overflow"]:
        return "Native octree pair queue capacity exceeded"
    return None


def near_error(w):
    if w["near_overflow"]:
        return "Native octree neighbor list capacity exceeded"
    if w["queue_overflow"]:
        return "Native octree pair queue capacity exceeded"
    return None


def oracle_runs(oracle, z, v, run):
    theta, fcap, ncap, q = z[f"{run}_params"]
    mac = str(z[f"{run}_mac"])
    kw = dict(max_interactions_per_node=int(fcap), max_neighbors_per_leaf=int(ncap),
              max_pair_queue=int(q))
    far = oracle.octree_native_walk(v, float(theta), mac, collect_far=True, collect_near=False,
                                    **kw)
    near = oracle.octree_native_walk(v, float(theta), mac, collect_far=False, collect_near=True,
                                     **kw)
    return far, near


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_octree_view_matches_reference(oracle, path):
    z = np.load(path)
    v = view_of(oracle, z)
    for k in ("centers", "half_extents", "radii", "max_extents"):
        assert np.array_equal(v["box"][k], z[f"box_{k}"]), k
    assert np.array_equal(v["oct_to_radix_node"], z["oct_to_radix_node"])
    assert np.array_equal(v["oct_to_radix_leaf"], z["oct_to_radix_leaf"])


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_octree_walk_matches_reference(oracle, path):
    z = np.load(path)
    v = view_of(oracle, z)
    for run in RUNS:
        far, near = oracle_runs(oracle, z, v, run)
        if f"{run}_far_error" in z:
            assert far_error(far) is not None and str(z[f"{run}_far_error"]).startswith(
                far_error(far)), run
        else:
            assert far_error(far) is None, run
            tg = z[f"{run}_far_targets"]
            assert np.array_equal(far["targets"], tg), run
            off = far_row_offsets(tg)
            assert np.array_equal(rows_sorted(off, far["sources"]),
                                  rows_sorted(off, z[f"{run}_far_sources"])), run
            assert (z[f"{run}_far_tags"] == -1).all()
        if f"{run}_near_error" in z:
            assert near_error(near) is not None and str(z[f"{run}_near_error"]).startswith(
                near_error(near)), run
        else:
            assert near_error(near) is None, run
            nl = oracle.octree_native_neighbor_list(near, z["oct_node_ranges"])
            for f in NEAR_FIELDS:
                assert np.array_equal(nl[f], z[f"{run}_near_{f}"]), (run, f)
            off = nl["offsets"]
            assert np.array_equal(rows_sorted(off, nl["neighbors"]),
                                  rows_sorted(off, z[f"{run}_near_neighbors"])), run
            pos, want = nl["neighbor_leaf_positions"], z[f"{run}_near_neighbor_leaf_positions"]
            assert pos.shape == want.shape
            assert np.array_equal(np.sort(pos, axis=1), np.sort(want, axis=1)), run


def test_octree_fixtures_cover_both_spaces():
    """The fixtures hold non-empty far pairs and non-empty near rows (the
    fixed-depth trees, whose carrier cells are true leaves)."""
    far = near = 0
    for path in FILES:
        z = np.load(path)
        if "dehnen06_far_sources" in z:
            far += z["dehnen06_far_sources"].shape[0]
        if "dehnen06_near_neighbors" in z:
            near += z["dehnen06_near_neighbors"].shape[0]
    assert far > 0 and near > 0

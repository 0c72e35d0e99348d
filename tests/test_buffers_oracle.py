"""Oracle of the level-major geometry, the dense M2L buffers and the
class-grouped far pairs against golden fixtures made by running the
reference's own geometry_to_level_major / densify_interactions /
build_grouped_interactions_from_pairs (tests/golden/make_golden.py
--buffers-only) on its own trees and far lists."""

import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [("uniform300_leaf4", "walk_dehnen_"), ("plummer400_leaf8", "walk_bh_")]


def _eq(name, got, want):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape, (name, got.shape, want.shape)
    if want.dtype.kind == "f":
        assert np.array_equal(got.astype(want.dtype).view(np.uint32), want.view(np.uint32)), name
    else:
        assert np.array_equal(got.astype(np.int64), want.astype(np.int64)), name


@pytest.mark.parametrize("case,walk", CASES, ids=[c for c, _ in CASES])
def test_buffers_oracle_matches_reference(oracle, case, walk):
    t = np.load(os.path.join(HERE, "golden", f"adaptive_{case}.npz"))
    z = np.load(os.path.join(HERE, "golden", f"buffers_{case}.npz"))
    lg = oracle.level_major_geometry(t["nodes_by_level"], t["level_offsets"], int(t["num_levels"]),
                                     t["geom_center"], t["geom_half_extent"], t["geom_radius"],
                                     t["geom_max_extent"])
    for k in ("centers", "half_extents", "radii", "max_extents", "level_counts", "node_indices"):
        _eq(k, lg[k], z[f"lm_{k}"])
    d = oracle.dense_m2l(lg["node_indices"], t[f"{walk}far_counts"], t[f"{walk}far_offsets"],
                         t[f"{walk}far_sources"], t["geom_center"])
    for k in ("m2l_sources", "m2l_mask", "m2l_counts", "m2l_displacements"):
        _eq(k, d[k], z[k])
    g = oracle.grouped_from_pairs(z["pair_sources"], z["pair_targets"], t["node_level"],
                                  t["geom_center"], t["bounds_min"], t["bounds_max"])
    for k in ("class_keys", "class_displacements", "class_offsets", "class_sources",
              "class_targets", "class_ids"):
        _eq(k, g[k], z[f"grp_{k}"])

"""The native octree walk on the GPU (build_octree_native_far_pairs,
build_octree_native_neighbor_lists, build_explicit_octree_traversal_view):
on the reference's own octree topologies (golden fixtures) the box geometry
and maps are equal, the lists equal the reference's (rows as sets) and the
oracle's (in full order); the same RuntimeErrors on overflow; and on larger
fixed-depth octrees built by this library, equal to the oracle in full."""

import glob
import os
import types

import numpy as np
import pytest

from test_octwalk_oracle import (FILES, NEAR_FIELDS, OCT_FIELDS, RUNS, far_error,
                                 far_row_offsets, near_error, oracle_runs, rows_sorted,
                                 view_of)

pytestmark = pytest.mark.gpu


def _topology(z, dev):
    import torch

    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    f = {k: t(z[k]) for k in OCT_FIELDS}
    for k in ("oct_child_mask", "oct_valid_mask", "oct_leaf_mask"):
        f[k] = f[k].to(torch.bool)
    ni = int(z["num_internal"])
    return types.SimpleNamespace(
        **f, bounds_min=t(z["bounds_min"]), bounds_max=t(z["bounds_max"]),
        left_child=torch.zeros(ni, dtype=torch.int64, device=dev),
        parent=torch.zeros(int(z["radix_total"]), dtype=torch.int64, device=dev))


def _np(x):
    return x.detach().cpu().numpy()


def _cfg(z, run):
    import yggdrax_b200 as yb

    theta, fcap, ncap, q = z[f"{run}_params"]
    return float(theta), str(z[f"{run}_mac"]), yb.DualTreeTraversalConfig(
        max_pair_queue=int(q), process_block=64, max_interactions_per_node=int(fcap),
        max_neighbors_per_leaf=int(ncap))


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_octree_walk_matches_reference_and_oracle(cuda_device, oracle, path):
    import yggdrax_b200 as yb

    z = np.load(path)
    topo = _topology(z, cuda_device)
    view = yb.build_explicit_octree_traversal_view(topo)
    for k in ("centers", "half_extents", "radii", "max_extents"):
        assert np.array_equal(_np(getattr(view, f"box_{k}")), z[f"box_{k}"]), k
    assert np.array_equal(_np(view.oct_to_radix_node), z["oct_to_radix_node"])
    assert np.array_equal(_np(view.oct_to_radix_leaf), z["oct_to_radix_leaf"])
    v = view_of(oracle, z)
    for run in RUNS:
        theta, mac, cfg = _cfg(z, run)
        far, near = oracle_runs(oracle, z, v, run)
        if f"{run}_far_error" in z:
            with pytest.raises(RuntimeError, match=far_error(far)):
                yb.build_octree_native_far_pairs(topo, None, theta=theta, mac_type=mac,
                                                 traversal_config=cfg)
        else:
            fp = yb.build_octree_native_far_pairs(topo, None, theta=theta, mac_type=mac,
                                                  traversal_config=cfg)
            assert np.array_equal(_np(fp.targets), z[f"{run}_far_targets"]), run
            assert np.array_equal(_np(fp.sources), far["sources"]), run  # full order
            off = far_row_offsets(z[f"{run}_far_targets"])
            assert np.array_equal(rows_sorted(off, _np(fp.sources)),
                                  rows_sorted(off, z[f"{run}_far_sources"])), run
            assert (_np(fp.tags) == -1).all()
        if f"{run}_near_error" in z:
            with pytest.raises(RuntimeError, match=near_error(near)):
                yb.build_octree_native_neighbor_lists(topo, None, theta=theta, mac_type=mac,
                                                      traversal_config=cfg)
        else:
            nb = yb.build_octree_native_neighbor_lists(topo, None, theta=theta, mac_type=mac,
                                                       traversal_config=cfg)
            nl = oracle.octree_native_neighbor_list(near, z["oct_node_ranges"])
            for f in NEAR_FIELDS:
                assert np.array_equal(_np(getattr(nb, f)), z[f"{run}_near_{f}"]), (run, f)
            assert np.array_equal(_np(nb.neighbors), nl["neighbors"]), run  # full order
            assert np.array_equal(_np(nb.neighbor_leaf_positions),
                                  nl["neighbor_leaf_positions"]), run
            off = nl["offsets"]
            assert np.array_equal(rows_sorted(off, _np(nb.neighbors)),
                                  rows_sorted(off, z[f"{run}_near_neighbors"])), run


@pytest.mark.parametrize("n,depth,theta,mac", [(20000, 4, 0.6, "dehnen"), (30000, 5, 0.5, "bh"),
                                               (30000, 4, 0.5, "engblom")])
def test_octree_walk_matches_oracle_on_built_trees(cuda_device, oracle, n, depth, theta, mac):
    """Fixed-depth octrees of Plummer clumps built here: far pairs and near
    rows equal to the oracle in full order (the same view restated from the
    tree's own oct tables), decisions and wavefronts exercised over several
    generations."""
    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs

    pos, mass = inputs.plummer_clumps(n, 7)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)
    tree = yb.build_fixed_depth_octree(P, M, max_depth=depth, return_reordered=True)[0]
    topo = tree.topology if hasattr(tree, "topology") else tree
    fields = {k: _np(getattr(topo, k)) for k in OCT_FIELDS}
    v = oracle.octree_traversal_view(fields, int(topo.left_child.shape[0]),
                                     _np(topo.bounds_min), _np(topo.bounds_max))
    cfg = yb.DualTreeTraversalConfig(max_pair_queue=1 << 22, process_block=64,
                                     max_interactions_per_node=1 << 20,
                                     max_neighbors_per_leaf=1 << 20)
    kw = dict(max_interactions_per_node=1 << 20, max_neighbors_per_leaf=1 << 20,
              max_pair_queue=1 << 22)
    far = oracle.octree_native_walk(v, theta, mac, collect_far=True, collect_near=False, **kw)
    near = oracle.octree_native_walk(v, theta, mac, collect_far=False, collect_near=True, **kw)
    fp = yb.build_octree_native_far_pairs(topo, None, theta=theta, mac_type=mac,
                                          traversal_config=cfg)
    assert np.array_equal(_np(fp.targets), far["targets"])
    assert np.array_equal(_np(fp.sources), far["sources"])
    nb = yb.build_octree_native_neighbor_lists(topo, None, theta=theta, mac_type=mac,
                                               traversal_config=cfg)
    nl = oracle.octree_native_neighbor_list(near, fields["oct_node_ranges"])
    for f in NEAR_FIELDS + ("neighbors", "neighbor_leaf_positions"):
        assert np.array_equal(_np(getattr(nb, f)), nl[f]), f
    assert far["sources"].shape[0] > 0 and nl["neighbors"].shape[0] > 0

"""The pipeline at the benchmark configurations' full sizes.

* 4,194,304-particle Plummer sphere, octree build, leaf 32, dehnen 0.6 and
  bh 0.5: tree, geometry and lists equal to the oracle's, bit for bit.
* The benchmarked workload -- 16,777,216 Plummer particles (seed 4), radix
  leaf 32, dehnen 0.6, exact lists -- and the 16,777,216-point clump mixture
  (seed 2, fixed-depth octree, max_depth 10, local refinement, dehnen 0.6):
  tree, octree tables, geometry, far / near lists and decision counts equal
  to the oracle's, bit for bit.
* The same two workloads through size-independent properties as well
  (cheap, and independent of the oracle): the sort is a permutation in
  code order, the far and near lists are symmetric, every sampled far entry
  passes the MAC and every sampled near entry fails it (recomputed in the
  reference's fp32 order), and for sampled leaves every other particle is
  covered exactly once by the far lists of the leaf's ancestors and its own
  near list (the completeness of a dual-tree walk) -- and the class-grouped
  far pairs keep every pair, with class keys recomputed for a sample.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def test_c2_octree_4m_matches_oracle(cuda_device, oracle):
    import torch

    import yggdrax_b200 as yb
    from test_gpu_parity import _assert_eq, _compare_lists
    from yggdrax_b200 import inputs

    pos, mass = inputs.plummer(4_194_304, 1)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)
    yb.set_reference_limits(False)
    try:
        gt, ps = yb.build_octree(P, M, leaf_size=32, return_reordered=True)[:2]
        ot = oracle.build_octree(pos, mass, leaf_size=32)
        for f in ("particle_indices", "parent", "left_child", "right_child", "node_ranges",
                  "nodes_by_level"):
            _assert_eq(f, _np(getattr(gt, f)), getattr(ot, f))
        for f in ("oct_children", "oct_level_offsets", "radix_node_to_oct"):
            _assert_eq(f, _np(getattr(gt, f)), ot.octree[f])
        gg = yb.compute_tree_geometry(gt, ps)
        og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
        for f in ("center", "radius", "max_extent"):
            _assert_eq(f, _np(getattr(gg, f)), getattr(og, f))
        for mac, theta in (("dehnen", 0.6), ("bh", 0.5)):
            gi, gn = yb.build_interactions_and_neighbors(gt, gg, theta=theta, mac_type=mac)
            r = oracle.build_interactions_and_neighbors(ot, og, theta=theta, mac_type=mac)
            _compare_lists(gi, gn, r)
            del gi, gn, r
    finally:
        yb.set_reference_limits(True)


def _symmetric(rows_of, vals, dev):
    """Every directed entry (row -> value) has its reverse."""
    import torch

    a = rows_of.to(torch.int64) << 32 | vals.to(torch.int64)
    b = vals.to(torch.int64) << 32 | rows_of.to(torch.int64)
    return torch.equal(torch.sort(a).values, torch.sort(b).values)


def _mac_ok(center, ext, t, s, theta):
    # _compute_mac_ok (_interactions_impl.py:338-395), dehnen form, fp32
    d = center[t] - center[s]
    d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    tsq = np.float32(theta) * np.float32(theta)
    sm = ext[t] + ext[s]
    return (sm * sm <= tsq * d2) & (d2 > 0)


def _check_lists(tree, geom, inter, nbrs, theta, rng, n_leaves_sample=24):
    import torch

    dev = tree.parent.device
    total = int(tree.parent.shape[0])
    ni = int(tree.left_child.shape[0])
    # far rows (node order) and near rows (native leaf order)
    counts = inter.counts.to(torch.int64)
    node_of_entry = torch.repeat_interleave(torch.arange(total, device=dev), counts)
    starts = inter.offsets.to(torch.int64)[:-1]
    # entries are stored level-major: map each node's block
    pos = torch.repeat_interleave(starts, counts) + (
        torch.arange(int(counts.sum()), device=dev)
        - torch.repeat_interleave(torch.cumsum(counts, 0) - counts, counts))
    far_src = inter.sources.to(torch.int64)[pos]
    assert _symmetric(node_of_entry, far_src, dev)
    leaf_idx = nbrs.leaf_indices.to(torch.int64)
    ncounts = nbrs.counts.to(torch.int64)
    near_row_node = torch.repeat_interleave(leaf_idx, ncounts)
    near_src = nbrs.neighbors.to(torch.int64)
    assert _symmetric(near_row_node, near_src, dev)
    # MAC on samples (radius x dehnen scale 1 = the MAC extent)
    center = _np(geom.center)
    ext = _np(geom.radius)
    k = min(1_000_000, far_src.numel())
    pick = torch.randint(0, far_src.numel(), (k,), device=dev) if k else None
    if k:
        t = _np(node_of_entry[pick]); s = _np(far_src[pick])
        assert _mac_ok(center, ext, t, s, theta).all()
    k = min(1_000_000, near_src.numel())
    if k:
        pick = torch.randint(0, near_src.numel(), (k,), device=dev)
        t = _np(near_row_node[pick]); s = _np(near_src[pick])
        assert not _mac_ok(center, ext, t, s, theta).any()
    # completeness on sampled leaves, in particle space
    n = int(tree.num_particles)
    ranges = _np(tree.node_ranges).astype(np.int64)
    parent = _np(tree.parent).astype(np.int64)
    far_cnt = _np(counts)
    far_off = _np(starts)
    sources = _np(inter.sources).astype(np.int64)
    row_of_leaf = np.full(total, -1, np.int64)
    row_of_leaf[_np(leaf_idx)] = np.arange(leaf_idx.numel())
    near_off = _np(nbrs.offsets).astype(np.int64)
    neighbors = _np(near_src)
    for leaf in rng.choice(np.arange(ni, total), size=n_leaves_sample, replace=False):
        diff = np.zeros(n + 1, np.int32)

        def cover(nodes):
            np.add.at(diff, ranges[nodes, 0], 1)
            np.add.at(diff, ranges[nodes, 1] + 1, -1)

        a = leaf
        while a >= 0:
            cover(sources[far_off[a]:far_off[a] + far_cnt[a]])
            a = parent[a]
        r = row_of_leaf[leaf]
        cover(neighbors[near_off[r]:near_off[r + 1]])
        cov = np.cumsum(diff)[:n]
        own = np.zeros(n, bool)
        own[ranges[leaf, 0]:ranges[leaf, 1] + 1] = True
        assert (cov[~own] == 1).all() and (cov[own] == 0).all(), leaf


def test_c5_plummer_16m_properties(cuda_device):
    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs

    pos, mass = inputs.plummer(16_777_216, 4)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)
    yb.set_reference_limits(False)
    try:
        t, ps = yb.build_tree(P, M, leaf_size=32, return_reordered=True)[:2]
        codes = t.morton_codes.to(torch.int64)
        assert bool((codes[1:] >= codes[:-1]).all())
        pidx = t.particle_indices.to(torch.int64)
        assert torch.equal(torch.sort(pidx).values, torch.arange(pidx.numel(), device=cuda_device))
        g = yb.compute_tree_geometry(t, ps)
        inter, nbrs = yb.build_interactions_and_neighbors(t, g, theta=0.6, mac_type="dehnen")
        _check_lists(t, g, inter, nbrs, 0.6, np.random.default_rng(0))
    finally:
        yb.set_reference_limits(True)


def test_c3_clumps_16m_fixed_depth_properties(cuda_device):
    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs

    pos, mass = inputs.plummer_clumps(16_777_216, 2)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)
    yb.set_reference_limits(False)
    try:
        t, ps = yb.build_fixed_depth_octree(P, M, max_depth=10, return_reordered=True)[:2]
        g = yb.compute_tree_geometry(t, ps)
        inter, nbrs, grp = yb.build_interactions_and_neighbors(t, g, theta=0.6, mac_type="dehnen",
                                                               return_grouped=True)
        _check_lists(t, g, inter, nbrs, 0.6, np.random.default_rng(1), n_leaves_sample=8)
        # grouped: every pair kept, classes contiguous, keys of sampled pairs
        P_ = int(inter.sources.numel())
        assert int(grp.class_offsets[-1]) == P_ and grp.class_sources.numel() == P_
        off = _np(grp.class_offsets).astype(np.int64)
        assert (np.diff(off) > 0).all()
        keys = _np(grp.class_keys)
        rng = np.random.default_rng(2)
        cls = rng.integers(0, keys.shape[0], 2000)
        src = _np(grp.class_sources).astype(np.int64)
        tgt = _np(grp.class_targets).astype(np.int64)
        lev = _np(t.node_level).astype(np.int64)
        c64 = _np(g.center).astype(np.float64)
        ext = (_np(t.bounds_max).astype(np.float64) - _np(t.bounds_min).astype(np.float64))
        for c in cls:
            j = off[c]  # first pair of the class
            tl = lev[tgt[j]]
            cell = np.maximum(ext / max(2.0 ** tl, 1.0), 1e-12)
            d = np.rint((c64[tgt[j]] - c64[src[j]]) / cell).astype(np.int64)
            assert [tl, lev[src[j]], *d] == keys[c].tolist()
        # the dense buffers at this size exceed the device, as in the reference
        with pytest.raises(MemoryError):
            yb.densify_interactions(t, g, inter)
    finally:
        yb.set_reference_limits(True)


def _compare_full(gt, ps, gg, ot, og, gi, gn, res, r, octree: bool):
    """Every output of the GPU pipeline against the oracle's (bit for bit),
    freeing host copies as it goes."""
    from test_gpu_parity import RADIX_FIELDS, _assert_eq, _compare_lists

    topo = gt.topology
    for f in RADIX_FIELDS:
        _assert_eq(f, _np(getattr(topo, f)), getattr(ot, f))
    assert int(topo.num_levels) == ot.num_levels
    _assert_eq("positions_sorted", _np(ps), ot.positions_sorted)
    if octree:
        for f in ("oct_parent", "oct_children", "oct_node_codes", "oct_node_depths",
                  "oct_node_ranges", "oct_level_offsets", "oct_leaf_nodes",
                  "radix_node_to_oct", "radix_leaf_to_oct"):
            _assert_eq(f, _np(getattr(gt, f)), ot.octree[f])
    for f in ("center", "half_extent", "radius", "max_extent"):
        _assert_eq(f, _np(getattr(gg, f)), getattr(og, f))
    _compare_lists(gi, gn, r)
    assert int(res.accept_decisions) == r["accept_decisions"]
    assert int(res.near_decisions) == r["near_decisions"]
    assert int(res.refine_decisions) == r["refine_decisions"]


def test_c5_plummer_16m_matches_oracle(cuda_device, oracle):
    """The benchmarked workload, bit for bit against the oracle."""
    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs

    pos, mass = inputs.plummer(16_777_216, 4)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)
    yb.set_reference_limits(False)
    try:
        gt, ps = yb.build_tree(P, M, leaf_size=32, return_reordered=True)[:2]
        gg = yb.compute_tree_geometry(gt, ps)
        gi, gn, res = yb.build_interactions_and_neighbors(gt, gg, theta=0.6, mac_type="dehnen",
                                                          return_result=True)
        del P, M
        ot = oracle.build_tree(pos, mass, leaf_size=32)
        og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
        r = oracle.build_interactions_and_neighbors(ot, og, theta=0.6, mac_type="dehnen")
        _compare_full(gt, ps, gg, ot, og, gi, gn, res, r, octree=False)
    finally:
        yb.set_reference_limits(True)


def test_c3_clumps_16m_matches_oracle(cuda_device, oracle):
    """The clump mixture on the fixed-depth octree, bit for bit against the
    oracle (octree tables included)."""
    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs

    pos, mass = inputs.plummer_clumps(16_777_216, 2)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)
    yb.set_reference_limits(False)
    try:
        gt, ps = yb.build_fixed_depth_octree(P, M, max_depth=10, return_reordered=True)[:2]
        gg = yb.compute_tree_geometry(gt, ps)
        gi, gn, res = yb.build_interactions_and_neighbors(gt, gg, theta=0.6, mac_type="dehnen",
                                                          return_result=True)
        del P, M
        ot = oracle.build_fixed_depth_octree(pos, mass, max_depth=10)
        og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
        r = oracle.build_interactions_and_neighbors(ot, og, theta=0.6, mac_type="dehnen")
        _compare_full(gt, ps, gg, ot, og, gi, gn, res, r, octree=True)
    finally:
        yb.set_reference_limits(True)

"""GPU parity: every stage of the CUDA path against the CPU oracle.

Integer, index and ordering outputs must be bit-exact; float32 geometry is
compared bit-exactly as well (the kernels evaluate the reference's fp32
operations in the same order with round-to-nearest intrinsics).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _to_dev(arr, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(arr)).to(dev)


def _cases():
    from yggdrax_b200 import inputs

    rng = np.random.default_rng(7)
    dup = np.zeros((64, 3), np.float32)
    collinear = np.array([[float(i), 0.0, 0.0] for i in range(128)], np.float32)
    return {
        "uniform65k": inputs.uniform_cube(65536, 0),
        "plummer40k": inputs.plummer(40000, 1),
        "clumps30k": inputs.plummer_clumps(30000, 2, clumps=8),
        "small17": (rng.uniform(-1, 1, (17, 3)).astype(np.float32), np.ones(17, np.float32)),
        "dup64": (dup, np.ones(64, np.float32)),
        "collinear128": (collinear, np.ones(128, np.float32)),
    }


CASES = _cases()
BOUNDS = {"collinear128": (np.array([-10.0, -1.0, -1.0], np.float32),
                           np.array([10.0, 1.0, 1.0], np.float32))}


def _assert_eq(name, got, want):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, f"{name}: shape {got.shape} != {want.shape}"
    if got.dtype.kind == "f":
        ok = np.array_equal(got.view(np.uint32), want.astype(got.dtype).view(np.uint32))
    else:
        ok = np.array_equal(got.astype(np.int64) if got.dtype != np.uint64 else got,
                            want.astype(np.int64) if want.dtype != np.uint64 else want)
    if not ok:
        bad = np.flatnonzero(got.reshape(-1) != want.reshape(-1).astype(got.dtype))[:5]
        raise AssertionError(f"{name}: mismatch at {bad}: got {got.reshape(-1)[bad]} "
                             f"want {want.reshape(-1)[bad]}")


RADIX_FIELDS = ["parent", "left_child", "right_child", "left_is_leaf", "right_is_leaf",
                "particle_indices", "morton_codes", "node_ranges", "node_level",
                "level_offsets", "nodes_by_level", "bounds_min", "bounds_max", "leaf_codes",
                "leaf_depths"]


def _compare_tree(gt, ot):
    topo = gt.topology
    for f in RADIX_FIELDS:
        _assert_eq(f, _np(getattr(topo, f)), getattr(ot, f))
    assert int(topo.num_levels) == ot.num_levels
    assert topo.num_internal_nodes == ot.num_internal_nodes
    _assert_eq("positions_sorted", _np(gt.positions_sorted), ot.positions_sorted)
    _assert_eq("masses_sorted", _np(gt.masses_sorted), ot.masses_sorted)
    _assert_eq("inverse", _np(gt.inverse_permutation), ot.inverse_permutation)


@pytest.mark.parametrize("case", ["uniform65k", "plummer40k", "small17", "dup64", "collinear128"])
@pytest.mark.parametrize("leaf_size", [1, 16])
def test_radix_build_matches_oracle(cuda_device, oracle, case, leaf_size):
    import yggdrax_b200 as yb

    pos, mass = CASES[case]
    b = BOUNDS.get(case)
    gt = yb.build_tree(_to_dev(pos, cuda_device), _to_dev(mass, cuda_device),
                       None if b is None else tuple(_to_dev(x, cuda_device) for x in b),
                       leaf_size=leaf_size, return_reordered=True)[0]
    ot = oracle.build_tree(pos, mass, b, leaf_size=leaf_size)
    _compare_tree(gt, ot)


def test_packed_reorder_matches_plain_reorder(cuda_device):
    """ygx_pack_particles + ygx_reorder_packed (the build's path) give the same
    sorted positions, masses, particle indices and inverse permutation as
    ygx_reorder, for a random order of an uneven count."""
    import torch

    from yggdrax_b200 import _lib as L

    lib = L.lib()
    n = 70_001
    rng = np.random.default_rng(3)
    P = _to_dev(rng.standard_normal((n, 3)).astype(np.float32), cuda_device)
    M = _to_dev(rng.random(n).astype(np.float32), cuda_device)
    order = torch.randperm(n, device=cuda_device).to(torch.int32)
    st = L.stream_handle(cuda_device)
    outs = [[torch.empty((n, 3), dtype=torch.float32, device=cuda_device),
             torch.empty(n, dtype=torch.float32, device=cuda_device),
             torch.empty(n, dtype=torch.int64, device=cuda_device),
             torch.empty(n, dtype=torch.int64, device=cuda_device)] for _ in range(2)]
    L.check(lib.ygx_reorder(L.ptr(P), L.ptr(M), L.ptr(order), n, 64,
                            *[L.ptr(o) for o in outs[0]], st), "ygx_reorder")
    packed = torch.empty((n, 4), dtype=torch.float32, device=cuda_device)
    L.check(lib.ygx_pack_particles(L.ptr(P), L.ptr(M), n, L.ptr(packed), st),
            "ygx_pack_particles")
    L.check(lib.ygx_reorder_packed(L.ptr(packed), L.ptr(order), n, 64,
                                   *[L.ptr(o) for o in outs[1]], st), "ygx_reorder_packed")
    for a, b in zip(*outs):
        assert torch.equal(a, b)


@pytest.mark.parametrize("case", ["clumps30k", "plummer40k", "collinear128", "dup64"])
@pytest.mark.parametrize("refine", [True, False])
def test_fixed_depth_build_matches_oracle(cuda_device, oracle, case, refine):
    import yggdrax_b200 as yb

    pos, mass = CASES[case]
    b = BOUNDS.get(case)
    gt = yb.build_fixed_depth_tree(
        _to_dev(pos, cuda_device), _to_dev(mass, cuda_device),
        None if b is None else tuple(_to_dev(x, cuda_device) for x in b),
        target_leaf_particles=8, refine_local=refine, return_reordered=True)[0]
    ot = oracle.build_fixed_depth_tree(pos, mass, b, target_leaf_particles=8,
                                       refine_local=refine)
    _compare_tree(gt, ot)


OCT_FIELDS = ["oct_parent", "oct_children", "oct_child_counts", "oct_child_mask",
              "oct_valid_mask", "oct_node_codes", "oct_node_depths", "oct_node_ranges",
              "oct_nodes_by_level", "oct_level_offsets", "oct_leaf_mask", "oct_leaf_nodes",
              "radix_node_to_oct", "radix_leaf_to_oct"]


@pytest.mark.parametrize("case", ["uniform65k", "plummer40k", "clumps30k", "dup64"])
@pytest.mark.parametrize("mode", ["adaptive", "fixed_depth"])
def test_octree_tables_match_oracle(cuda_device, oracle, case, mode):
    import yggdrax_b200 as yb

    pos, mass = CASES[case]
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    if mode == "adaptive":
        gt = yb.build_octree(P, M, leaf_size=32)
        ot = oracle.build_octree(pos, mass, leaf_size=32)
    else:
        gt = yb.build_fixed_depth_octree(P, M, target_leaf_particles=16)
        ot = oracle.build_fixed_depth_octree(pos, mass, target_leaf_particles=16)
    for f in OCT_FIELDS:
        _assert_eq(f, _np(getattr(gt.topology, f)), ot.octree[f])
    assert int(gt.topology.oct_num_levels) == ot.octree["oct_num_levels"]


@pytest.mark.parametrize("case,mode", [("uniform65k", "adaptive"), ("plummer40k", "adaptive"),
                                       ("clumps30k", "fixed_depth"), ("dup64", "adaptive"),
                                       ("collinear128", "fixed_depth"), ("small17", "adaptive")])
def test_geometry_matches_oracle(cuda_device, oracle, case, mode):
    import yggdrax_b200 as yb

    pos, mass = CASES[case]
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    if mode == "adaptive":
        gt, ps = yb.build_tree(P, M, leaf_size=4, return_reordered=True)[:2]
        ot = oracle.build_tree(pos, mass, leaf_size=4)
    else:
        gt, ps = yb.build_fixed_depth_tree(P, M, return_reordered=True)[:2]
        ot = oracle.build_fixed_depth_tree(pos, mass)
    gg = yb.compute_tree_geometry(gt, ps)
    og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
    for f in ("center", "half_extent", "radius", "max_extent"):
        _assert_eq(f, _np(getattr(gg, f)), getattr(og, f))


def _compare_lists(gi, gn, r):
    _assert_eq("far.counts", _np(gi.counts), r["far_counts"])
    _assert_eq("far.offsets", _np(gi.offsets), r["offsets"])
    _assert_eq("far.sources", _np(gi.sources), r["sources"])
    _assert_eq("far.targets", _np(gi.targets), r["targets"])
    _assert_eq("far.level_offsets", _np(gi.level_offsets), r["level_offsets"])
    _assert_eq("far.target_levels", _np(gi.target_levels), r["target_levels"])
    _assert_eq("near.counts", _np(gn.counts), r["near_counts"])
    _assert_eq("near.offsets", _np(gn.offsets), r["near_offsets"])
    _assert_eq("near.neighbors", _np(gn.neighbors), r["neighbors"])
    _assert_eq("near.leaf_indices", _np(gn.leaf_indices), r["leaf_indices"])
    _assert_eq("near.po_to_native", _np(gn.particle_order_to_native_leaf),
               r["particle_order_to_native_leaf"])


@pytest.mark.parametrize("case,tree_kind,leaf,mac,theta", [
    ("uniform65k", "radix", 16, "dehnen", 0.6),
    ("uniform65k", "radix", 16, "bh", 0.5),
    ("plummer40k", "octree", 32, "dehnen", 0.6),
    ("plummer40k", "octree", 32, "engblom", 0.5),
    ("clumps30k", "fixed_octree", 16, "dehnen", 0.6),
    ("small17", "radix", 4, "bh", 0.5),
    ("dup64", "radix", 4, "dehnen", 0.6),
])
def test_traversal_matches_oracle(cuda_device, oracle, case, tree_kind, leaf, mac, theta):
    import yggdrax_b200 as yb

    pos, mass = CASES[case]
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    if tree_kind == "radix":
        gt, ps = yb.build_tree(P, M, leaf_size=leaf, return_reordered=True)[:2]
        ot = oracle.build_tree(pos, mass, leaf_size=leaf)
    elif tree_kind == "octree":
        gt, ps = yb.build_octree(P, M, leaf_size=leaf, return_reordered=True)[:2]
        ot = oracle.build_octree(pos, mass, leaf_size=leaf)
    else:
        gt, ps = yb.build_fixed_depth_octree(P, M, target_leaf_particles=leaf,
                                             return_reordered=True)[:2]
        ot = oracle.build_fixed_depth_octree(pos, mass, target_leaf_particles=leaf)
    gg = yb.compute_tree_geometry(gt, ps)
    og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
    gi, gn, res = yb.build_interactions_and_neighbors(gt, gg, theta=theta, mac_type=mac,
                                                      return_result=True)
    r = oracle.build_interactions_and_neighbors(ot, og, theta=theta, mac_type=mac)
    _compare_lists(gi, gn, r)
    assert int(res.accept_decisions) == r["accept_decisions"]
    assert int(res.near_decisions) == r["near_decisions"]
    assert int(res.refine_decisions) == r["refine_decisions"]
    nlp = oracle.neighbor_leaf_positions(r["leaf_indices"], r["near_offsets"],
                                         r["near_counts"], r["neighbors"],
                                         ot.node_ranges.shape[0])
    _assert_eq("neighbor_leaf_positions", _np(gn.neighbor_leaf_positions), nlp)


def test_capacity_errors_match_reference_messages(cuda_device):
    import yggdrax_b200 as yb

    pos, mass = CASES["uniform65k"]
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    gt, ps = yb.build_tree(P, M, leaf_size=16, return_reordered=True)[:2]
    gg = yb.compute_tree_geometry(gt, ps)
    cfg = yb.DualTreeTraversalConfig(max_pair_queue=65536, process_block=256,
                                     max_interactions_per_node=4, max_neighbors_per_leaf=2048)
    with pytest.raises(RuntimeError, match="Interaction list capacity exceeded"):
        yb.build_interactions_and_neighbors(gt, gg, theta=0.6, mac_type="dehnen",
                                            traversal_config=cfg)
    cfg_ok = yb.DualTreeTraversalConfig(65536, 256, 2048, 2048)
    gi, gn = yb.build_interactions_and_neighbors(gt, gg, theta=0.6, mac_type="dehnen",
                                                 traversal_config=cfg_ok)
    assert int(gi.counts.max()) <= 2048
    with pytest.raises(ValueError, match="dehnen_radius_scale must be > 0"):
        yb.build_interactions_and_neighbors(gt, gg, mac_type="dehnen", dehnen_radius_scale=0.0)


def test_single_leaf_tree(cuda_device, oracle):
    import yggdrax_b200 as yb

    pos, mass = CASES["small17"]
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    gt, ps = yb.build_tree(P, M, leaf_size=64, return_reordered=True)[:2]
    ot = oracle.build_tree(pos, mass, leaf_size=64)
    _compare_tree(gt, ot)
    gg = yb.compute_tree_geometry(gt, ps)
    og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
    _assert_eq("center", _np(gg.center), og.center)
    gi, gn = yb.build_interactions_and_neighbors(gt, gg, theta=0.5)
    assert gi.sources.numel() == 0 and gn.neighbors.numel() == 0
    assert int(gn.counts.sum()) == 0


@pytest.mark.parametrize("tile,digit_bits", [(0, 8), (1, 8), (2, 8), (3, 8), (0, 11)])
def test_sort_pairs_is_stable(cuda_device, tile, digit_bits):
    """Stable sort under every onesweep tile shape (3072-6144 keys per tile)
    and with 11-bit digits (4096-key tiles; used for 9-11, 17-22, 25-33,
    ... bit ranges, where it cuts passes); sizes straddle tile boundaries of
    each shape."""
    import torch

    from yggdrax_b200 import _lib as L
    from yggdrax_b200 import autotune

    rng = np.random.default_rng(3 + tile + digit_bits)
    saved = autotune.current()
    autotune.apply({"sort_tile": tile, "sort_bits": digit_bits})
    try:
        for n, bits in [(1, 8), (3071, 8), (4095, 8), (4097, 16), (5121, 12), (6145, 24),
                        (100003, 63), (300000, 20), (1, 63), (4095, 11), (4096, 9),
                        (8193, 63), (12289, 33), (200001, 64)]:
            keys = rng.integers(0, 1 << 63, size=n, dtype=np.uint64) * np.uint64(2) + \
                rng.integers(0, 2, size=n, dtype=np.uint64)
            if bits < 64:
                keys &= np.uint64((1 << bits) - 1)
            keys[: n // 3] = keys[0]  # many ties
            k = torch.from_numpy(keys).to(cuda_device)
            ko = torch.empty_like(k)
            vo = torch.empty(n, dtype=torch.int32, device=cuda_device)
            lib = L.lib()
            ws = L.workspace(lib.ygx_sort_pairs_workspace_size(n), cuda_device)
            L.check(lib.ygx_sort_pairs(L.ptr(k), None, n, 0, bits, L.ptr(ko), L.ptr(vo),
                                       L.ptr(ws), ws.numel(), L.stream_handle(cuda_device)),
                    "sort")
            want = np.argsort(keys, kind="stable")
            np.testing.assert_array_equal(vo.cpu().numpy(), want)
            np.testing.assert_array_equal(ko.cpu().numpy(), keys[want])
            assert L.read_status(ws) == 0
    finally:
        autotune.apply(saved)


def test_long_rows_match_oracle(cuda_device, oracle):
    """Plummer halo leaves are near to every other leaf: rows of > 8192
    entries take the bitmap ordering path."""
    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs

    pos, mass = inputs.plummer(300_000, 5)
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    gt, ps = yb.build_tree(P, M, leaf_size=32, return_reordered=True)[:2]
    gg = yb.compute_tree_geometry(gt, ps)
    gi, gn = yb.build_interactions_and_neighbors(gt, gg, theta=0.6, mac_type="dehnen")
    ot = oracle.build_tree(pos, mass, leaf_size=32)
    og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
    r = oracle.build_interactions_and_neighbors(ot, og, theta=0.6, mac_type="dehnen")
    assert r["near_counts"].max() > 8192
    _compare_lists(gi, gn, r)


def test_reference_count_pass_limit(cuda_device):
    """The reference's count-pass sizing check (max near row vs
    int32_max // L) raises on a 2M Plummer sphere; with the limits off the
    exact lists are returned."""
    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs

    pos, mass = inputs.plummer(1 << 21, 6)
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    gt, ps = yb.build_tree(P, M, leaf_size=32, return_reordered=True)[:2]
    gg = yb.compute_tree_geometry(gt, ps)
    with pytest.raises(RuntimeError, match="Suggested per-leaf neighbor capacity"):
        yb.build_interactions_and_neighbors(gt, gg, theta=0.6, mac_type="dehnen")
    yb.set_reference_limits(False)
    try:
        gi, gn = yb.build_interactions_and_neighbors(gt, gg, theta=0.6, mac_type="dehnen")
    finally:
        yb.set_reference_limits(True)
    nl = gt.num_leaves
    assert int(gn.counts.max()) > (2**31 - 1) // nl
    assert int(gn.offsets[-1]) == int(gn.neighbors.numel())
    # every row strictly ascending
    nb = gn.neighbors.cpu().numpy()
    off = gn.offsets.cpu().numpy()
    d = np.diff(nb)
    starts = off[1:-1]
    mask = np.ones(d.shape[0], bool)
    mask[starts[(starts > 0) & (starts <= d.shape[0])] - 1] = False
    assert (d[mask] > 0).all()


def test_wavefront_overflow_retries_with_larger_capacity(cuda_device):
    """A wavefront capacity far below the walk's peak makes the count pass
    report a queue overflow; the walk is re-run with a larger wavefront and
    returns the same lists as a walk that never overflowed."""
    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs
    from yggdrax_b200.interactions import LAST_WALK_STATS, _run_walk

    pos, mass = inputs.uniform_cube(1 << 20, 3)
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    gt, ps = yb.build_tree(P, M, leaf_size=8, return_reordered=True)[:2]
    gg = yb.compute_tree_geometry(gt, ps)
    prev = yb.get_traversal_mode()
    yb.set_traversal_mode("log")  # the generation walk's wavefront ladder
    try:
        a = _run_walk(gt, gg, 0.6, "dehnen", 1.0)
        peak = LAST_WALK_STATS["max_wf"]
        assert peak > 2_000_000
        b = _run_walk(gt, gg, 0.6, "dehnen", 1.0, wf_capacity=4)
        assert LAST_WALK_STATS["wf_capacity"] > 4
        assert LAST_WALK_STATS["max_wf"] == peak
    finally:
        yb.set_traversal_mode(prev)
    for f in ("far_counts", "node_offsets", "level_offsets", "sources", "targets",
              "near_counts", "near_offsets", "neighbors"):
        np.testing.assert_array_equal(_np(getattr(a, f)), _np(getattr(b, f)), err_msg=f)


@pytest.mark.parametrize("mode", ["two_pass", "log", "target", "target_ordered"])
def test_traversal_modes_give_identical_lists(cuda_device, oracle, mode):
    """The plain two-pass schedule (count walk, then a fill walk), the
    one-walk pair log and the per-target walks return the same lists as the
    oracle."""
    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs

    pos, mass = inputs.plummer(200_000, 11)
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    gt, ps = yb.build_tree(P, M, leaf_size=16, return_reordered=True)[:2]
    gg = yb.compute_tree_geometry(gt, ps)
    prev = yb.get_traversal_mode()
    yb.set_traversal_mode(mode)
    try:
        gi, gn = yb.build_interactions_and_neighbors(gt, gg, theta=0.5, mac_type="bh")
    finally:
        yb.set_traversal_mode(prev)
    ot = oracle.build_tree(pos, mass, leaf_size=16)
    og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
    r = oracle.build_interactions_and_neighbors(ot, og, theta=0.5, mac_type="bh")
    _compare_lists(gi, gn, r)


def test_compact_far_pairs_and_leaf_neighbors(cuda_device, oracle):
    """build_compact_far_pairs / build_leaf_neighbor_lists /
    build_compact_far_pairs_and_leaf_neighbor_lists: the oracle's far rows in
    node order (targets = the row's node, tags -1) and its near lists; the
    fixed-capacity form pads with -1 and raises above the capacity."""
    import yggdrax_b200 as yb

    pos, mass = CASES["uniform65k"]
    P, M = _to_dev(pos, cuda_device), _to_dev(mass, cuda_device)
    t, ps = yb.build_tree(P, M, leaf_size=16, return_reordered=True)[:2]
    g = yb.compute_tree_geometry(t, ps)
    ot = oracle.build_tree(pos, mass, leaf_size=16)
    og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
    r = oracle.build_interactions_and_neighbors(ot, og, theta=0.6, mac_type="dehnen")
    off, cnt = np.asarray(r["offsets"]), np.asarray(r["far_counts"])
    src = np.concatenate([np.asarray(r["sources"])[off[k]:off[k] + cnt[k]]
                          for k in range(cnt.shape[0])])
    tgt = np.repeat(np.arange(cnt.shape[0]), cnt)
    cf = yb.build_compact_far_pairs(t, g, theta=0.6, mac_type="dehnen")
    _assert_eq("compact.sources", _np(cf.sources), src)
    _assert_eq("compact.targets", _np(cf.targets), tgt)
    assert int(cf.far_pair_count) == src.shape[0] and bool((_np(cf.tags) == -1).all())
    nb = yb.build_leaf_neighbor_lists(t, g, theta=0.6, mac_type="dehnen")
    _assert_eq("leaf_nbrs.neighbors", _np(nb.neighbors), r["neighbors"])
    _assert_eq("leaf_nbrs.offsets", _np(nb.offsets), r["near_offsets"])
    cap = src.shape[0] + 100
    cf2, nb2 = yb.build_compact_far_pairs_and_leaf_neighbor_lists(
        t, g, theta=0.6, mac_type="dehnen", compact_far_pair_capacity=cap)
    s2 = _np(cf2.sources)
    assert s2.shape[0] == cap and (s2[src.shape[0]:] == -1).all()
    _assert_eq("fused.sources", s2[:src.shape[0]], src)
    _assert_eq("fused.neighbors", _np(nb2.neighbors), r["neighbors"])
    with pytest.raises(RuntimeError, match="compact far-pair cap exceeded"):
        yb.build_compact_far_pairs_and_leaf_neighbor_lists(
            t, g, theta=0.6, mac_type="dehnen", compact_far_pair_capacity=src.shape[0] - 1)

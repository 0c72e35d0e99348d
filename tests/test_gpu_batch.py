"""Batched point sets on the GPU: every set's slice of the batched build,
geometry and lists equals (bit for bit) what the single-set path returns for
that set alone -- uneven sizes, single-leaf sets, sets with many identical
points (tied leaf codes) and collinear sets included."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOPO_FIELDS = ["parent", "left_child", "right_child", "left_is_leaf", "right_is_leaf",
               "particle_indices", "morton_codes", "node_ranges", "node_level", "level_offsets",
               "nodes_by_level", "num_levels", "bounds_min", "bounds_max", "leaf_codes",
               "leaf_depths"]
FAR_FIELDS = ["offsets", "sources", "targets", "counts", "level_offsets", "target_levels"]
NEAR_FIELDS = ["offsets", "neighbors", "leaf_indices", "counts", "particle_order_leaf_indices",
               "particle_order_to_native_leaf", "neighbor_leaf_positions"]


def _sets(seed=5):
    from yggdrax_b200 import inputs

    rng = np.random.default_rng(seed)
    sets = []
    sizes = [1, 3, 16, 17, 33, 250, 1000, 4097] + list(rng.integers(2, 3000, 24))
    for k, n in enumerate(sizes):
        if k % 2:
            p, m = inputs.plummer(int(n), 100 + k)
        else:
            p, m = inputs.uniform_cube(int(n), 100 + k)
        sets.append((p, m))
    dup = np.zeros((80, 3), np.float32)
    dup[40:] = rng.uniform(-1, 1, (40, 3))
    sets.append((dup, np.ones(80, np.float32)))                       # tied codes
    sets.append((np.zeros((50, 3), np.float32), np.ones(50, np.float32)))  # all identical
    col = np.stack([np.arange(300, dtype=np.float32), np.zeros(300, np.float32),
                    np.zeros(300, np.float32)], 1)
    sets.append((col, np.ones(300, np.float32)))
    return sets


def _eq(name, a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    b = b.detach().cpu().numpy() if hasattr(b, "detach") else np.asarray(b)
    assert a.shape == b.shape, f"{name}: {a.shape} vs {b.shape}"
    if a.dtype.kind == "f":
        assert np.array_equal(a.view(np.uint32), b.astype(a.dtype).view(np.uint32)), name
    else:
        assert np.array_equal(a.astype(np.int64) if a.dtype != np.uint64 else a,
                              b.astype(np.int64) if b.dtype != np.uint64 else b), name


@pytest.mark.parametrize("leaf", [16, 1])
def test_batched_sets_match_single_set_path(cuda_device, leaf):
    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200 import batch as B

    sets = _sets()
    pos = np.concatenate([p for p, _ in sets])
    mass = np.concatenate([m for _, m in sets])
    off = np.concatenate([[0], np.cumsum([len(p) for p, _ in sets])]).astype(np.int64)
    P = torch.from_numpy(pos).to(cuda_device)
    M = torch.from_numpy(mass).to(cuda_device)
    bt = B.build_trees_batched(P, M, off, leaf_size=leaf)
    bg = B.compute_tree_geometry_batched(bt)
    bi = B.build_interactions_and_neighbors_batched(bt, bg, theta=0.6, mac_type="dehnen")
    for i, (p, m) in enumerate(sets):
        pi, mi = torch.from_numpy(p).to(cuda_device), torch.from_numpy(m).to(cuda_device)
        t, ps, ms, inv = yb.build_tree(pi, mi, leaf_size=leaf, return_reordered=True)[:4]
        tb = bt.tree(i)
        for f in TOPO_FIELDS:
            _eq(f"set {i} {f}", getattr(tb, f), getattr(t, f))
        a, b = int(off[i]), int(off[i + 1])
        _eq(f"set {i} positions_sorted", bt.positions_sorted[a:b], ps)
        _eq(f"set {i} masses_sorted", bt.masses_sorted[a:b], ms)
        _eq(f"set {i} inverse", bt.inverse_permutation[a:b], inv)
        g = yb.compute_tree_geometry(t, ps)
        gb = bg.geometry(bt, i)
        for f in ("center", "half_extent", "radius", "max_extent"):
            _eq(f"set {i} {f}", getattr(gb, f), getattr(g, f))
        if int(t.num_internal_nodes) == 0:
            continue
        fi, ni_ = yb.build_interactions_and_neighbors(t, g, theta=0.6, mac_type="dehnen")
        fb, nb = bi.lists(bt, i)
        for f in FAR_FIELDS:
            _eq(f"set {i} far.{f}", getattr(fb, f), getattr(fi, f))
        for f in NEAR_FIELDS:
            _eq(f"set {i} near.{f}", getattr(nb, f), getattr(ni_, f))


def _flat(bt, bg, bi):
    return [x.detach().cpu().numpy().copy() for x in (
        bt.particle_indices, bt.morton_codes, bt.parent, bt.node_ranges, bt.nodes_by_level,
        bt.inverse_permutation, bg.center, bg.radius, bi.node_offsets, bi.far_counts,
        bi.sources, bi.targets, bi.target_levels, bi.near_offsets, bi.neighbors)]


def test_graph_pipeline_replays_equal_the_ordinary_path(cuda_device):
    """BatchedPipeline: the captured graph's replays return exactly what the
    ordinary batched functions return for the same inputs -- on the inputs it
    was captured with, on new positions, and (through a re-capture) on inputs
    whose lists outgrow the captured sizes."""
    import torch

    from yggdrax_b200 import batch as B
    from yggdrax_b200 import inputs

    pos, mass, off = inputs.batched_sets(48, 11, lo=16, hi=5000)
    P = torch.from_numpy(pos).to(cuda_device)
    M = torch.from_numpy(mass).to(cuda_device)

    def ordinary(p):
        bt = B.build_trees_batched(p, M, off, leaf_size=16)
        bg = B.compute_tree_geometry_batched(bt)
        bi = B.build_interactions_and_neighbors_batched(bt, bg, theta=0.6, mac_type="dehnen")
        return _flat(bt, bg, bi)

    pipe = B.BatchedPipeline(off, leaf_size=16, theta=0.6, mac_type="dehnen", margin=1.2,
                             device=cuda_device)
    first = _flat(*pipe(P, M))
    assert not pipe.last_replayed and pipe.captures == 1
    ref = ordinary(P)
    for a, b in zip(first, ref):
        assert np.array_equal(a, b)
    for step in range(3):  # new positions each call, same layout
        g = torch.Generator(device=cuda_device)
        g.manual_seed(step)
        P2 = (P * (1.0 + 0.02 * torch.rand(P.shape, device=cuda_device, generator=g))).contiguous()
        got = _flat(*pipe(P2, M))
        assert pipe.last_replayed
        for k, (a, b) in enumerate(zip(got, ordinary(P2))):
            assert np.array_equal(a, b), (step, k)
    # a pipeline whose capacities are too small on purpose: every replay
    # overflows, is flagged, and the call falls back to the ordinary path
    small = B.BatchedPipeline(off, leaf_size=16, theta=0.6, mac_type="dehnen", margin=0.5,
                              device=cuda_device)
    small(P, M)
    for k in range(2):
        got = _flat(*small(P, M))
        assert not small.last_replayed and small.captures == 2 + k
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)


def test_batched_c4_workload_sampled_sets_match_oracle(cuda_device, oracle):
    """The full batched workload (4096 sets, sizes floor(exp(U[ln 256,
    ln 65536])), half uniform cubes, half Plummer spheres, seed 3; about 48M
    points) built, measured and walked in one pass per stage; 48 sampled sets
    plus the smallest and the largest compared with the oracle run on that
    set alone (radix leaf 16, dehnen 0.6): topology, geometry and lists, bit
    for bit."""
    import torch

    from yggdrax_b200 import batch as B
    from yggdrax_b200 import inputs

    pos, mass, off = inputs.batched_sets(4096, 3)
    P = torch.from_numpy(pos).to(cuda_device)
    M = torch.from_numpy(mass).to(cuda_device)
    bt = B.build_trees_batched(P, M, off, leaf_size=16)
    bg = B.compute_tree_geometry_batched(bt)
    bi = B.build_interactions_and_neighbors_batched(bt, bg, theta=0.6, mac_type="dehnen")
    sizes = np.diff(off)
    rng = np.random.default_rng(17)
    pick = set(rng.choice(4096, size=48, replace=False).tolist())
    pick |= {int(np.argmin(sizes)), int(np.argmax(sizes))}
    for i in sorted(pick):
        a, b = int(off[i]), int(off[i + 1])
        ot = oracle.build_tree(pos[a:b], mass[a:b], leaf_size=16)
        tb = bt.tree(i)
        for f in ("parent", "left_child", "right_child", "particle_indices", "morton_codes",
                  "node_ranges", "node_level", "level_offsets", "nodes_by_level",
                  "bounds_min", "bounds_max", "leaf_codes"):
            _eq(f"set {i} {f}", getattr(tb, f), getattr(ot, f))
        _eq(f"set {i} positions_sorted", bt.positions_sorted[a:b], ot.positions_sorted)
        og = oracle.compute_tree_geometry(ot, ot.positions_sorted)
        gb = bg.geometry(bt, i)
        for f in ("center", "half_extent", "radius", "max_extent"):
            _eq(f"set {i} {f}", getattr(gb, f), getattr(og, f))
        if ot.num_internal_nodes == 0:
            continue
        r = oracle.build_interactions_and_neighbors(ot, og, theta=0.6, mac_type="dehnen")
        fb, nb = bi.lists(bt, i)
        _eq(f"set {i} far.counts", fb.counts, r["far_counts"])
        _eq(f"set {i} far.offsets", fb.offsets, r["offsets"])
        _eq(f"set {i} far.sources", fb.sources, r["sources"])
        _eq(f"set {i} far.targets", fb.targets, r["targets"])
        _eq(f"set {i} far.level_offsets", fb.level_offsets, r["level_offsets"])
        _eq(f"set {i} far.target_levels", fb.target_levels, r["target_levels"])
        _eq(f"set {i} near.counts", nb.counts, r["near_counts"])
        _eq(f"set {i} near.offsets", nb.offsets, r["near_offsets"])
        _eq(f"set {i} near.neighbors", nb.neighbors, r["neighbors"])
        _eq(f"set {i} near.leaf_indices", nb.leaf_indices, r["leaf_indices"])

"""Level-major geometry, dense M2L buffers and class-grouped far pairs on the
GPU: equal to the reference's own outputs (golden fixtures) on its small
cases and to the oracle on larger trees -- one where the packed class key
fits 64 bits and one where it needs the two-word sort."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
LM = ("centers", "half_extents", "radii", "max_extents", "level_counts", "node_indices")
DENSE = ("m2l_sources", "m2l_mask", "m2l_counts", "m2l_displacements")
GRP = ("class_keys", "class_displacements", "class_offsets", "class_sources", "class_targets",
       "class_ids")


def _eq(name, got, want):
    got = got.detach().cpu().numpy() if hasattr(got, "detach") else np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, (name, got.shape, want.shape)
    if want.dtype.kind == "f":
        assert np.array_equal(got.astype(want.dtype).view(np.uint32), want.view(np.uint32)), name
    else:
        assert np.array_equal(got.astype(np.int64), want.astype(np.int64)), name


def _pipeline(dev, pos, mass, leaf, theta, mac):
    import torch

    import yggdrax_b200 as yb

    P, M = torch.from_numpy(pos).to(dev), torch.from_numpy(mass).to(dev)
    t, ps = yb.build_tree(P, M, leaf_size=leaf, return_reordered=True)[:2]
    g = yb.compute_tree_geometry(t, ps)
    inter, _, grp = yb.build_interactions_and_neighbors(t, g, theta=theta, mac_type=mac,
                                                        return_grouped=True)
    lg = yb.geometry_to_level_major(t, g)
    dense = yb.densify_interactions(t, g, inter)
    return t, g, inter, lg, dense, grp


@pytest.mark.parametrize("case,theta,mac", [("uniform300_leaf4", 0.6, "dehnen"),
                                            ("plummer400_leaf8", 0.5, "bh")])
def test_buffers_match_reference_fixtures(cuda_device, case, theta, mac):
    z = np.load(os.path.join(HERE, "golden", f"buffers_{case}.npz"))
    a = np.load(os.path.join(HERE, "golden", f"adaptive_{case}.npz"))
    leaf = int(z["leaf"])
    _, _, _, lg, dense, grp = _pipeline(cuda_device, a["pos"], a["mass"], leaf, theta, mac)
    for k in LM:
        _eq(k, getattr(lg, k), z[f"lm_{k}"])
    for k in DENSE:
        _eq(k, getattr(dense, k), z[k])
    for k in GRP:
        _eq(k, getattr(grp, k), z[f"grp_{k}"])


@pytest.mark.parametrize("kind,n,leaf,theta,mac", [("uniform", 65536, 16, 0.6, "dehnen"),
                                                   ("plummer", 50000, 8, 0.5, "bh")])
def test_buffers_match_oracle(cuda_device, oracle, kind, n, leaf, theta, mac):
    from yggdrax_b200 import inputs

    pos, mass = inputs.uniform_cube(n, 7) if kind == "uniform" else inputs.plummer(n, 7)
    t, g, inter, lg, dense, grp = _pipeline(cuda_device, pos, mass, leaf, theta, mac)
    cpu = lambda x: x.detach().cpu().numpy()  # noqa: E731
    nlev = int(t.num_levels)
    olg = oracle.level_major_geometry(cpu(t.nodes_by_level), cpu(t.level_offsets), nlev,
                                      cpu(g.center), cpu(g.half_extent), cpu(g.radius),
                                      cpu(g.max_extent))
    for k in LM:
        _eq(k, getattr(lg, k), olg[k])
    od = oracle.dense_m2l(olg["node_indices"], cpu(inter.counts), cpu(inter.offsets),
                          cpu(inter.sources), cpu(g.center))
    for k in DENSE:
        _eq(k, getattr(dense, k), od[k])
    cnt = cpu(inter.counts)
    off = cpu(inter.offsets)
    src = np.concatenate([cpu(inter.sources)[off[k]:off[k] + cnt[k]] for k in range(cnt.shape[0])])
    tgt = np.repeat(np.arange(cnt.shape[0]), cnt)
    og = oracle.grouped_from_pairs(src, tgt, cpu(t.node_level), cpu(g.center), cpu(t.bounds_min),
                                   cpu(t.bounds_max))
    for k in GRP:
        _eq(k, getattr(grp, k), og[k])

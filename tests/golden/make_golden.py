"""Generate golden fixtures by running the reference yggdrax source.

Run in a container that has the reference checkout (its package directory,
the one holding ``tree.py``, is a required argument) but no JAX: the
reference modules are imported over
``jaxshim`` (NumPy with JAX's indexing / scatter / search semantics) and
executed on small seeded inputs.  The outputs are written as ``*.npz`` next
to this script and are what ``tests/test_golden.py`` checks the oracle
against.  Within-row order of the interaction / neighbour lists is
unspecified in the reference (unstable argsort), so rows are stored sorted.

Usage: python tests/golden/make_golden.py REFERENCE_PACKAGE_DIR
       [--mutual-only | --buffers-only | --moments-only | --octwalk-only]
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import jaxshim  # noqa: E402

TREE_FIELDS = ["parent", "left_child", "right_child", "left_is_leaf", "right_is_leaf",
               "particle_indices", "morton_codes", "node_ranges", "node_level", "level_offsets",
               "nodes_by_level", "num_levels", "bounds_min", "bounds_max", "leaf_codes",
               "leaf_depths"]
OCT_FIELDS = ["oct_parent", "oct_children", "oct_child_counts", "oct_child_mask",
              "oct_valid_mask", "oct_node_codes", "oct_node_depths", "oct_node_ranges",
              "oct_nodes_by_level", "oct_level_offsets", "oct_num_levels", "oct_leaf_mask",
              "oct_leaf_nodes", "radix_node_to_oct", "radix_leaf_to_oct"]


def _rows_sorted(offsets, counts, vals):
    out = np.array(vals, copy=True)
    for s, c in zip(np.asarray(offsets)[: len(counts)], np.asarray(counts)):
        if c > 1:
            out[s: s + c] = np.sort(out[s: s + c])
    return out


def _inputs():
    rng = np.random.default_rng(2024)
    uni = rng.uniform(-1, 1, (300, 3)).astype(np.float32)
    # Plummer-like radial profile (small)
    x = rng.uniform(0, 1, 400)
    r = 1.0 / np.sqrt(x ** (-2.0 / 3.0) - 1.0)
    r = np.minimum(r, 20.0)
    d = rng.normal(size=(400, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    plum = (r[:, None] * d).astype(np.float32)
    cl = np.concatenate([rng.normal(c, s, (200, 3)) for c, s in
                         [((-3, 0, 1), 0.05), ((2, 2, -1), 0.3), ((0, -2, 2), 0.02)]])
    clumps = cl.astype(np.float32)
    col = np.array([[float(i), 0.0, 0.0] for i in range(128)], np.float32)
    dup = np.zeros((16, 3), np.float32)
    return dict(uniform300=uni, plummer400=plum, clumps600=clumps, collinear128=col, dup16=dup)


def mutual(root: str) -> None:
    """dual_tree_walk_mutual (the canonical-pair emitter) on the reference's
    own trees and geometry: left / right children padded to all nodes with -1
    on leaves, bounding-sphere centres and radii as the MAC inputs, and
    capacities that fit as well as ones that overflow each buffer."""
    m = jaxshim.load_reference(root)
    jnp = sys.modules["jax.numpy"]
    ti, gi, ii, bd = m["_tree_impl"], m["_geometry_impl"], m["_interactions_impl"], m["bounds"]
    inputs = _inputs()
    for name, leaf in (("uniform300", 4), ("plummer400", 8), ("clumps600", 2)):
        pos = inputs[name]
        mass = np.linspace(0.5, 1.5, pos.shape[0]).astype(np.float32)
        p, ms = jnp.asarray(pos), jnp.asarray(mass)
        b = bd.infer_bounds(p)
        t, ps, _, _ = ti.build_tree(p, ms, b, leaf_size=leaf, return_reordered=True)
        g = gi.compute_tree_geometry(t, ps, max_leaf_size=leaf)
        total = int(np.asarray(t.parent).shape[0])
        ni = int(t.num_internal_nodes)
        lf = np.full(total, -1, np.int64)
        rt = np.full(total, -1, np.int64)
        lf[:ni] = np.asarray(t.left_child)
        rt[:ni] = np.asarray(t.right_child)
        out = dict(left=lf, right=rt, centers=np.asarray(g.center), radii=np.asarray(g.radius))
        q = 4096
        runs = [("fit", 0.6, q, 1 << 16, 1 << 16), ("fit_t4", 0.4, q, 1 << 16, 1 << 16),
                ("far_over", 0.6, q, 50, 1 << 16), ("near_over", 0.6, q, 1 << 16, 40),
                ("queue_over", 0.6, 24, 1 << 16, 1 << 16)]
        for tag, theta, q, fc, nc in runs:
            r = ii.dual_tree_walk_mutual(jnp.asarray(lf), jnp.asarray(rt), jnp.asarray(g.center),
                                         jnp.asarray(g.radius), theta, jnp.asarray(0),
                                         max_pair_queue=q, far_cap=fc, near_cap=nc)
            out[f"{tag}_params"] = np.array([theta, q, fc, nc], np.float64)
            for f in r._fields:
                out[f"{tag}_{f}"] = np.asarray(getattr(r, f))
        np.savez_compressed(os.path.join(HERE, f"mutual_{name}_leaf{leaf}.npz"), **out)
        print("wrote", f"mutual_{name}_leaf{leaf}")


def buffers(root: str) -> None:
    """Dense level-major M2L buffers and class-grouped far pairs, computed by
    the reference's own densify_interactions / geometry_to_level_major /
    build_grouped_interactions_from_pairs from its own tree, geometry and
    far lists (rows sorted, the canonical order both sides use), with the
    grouped input pairs in node order."""
    m = jaxshim.load_reference(root)
    jnp = sys.modules["jax.numpy"]
    ti, gi, ii, bd = m["_tree_impl"], m["_geometry_impl"], m["_interactions_impl"], m["bounds"]
    import importlib

    di = importlib.import_module("yggdrax.dense_interactions")
    gr = m["grouped_interactions"]
    inputs = _inputs()
    for name, leaf, theta, mac in (("uniform300", 4, 0.6, "dehnen"), ("plummer400", 8, 0.5, "bh")):
        pos = inputs[name]
        mass = np.linspace(0.5, 1.5, pos.shape[0]).astype(np.float32)
        p, ms = jnp.asarray(pos), jnp.asarray(mass)
        b = bd.infer_bounds(p)
        t, ps, _, _ = ti.build_tree(p, ms, b, leaf_size=leaf, return_reordered=True)
        g = gi.compute_tree_geometry(t, ps, max_leaf_size=leaf)
        inter, _ = ii.build_interactions_and_neighbors(t, g, theta=theta, mac_type=mac)
        srt = _rows_sorted(inter.offsets, inter.counts, inter.sources)
        inter = inter._replace(sources=jnp.asarray(srt))
        dense = di.densify_interactions(t, g, inter)
        lg = dense.geometry
        off, cnt = np.asarray(inter.offsets), np.asarray(inter.counts)
        src = np.concatenate([srt[off[k]:off[k] + cnt[k]] for k in range(cnt.shape[0])])
        tgt = np.repeat(np.arange(cnt.shape[0]), cnt)
        grp = gr.build_grouped_interactions_from_pairs(t, g, jnp.asarray(src), jnp.asarray(tgt),
                                                       level_offsets=inter.level_offsets)
        out = dict(theta=np.float64(theta), mac=np.array(mac), leaf=np.int64(leaf),
                   lm_centers=lg.centers, lm_half_extents=lg.half_extents, lm_radii=lg.radii,
                   lm_max_extents=lg.max_extents, lm_level_counts=lg.level_counts,
                   lm_node_indices=lg.node_indices, m2l_sources=dense.m2l_sources,
                   m2l_displacements=dense.m2l_displacements, m2l_mask=dense.m2l_mask,
                   m2l_counts=dense.m2l_counts, pair_sources=src, pair_targets=tgt)
        for f in grp._fields:
            out[f"grp_{f}"] = np.asarray(getattr(grp, f))
        np.savez_compressed(os.path.join(HERE, f"buffers_{name}_leaf{leaf}.npz"),
                            **{k: np.asarray(v) for k, v in out.items()})
        print("wrote", f"buffers_{name}_leaf{leaf}")


def moments(root: str) -> None:
    """compute_tree_mass_moments / compute_tree_multipole_moments (orders 0-4,
    about the centres of mass and about the geometric centres) on the
    reference's own trees."""
    m = jaxshim.load_reference(root)
    jnp = sys.modules["jax.numpy"]
    import importlib

    tm = importlib.import_module("yggdrax.tree_moments")
    ti, gi, bd = m["_tree_impl"], m["_geometry_impl"], m["bounds"]
    inputs = _inputs()
    for name, leaf in (("uniform300", 4), ("plummer400", 8)):
        pos = inputs[name]
        mass = np.linspace(0.5, 1.5, pos.shape[0]).astype(np.float32)
        p, ms = jnp.asarray(pos), jnp.asarray(mass)
        b = bd.infer_bounds(p)
        t, ps, msrt, _ = ti.build_tree(p, ms, b, leaf_size=leaf, return_reordered=True)
        g = gi.compute_tree_geometry(t, ps, max_leaf_size=leaf)
        mm = tm.compute_tree_mass_moments(t, ps, msrt)
        out = dict(mass=mm.mass, center_of_mass=mm.center_of_mass)
        for order in range(5):
            for tag, ctr in (("com", None), ("geo", jnp.asarray(g.center))):
                r = tm.compute_tree_multipole_moments(t, ps, msrt, expansion_centers=ctr,
                                                      max_order=order)
                for f in ("mass", "center", "dipole", "second_moment", "quadrupole",
                          "third_moment", "octupole", "fourth_moment", "hexadecapole",
                          "raw_packed"):
                    out[f"o{order}_{tag}_{f}"] = getattr(r, f)
                if order == 4:
                    out[f"o4_{tag}_packed2"] = tm.pack_multipole_expansions(r, 2)
        np.savez_compressed(os.path.join(HERE, f"moments_{name}_leaf{leaf}.npz"),
                            **{k: np.asarray(v) for k, v in out.items()})
        print("wrote", f"moments_{name}_leaf{leaf}")


def octree_native(root: str) -> None:
    """build_octree_native_far_pairs / build_octree_native_neighbor_lists on
    the reference's own octree topologies (adaptive and fixed depth), with
    capacities that fit and ones that overflow a far row or the queue (the
    error text is stored)."""
    m = jaxshim.load_reference(root)
    jnp = sys.modules["jax.numpy"]
    ti, oc, gi, ii, bd = (m["_tree_impl"], m["octree"], m["_geometry_impl"],
                          m["_interactions_impl"], m["bounds"])
    inputs = _inputs()
    # a jittered 8x8x8 lattice: every cell of a depth-2 (3) octree occupied,
    # so the octant-slot refinement keeps every child and both lists are full
    rng = np.random.default_rng(77)
    g = (np.stack(np.meshgrid(*[np.arange(8)] * 3, indexing="ij"), -1).reshape(-1, 3) + 0.5) / 4
    inputs["lattice512"] = (g - 1.0 + rng.uniform(-0.05, 0.05, g.shape)).astype(np.float32)
    inputs["uniform512"] = rng.uniform(-1, 1, (512, 3)).astype(np.float32)
    cases = (("uniform300", "adaptive", 4), ("plummer400", "adaptive", 8),
             ("clumps600", "fixed", 8), ("plummer400", "fixed", 4), ("lattice512", "fixed", 8),
             ("lattice512", "fixed", 1), ("uniform512", "fixed", 4))
    only = os.environ.get("OCTWALK_CASES")
    if only:
        cases = tuple(c for c in cases if f"{c[0]}_{c[1]}{c[2]}" in only.split(","))
    for name, kind, leaf in cases:
        pos = inputs[name]
        mass = np.linspace(0.5, 1.5, pos.shape[0]).astype(np.float32)
        p, ms = jnp.asarray(pos), jnp.asarray(mass)
        b = bd.infer_bounds(p)
        if kind == "fixed":
            t, ps, _, _ = ti.build_fixed_depth_tree(p, ms, b, target_leaf_particles=leaf,
                                                    refine_local=True, return_reordered=True)
            g = gi.compute_tree_geometry(t, ps)
        else:
            t, ps, _, _ = ti.build_tree(p, ms, b, leaf_size=leaf, return_reordered=True)
            g = gi.compute_tree_geometry(t, ps, max_leaf_size=leaf)
        aug = oc.augment_radix_topology_with_octree(t)
        view = oc.build_explicit_octree_traversal_view(aug)
        out = {f: np.asarray(getattr(aug, f)) for f in OCT_FIELDS}
        out.update(num_internal=np.int64(int(t.num_internal_nodes)),
                   radix_total=np.int64(int(np.asarray(t.parent).shape[0])),
                   bounds_min=np.asarray(t.bounds_min), bounds_max=np.asarray(t.bounds_max),
                   oct_to_radix_node=np.asarray(view.oct_to_radix_node),
                   oct_to_radix_leaf=np.asarray(view.oct_to_radix_leaf),
                   box_centers=np.asarray(view.box_centers),
                   box_half_extents=np.asarray(view.box_half_extents),
                   box_radii=np.asarray(view.box_radii),
                   box_max_extents=np.asarray(view.box_max_extents))
        q = 8192
        runs = [("dehnen06", 0.6, "dehnen", 512, 2048, q), ("bh05", 0.5, "bh", 512, 2048, q),
                ("far_over", 0.6, "dehnen", 3, 2048, q), ("near_over", 0.6, "dehnen", 512, 2, q),
                ("queue_over", 0.6, "dehnen", 512, 2048, 16)]
        for tag, theta, mac, fcap, ncap, qcap in runs:
            cfg = ii.DualTreeTraversalConfig(max_pair_queue=qcap, process_block=64,
                                             max_interactions_per_node=fcap,
                                             max_neighbors_per_leaf=ncap)
            out[f"{tag}_params"] = np.array([theta, fcap, ncap, qcap], np.float64)
            out[f"{tag}_mac"] = np.array(mac)
            try:
                fp = ii.build_octree_native_far_pairs(aug, g, theta=theta, mac_type=mac,
                                                      traversal_config=cfg)
                for f in fp._fields:
                    out[f"{tag}_far_{f}"] = np.asarray(getattr(fp, f))
            except RuntimeError as e:
                out[f"{tag}_far_error"] = np.array(str(e))
            try:
                nb = ii.build_octree_native_neighbor_lists(aug, g, theta=theta, mac_type=mac,
                                                           traversal_config=cfg)
                for f in ("offsets", "neighbors", "leaf_indices", "counts",
                          "particle_order_leaf_indices", "particle_order_to_native_leaf",
                          "neighbor_leaf_positions"):
                    out[f"{tag}_near_{f}"] = np.asarray(getattr(nb, f))
            except RuntimeError as e:
                out[f"{tag}_near_error"] = np.array(str(e))
        fname = f"octwalk_{name}_{kind}{leaf}"
        np.savez_compressed(os.path.join(HERE, f"{fname}.npz"), **out)
        print("wrote", fname, flush=True)


def main(root: str) -> None:
    m = jaxshim.load_reference(root)
    jnp = sys.modules["jax.numpy"]
    ti, oc, gi, ii, bd, mo = (m["_tree_impl"], m["octree"], m["_geometry_impl"],
                              m["_interactions_impl"], m["bounds"], m["morton"])
    inputs = _inputs()
    col_bounds = (np.array([-10.0, -1.0, -1.0], np.float32), np.array([10.0, 1.0, 1.0], np.float32))

    def save(name, **arrs):
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"),
                            **{k: np.asarray(v) for k, v in arrs.items()})
        print("wrote", name, len(arrs), "arrays")

    def tree_arrays(prefix, t):
        out = {}
        for f in TREE_FIELDS:
            out[f"{prefix}{f}"] = np.asarray(getattr(t, f))
        out[f"{prefix}num_internal_nodes"] = np.asarray(int(t.num_internal_nodes))
        return out

    def geometry_arrays(prefix, g):
        return {f"{prefix}center": g.center, f"{prefix}half_extent": g.half_extent,
                f"{prefix}radius": g.radius, f"{prefix}max_extent": g.max_extent}

    def walk_arrays(prefix, topo, g, theta, mac, cfg=None):
        kw = {} if cfg is None else {"traversal_config": cfg}
        inter, nbr = ii.build_interactions_and_neighbors(topo, g, theta=theta, mac_type=mac, **kw)
        return {
            f"{prefix}far_offsets": inter.offsets, f"{prefix}far_counts": inter.counts,
            f"{prefix}far_sources": _rows_sorted(inter.offsets, inter.counts, inter.sources),
            f"{prefix}far_targets": inter.targets,
            f"{prefix}far_level_offsets": inter.level_offsets,
            f"{prefix}far_target_levels": inter.target_levels,
            f"{prefix}near_offsets": nbr.offsets, f"{prefix}near_counts": nbr.counts,
            f"{prefix}near_neighbors": _rows_sorted(nbr.offsets, nbr.counts, nbr.neighbors),
            f"{prefix}near_leaf_indices": nbr.leaf_indices,
            f"{prefix}near_po_to_native": nbr.particle_order_to_native_leaf,
        }

    # -- L0: bounds, Morton codes, stable order ---------------------------------
    arrs = {}
    for name in ("uniform300", "plummer400", "clumps600"):
        p = jnp.asarray(inputs[name])
        b = bd.infer_bounds(p)
        c = mo.morton_encode_impl(p, b)
        arrs[f"{name}_pos"] = inputs[name]
        arrs[f"{name}_bmin"], arrs[f"{name}_bmax"] = b
        arrs[f"{name}_codes"] = c
        arrs[f"{name}_order"] = jnp.argsort(c, stable=True)
    p = jnp.asarray(inputs["collinear128"])
    arrs["collinear128_pos"] = inputs["collinear128"]
    arrs["collinear128_codes"] = mo.morton_encode_impl(p, (jnp.asarray(col_bounds[0]),
                                                          jnp.asarray(col_bounds[1])))
    save("morton", **arrs)

    # -- L1/L2/L3 on adaptive trees ---------------------------------------------
    for name, leaf in (("uniform300", 4), ("uniform300", 1), ("plummer400", 8), ("dup16", 1),
                       ("dup16", 4)):
        pos = inputs[name]
        mass = np.linspace(0.5, 1.5, pos.shape[0]).astype(np.float32)
        p, ms = jnp.asarray(pos), jnp.asarray(mass)
        b = bd.infer_bounds(p)
        t, ps, msrt, inv = ti.build_tree(p, ms, b, leaf_size=leaf, return_reordered=True)
        out = dict(pos=pos, mass=mass, positions_sorted=ps, masses_sorted=msrt, inverse=inv)
        out.update(tree_arrays("", t))
        g = gi.compute_tree_geometry(t, ps, max_leaf_size=leaf)
        out.update(geometry_arrays("geom_", g))
        aug = oc.augment_radix_topology_with_octree(t)
        for f in OCT_FIELDS:
            out[f] = np.asarray(getattr(aug, f))
        if name != "dup16" and leaf > 1:
            for theta, mac in ((0.6, "dehnen"), (0.5, "bh"), (0.5, "engblom")):
                out.update(walk_arrays(f"walk_{mac}_", t, g, theta, mac))
            out.update(walk_arrays("walkoct_dehnen_", aug, g, 0.6, "dehnen"))
            cfg = ii.DualTreeTraversalConfig(max_pair_queue=4096, process_block=64,
                                             max_interactions_per_node=256,
                                             max_neighbors_per_leaf=256)
            out.update(walk_arrays("padded_dehnen_", t, g, 0.6, "dehnen", cfg))
        save(f"adaptive_{name}_leaf{leaf}", **out)

    # -- fixed depth (+ local refinement) ---------------------------------------
    for name, target, bounds in (("clumps600", 8, None), ("collinear128", 8, col_bounds),
                                 ("plummer400", 4, None)):
        pos = inputs[name]
        mass = np.linspace(0.5, 1.5, pos.shape[0]).astype(np.float32)
        p, ms = jnp.asarray(pos), jnp.asarray(mass)
        b = bd.infer_bounds(p) if bounds is None else (jnp.asarray(bounds[0]),
                                                       jnp.asarray(bounds[1]))
        for refine in (True, False):
            t, ps, msrt, inv = ti.build_fixed_depth_tree(
                p, ms, b, target_leaf_particles=target, refine_local=refine,
                return_reordered=True)
            out = dict(pos=pos, mass=mass, positions_sorted=ps, masses_sorted=msrt, inverse=inv,
                       bmin_in=np.asarray(b[0]), bmax_in=np.asarray(b[1]))
            out.update(tree_arrays("", t))
            g = gi.compute_tree_geometry(t, ps)
            out.update(geometry_arrays("geom_", g))
            aug = oc.augment_radix_topology_with_octree(t)
            for f in OCT_FIELDS:
                out[f] = np.asarray(getattr(aug, f))
            if name != "collinear128":
                out.update(walk_arrays("walkoct_dehnen_", aug, g, 0.6, "dehnen"))
            save(f"fixed_{name}_t{target}_{'refine' if refine else 'plain'}", **out)

    # -- refinement helper on its own (pure NumPy in the reference) --------------
    rng = np.random.default_rng(5)
    pts = np.concatenate([rng.normal(0, [1.0, 0.01, 0.01], (300, 3)),
                          rng.normal(0.5, [0.02, 0.5, 0.02], (300, 3))]).astype(np.float32)
    p = jnp.asarray(pts)
    b = bd.infer_bounds(p)
    codes = np.asarray(mo.morton_encode_impl(p, b))
    order = np.argsort(codes, kind="stable")
    sc = codes[order]
    for depth in (1, 2):
        starts, ends, lc, ld = (np.asarray(a) for a in ti._fixed_depth_leaf_partitions(
            jnp.asarray(sc), depth, pts.shape[0]))
        r = ti._refine_leaf_partitions_by_aspect(pts[order], sc, starts.astype(np.int64),
                                                 ends.astype(np.int64), lc.astype(np.uint64),
                                                 ld.astype(np.int64), depth)
        save(f"refine_d{depth}", pos_sorted=pts[order], sorted_codes=sc, starts=starts,
             ends=ends, codes=lc, depths=ld, out_starts=r[0], out_ends=r[1], out_codes=r[2],
             out_depths=r[3])


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if len(args) != 1 or not os.path.isfile(os.path.join(args[0], "tree.py")):
        sys.exit("usage: make_golden.py REFERENCE_PACKAGE_DIR [--mutual-only | --buffers-only"
                 " | --moments-only | --octwalk-only]\n(the directory of the reference's"
                 " yggdrax package, which holds tree.py)")
    ref = args[0]
    if "--mutual-only" in sys.argv:
        mutual(ref)
    elif "--buffers-only" in sys.argv:
        buffers(ref)
    elif "--moments-only" in sys.argv:
        moments(ref)
    elif "--octwalk-only" in sys.argv:
        octree_native(ref)
    else:
        main(ref)
        mutual(ref)
        buffers(ref)
        moments(ref)
        octree_native(ref)

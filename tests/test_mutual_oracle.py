"""The mutual (canonical-pair) walk oracle against golden fixtures made by
running the reference's own dual_tree_walk_mutual (tests/golden/
make_golden.py --mutual-only): fitting capacities at two opening angles and
capacities that overflow the far list, the near list and the wavefront --
every array, count and flag equal, emission order included."""

import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "mutual_*.npz")))
RUNS = ("fit", "fit_t4", "far_over", "near_over", "queue_over")
FIELDS = ("far_a", "far_b", "far_count", "near_a", "near_b", "near_count", "far_overflow",
          "near_overflow", "queue_overflow")


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_mutual_oracle_matches_reference(oracle, path):
    z = np.load(path)
    for run in RUNS:
        theta, q, fc, nc = z[f"{run}_params"]
        got = oracle.dual_tree_walk_mutual(z["left"], z["right"], z["centers"], z["radii"],
                                               float(theta), 0, max_pair_queue=int(q),
                                               far_cap=int(fc), near_cap=int(nc))
        for f in FIELDS:
            want = z[f"{run}_{f}"]
            g = np.asarray(got[f])
            assert g.shape == want.shape and np.array_equal(g.astype(want.dtype), want), (run, f)


def test_mutual_oracle_covers_every_leaf_pair_once(oracle):
    """Completeness of the emitted pairs on a fitting run: every unordered
    pair of distinct leaves lies under exactly one far pair (as descendants
    of its two nodes) or is exactly one near pair."""
    z = np.load(FILES[0])
    left, right = z["left"], z["right"]
    r = oracle.dual_tree_walk_mutual(left, right, z["centers"], z["radii"], 0.6, 0,
                                         max_pair_queue=4096, far_cap=1 << 16, near_cap=1 << 16)
    total = left.shape[0]
    leaves_under = [None] * total

    def under(k):
        if leaves_under[k] is None:
            leaves_under[k] = [k] if left[k] < 0 else under(left[k]) + under(right[k])
        return leaves_under[k]

    leaves = [k for k in range(total) if left[k] < 0]
    idx = {k: i for i, k in enumerate(leaves)}
    cover = np.zeros((len(leaves), len(leaves)), np.int32)
    for a, b in zip(r["far_a"][:r["far_count"]], r["far_b"][:r["far_count"]]):
        assert a < b
        for x in under(int(a)):
            for y in under(int(b)):
                cover[idx[x], idx[y]] += 1
                cover[idx[y], idx[x]] += 1
    for a, b in zip(r["near_a"][:r["near_count"]], r["near_b"][:r["near_count"]]):
        assert a < b
        cover[idx[int(a)], idx[int(b)]] += 1
        cover[idx[int(b)], idx[int(a)]] += 1
    off = ~np.eye(len(leaves), dtype=bool)
    assert (cover[off] == 1).all() and (np.diag(cover) == 0).all()

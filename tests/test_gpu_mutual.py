"""The mutual (canonical-pair) walk on the GPU: equal to the reference's
own outputs (golden fixtures: every array, count and flag, emission order
included) and to the oracle on larger trees built by this library, with
fitting capacities and with each buffer overflowing."""

import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "mutual_*.npz")))
RUNS = ("fit", "fit_t4", "far_over", "near_over", "queue_over")
FIELDS = ("far_a", "far_b", "far_count", "near_a", "near_b", "near_count", "far_overflow",
          "near_overflow", "queue_overflow")


def _check(got, want, tag):
    for f in FIELDS:
        g = getattr(got, f).cpu().numpy()
        w = np.asarray(want[f])
        assert g.shape == w.shape and np.array_equal(g.astype(np.int64), w.astype(np.int64)), \
            (tag, f)


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_mutual_walk_matches_reference_fixtures(cuda_device, path):
    import torch

    import yggdrax_b200 as yb

    z = np.load(path)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda_device)  # noqa: E731
    for run in RUNS:
        theta, q, fc, nc = z[f"{run}_params"]
        got = yb.dual_tree_walk_mutual(t(z["left"]), t(z["right"]), t(z["centers"]),
                                       t(z["radii"]), float(theta), 0, max_pair_queue=int(q),
                                       far_cap=int(fc), near_cap=int(nc))
        _check(got, {f: z[f"{run}_{f}"] for f in FIELDS}, run)


@pytest.mark.parametrize("n,leaf,theta,caps", [
    (65536, 16, 0.6, (1 << 22, 1 << 22, 1 << 22)),
    (40000, 8, 0.5, (1 << 22, 1 << 22, 1 << 22)),
    (40000, 8, 0.5, (1 << 22, 5000, 1 << 22)),       # far list overflows
    (40000, 8, 0.5, (1 << 22, 1 << 22, 3000)),       # near list overflows
    (40000, 8, 0.5, (2000, 1 << 22, 1 << 22)),       # wavefront overflows
])
def test_mutual_walk_matches_oracle(cuda_device, oracle, n, leaf, theta, caps):
    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs

    pos, mass = inputs.plummer(n, 13) if leaf == 8 else inputs.uniform_cube(n, 13)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)
    tr, ps = yb.build_tree(P, M, leaf_size=leaf, return_reordered=True)[:2]
    g = yb.compute_tree_geometry(tr, ps)
    total, ni = int(tr.parent.shape[0]), int(tr.left_child.shape[0])
    lf = torch.full((total,), -1, dtype=torch.int64, device=cuda_device)
    rt = lf.clone()
    lf[:ni] = tr.left_child.to(torch.int64)
    rt[:ni] = tr.right_child.to(torch.int64)
    q, fc, nc = caps
    got = yb.dual_tree_walk_mutual(lf, rt, g.center, g.radius, theta, 0, max_pair_queue=q,
                                   far_cap=fc, near_cap=nc)
    want = oracle.dual_tree_walk_mutual(lf.cpu().numpy(), rt.cpu().numpy(),
                                        g.center.cpu().numpy(), g.radius.cpu().numpy(), theta, 0,
                                        max_pair_queue=q, far_cap=fc, near_cap=nc)
    _check(got, want, (n, leaf, theta, caps))

"""Tree mass / multipole moments on the GPU against the reference's own
outputs (golden fixtures, orders 0-4, about the centres of mass and about
the geometric centres) and against float64 sums on a larger tree.

Tolerance: the reference differences fp32 prefix sums over the particles
(sequentially summed), and this implementation does too with a parallel scan,
so the two agree to the rounding of those sums, not bit for bit.  The terms
that cancel in an order-k field are bounded by M (2R)^k (M the total mass, R
the largest |coordinate| of particles and centres), and a sum of n fp32
terms is off by at most about n eps of its magnitude: atol = 5e-5 M (2R)^k
for the 300-400 particle fixtures, rtol 1e-4."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIELDS = ("mass", "center", "dipole", "second_moment", "quadrupole", "third_moment", "octupole",
          "fourth_moment", "hexadecapole", "raw_packed")


ORDER = dict(mass=0, center=1, dipole=1, second_moment=2, quadrupole=2, third_moment=3,
             octupole=3, fourth_moment=4, hexadecapole=4)


def _close(name, got, want, scale):
    got = got.detach().cpu().numpy() if hasattr(got, "detach") else np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, (name, got.shape, want.shape)
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=5e-5 * scale, err_msg=name)


@pytest.mark.parametrize("case,leaf", [("uniform300_leaf4", 4), ("plummer400_leaf8", 8)])
def test_moments_match_reference_fixtures(cuda_device, case, leaf):
    import torch

    import yggdrax_b200 as yb

    a = np.load(os.path.join(HERE, "golden", f"adaptive_{case}.npz"))
    z = np.load(os.path.join(HERE, "golden", f"moments_{case}.npz"))
    P = torch.from_numpy(a["pos"]).to(cuda_device)
    M = torch.from_numpy(a["mass"]).to(cuda_device)
    t, ps, ms = yb.build_tree(P, M, leaf_size=leaf, return_reordered=True)[:3]
    g = yb.compute_tree_geometry(t, ps)
    Mt = float(a["mass"].sum())
    R = 2.0 * max(float(np.abs(a["pos"]).max()), float(np.abs(g.center.cpu().numpy()).max()))
    sc = lambda k: Mt * R ** k  # noqa: E731
    mm = yb.compute_tree_mass_moments(t, ps, ms)
    _close("mass", mm.mass, z["mass"], sc(0))
    _close("center_of_mass", mm.center_of_mass, z["center_of_mass"], R)
    for order in range(5):
        for tag, ctr in (("com", None), ("geo", g.center)):
            r = yb.compute_tree_multipole_moments(t, ps, ms, expansion_centers=ctr,
                                                  max_order=order)
            assert r.max_order == order
            for f in FIELDS:
                k = order if f == "raw_packed" else ORDER[f]
                _close(f"{order} {tag} {f}", getattr(r, f), z[f"o{order}_{tag}_{f}"],
                       R if f == "center" else sc(k))
            if order == 4:
                _close(f"{tag} packed2", yb.pack_multipole_expansions(r, 2),
                       z[f"o4_{tag}_packed2"], sc(2))


def test_mass_moments_against_float64(cuda_device):
    import torch

    import yggdrax_b200 as yb
    from yggdrax_b200 import inputs

    pos, mass = inputs.plummer(65536, 5)
    P, M = torch.from_numpy(pos).to(cuda_device), torch.from_numpy(mass).to(cuda_device)
    t, ps, ms = yb.build_tree(P, M, leaf_size=16, return_reordered=True)[:3]
    mm = yb.compute_tree_mass_moments(t, ps, ms)
    r = t.node_ranges.cpu().numpy()
    p64 = ps.cpu().numpy().astype(np.float64)
    m64 = ms.cpu().numpy().astype(np.float64)
    cm = np.concatenate([[0.0], np.cumsum(m64)])
    cw = np.concatenate([np.zeros((1, 3)), np.cumsum(m64[:, None] * p64, axis=0)])
    tot = cm[r[:, 1] + 1] - cm[r[:, 0]]
    com = (cw[r[:, 1] + 1] - cw[r[:, 0]]) / tot[:, None]
    got = mm.mass.cpu().numpy()
    # absolute error of a prefix difference: a few fp32 ulps of the total
    np.testing.assert_allclose(got, tot, rtol=0, atol=1e-5 * cm[-1])
    big = tot > 0.01 * cm[-1]  # centres of mass are meaningful where the mass is
    np.testing.assert_allclose(mm.center_of_mass.cpu().numpy()[big], com[big], rtol=0,
                               atol=1e-3 * np.abs(p64).max())

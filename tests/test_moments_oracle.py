"""Oracle of the tree mass / multipole moments against golden fixtures made
by running the reference's own compute_tree_mass_moments /
compute_tree_multipole_moments (tests/golden/make_golden.py --moments-only)
on its own trees: orders 0-4, about the centres of mass and about the
geometric centres."""

import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["uniform300_leaf4", "plummer400_leaf8"]
FIELDS = ("mass", "center", "dipole", "second_moment", "quadrupole", "third_moment", "octupole",
          "fourth_moment", "hexadecapole", "raw_packed")


@pytest.mark.parametrize("case", CASES)
def test_moments_oracle_matches_reference(oracle, case):
    t = np.load(os.path.join(HERE, "golden", f"adaptive_{case}.npz"))
    z = np.load(os.path.join(HERE, "golden", f"moments_{case}.npz"))
    m, c = oracle.tree_mass_moments(t["node_ranges"], t["positions_sorted"], t["masses_sorted"])
    assert np.array_equal(m, z["mass"]) and np.array_equal(c, z["center_of_mass"])
    for order in range(5):
        for tag, ctr in (("com", None), ("geo", t["geom_center"])):
            r = oracle.tree_multipole_moments(t["node_ranges"], t["positions_sorted"],
                                              t["masses_sorted"], ctr, order)
            for f in FIELDS:
                want = z[f"o{order}_{tag}_{f}"]
                got = np.asarray(r[f])
                assert got.shape == want.shape, (order, tag, f)
                np.testing.assert_allclose(got, want, rtol=2e-6, atol=1e-7 * (
                    float(np.abs(want).max()) + 1e-30), err_msg=f"{order} {tag} {f}")

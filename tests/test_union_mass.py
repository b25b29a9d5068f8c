"""Clump-template mass properties (nbc_union_mass) and the cfg2 / cfg4
template generator built on it.

The reference's template builder integrates the union of a clump's spheres
by Monte Carlo over its bounding box (make_clump_template_lambda.m:172-209).
Checked here against closed forms (one sphere; two equal spheres whose
overlap is a lens) and against an independent numpy Monte Carlo, and the
generated beds for their radius distribution and principal frames.
"""
import numpy as np
import pytest

import nbc
import scenegen as sg

pytestmark = pytest.mark.gpu


def test_one_sphere_closed_form():
    r, c = 2e-3, np.array([[1e-3, -2e-3, 0.5e-3]])
    vol, com, mom = nbc.union_mass(c, [r], [0, 1])
    assert abs(vol[0] / (4.0 / 3.0 * np.pi * r ** 3) - 1) < 1e-3
    assert np.abs(com[0] - c[0]).max() < 1e-3 * r
    # second moment of a ball per unit volume: r^2 / 5 on the diagonal
    assert np.abs(np.diag(mom[0]) / (r * r / 5) - 1).max() < 3e-3
    assert np.abs(mom[0] - np.diag(np.diag(mom[0]))).max() < 1e-3 * r * r


def test_two_spheres_lens():
    r, dist = 1.5e-3, 1.2e-3
    c = np.array([[0, 0, 0], [dist, 0, 0]])
    vol, com, _ = nbc.union_mass(c, [r, r], [0, 2])
    lens = np.pi * (4 * r + dist) * (2 * r - dist) ** 2 / 12.0
    exact = 2 * 4.0 / 3.0 * np.pi * r ** 3 - lens
    assert abs(vol[0] / exact - 1) < 1e-3
    assert abs(com[0, 0] - dist / 2) < 1e-3 * r and np.abs(com[0, 1:]).max() < 1e-3 * r


def test_matches_numpy_monte_carlo_and_is_deterministic():
    rng = np.random.default_rng(4)
    cen = rng.uniform(-1e-3, 1e-3, (5, 3))
    rad = rng.uniform(0.6e-3, 1.2e-3, 5)
    st = [0, 5]
    v1, c1, m1 = nbc.union_mass(cen, rad, st)
    v2, c2, m2 = nbc.union_mass(cen, rad, st)
    assert np.array_equal(v1, v2) and np.array_equal(c1, c2) and np.array_equal(m1, m2)
    M, com, I = sg.union_mass_properties(cen, rad, 1.0, samples=2_000_000, seed=3)
    assert abs(v1[0] / M - 1) < 5e-3
    assert np.abs(c1[0] - com).max() < 5e-3 * rad.max()
    I_gpu = v1[0] * (np.trace(m1[0]) * np.eye(3) - m1[0])
    assert np.abs(I_gpu - I).max() < 1e-2 * np.abs(I).max()


def test_poly_bed_templates():
    """cfg2-style templates: radii log-uniform per subsphere, members in the
    principal frame (centre of mass at the origin, diagonal inertia), clump
    mass split equally."""
    sc = sg.make_poly_bed(6000, 5, 0.05)
    r = sc["sub"]["radius"]
    lr = np.log(r)
    lo, hi = np.log(0.5e-3), np.log(5e-3)
    assert lr.min() >= lo - 1e-12 and lr.max() <= hi + 1e-12
    # log-uniform: each tenth of the log range holds about a tenth of the subspheres
    h, _ = np.histogram(lr, bins=10, range=(lo, hi))
    assert np.abs(h / len(r) - 0.1).max() < 0.03
    prop = sc["clump"]["prop"]
    assert (prop > 0).all()
    cid = sc["sub"]["clump_id"]
    K = len(prop)
    m = sc["sub"]["mass"]
    for k in range(0, K, max(1, K // 50)):
        sel = cid == k
        assert np.allclose(m[sel], prop[k, 3] / sel.sum())

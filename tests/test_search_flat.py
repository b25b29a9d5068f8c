"""The block-cooperative neighbour search (search_lanes = 1, k_search_flat).

It must build the reference's list exactly as the lane-group search does:
  * a dense lattice (spacing 0.6 r, about 3,400 candidates and 520 listed
    partners per subsphere) whose chunks span several bitmap windows and
    whose rows overflow the scratch rows (refilled by the compaction), against
    the FP64 oracle: pair list bit-exact;
  * the cfg1 contact-rich state (5 grid levels) and a polydisperse scene with
    a radius ratio of 10, against the oracle: sort order and pair list
    bit-exact, and 24 steps with rebuilds bitwise equal to the default search.
"""
import os

import numpy as np
import pytest

import nbc
import oracle
import scenegen as sg

pytestmark = pytest.mark.gpu


def _dense_lattice(n=14, r=1e-3, spacing=0.6):
    """n^3 spheres (one-sphere clumps) on a cubic lattice of spacing
    `spacing` r in a cube wall; a soft material so the overlaps stay
    harmless for one step."""
    a = spacing * r
    g = (np.arange(n) - (n - 1) / 2.0) * a
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + 0.02
    pos += np.random.default_rng(3).uniform(-0.05 * a, 0.05 * a, pos.shape)
    m = 2650 * 4 / 3 * np.pi * r ** 3
    K = len(pos)
    params = sg.default_params(StepSize=1e-8, EndStep=1, Thresh=1e-5, Gravity=0.0, Ymod=1e3,
                               BranchLmtLen=1400)
    lo, hi = pos.min(0) - 3 * r, pos.max(0) + 3 * r
    sg.set_world_box(params, lo, hi)
    quat = np.tile([0, 0, 0, 1.0], (K, 1))
    prop = np.tile([0.4 * m * r * r] * 3 + [m], (K, 1))
    return sg.assemble(params, pos, quat, np.zeros((K, 3)), np.zeros((K, 3)), prop,
                       [np.zeros((1, 3))] * K, [np.array([r])] * K, [np.array([m])] * K,
                       cube=sg.make_cube(0.5 * (hi - lo), 0.5 * (hi + lo)))


def _list_vs_oracle(sc, precision="f64"):
    e = nbc.Engine([sc], precision=precision, use_graph=False, tuned={"search_lanes": 1})
    e.step(1)
    e.sync()
    o = oracle.OracleScene(sc, threads=os.cpu_count() or 1)
    o.step(1)
    assert np.array_equal(e.subspheres()["part_fix"], o.sub()["part_fix"]), "sort order"
    la, lb = e.pairs()
    oa, ob = o.pairs()
    assert len(la) > 0
    assert np.array_equal(la, oa) and np.array_equal(lb, ob), "pair list"
    e.close()
    return len(la)


def test_flat_search_dense_lattice_windows_and_long_rows():
    sc = _dense_lattice()
    n = _list_vs_oracle(sc)
    # about 260 front entries per interior subsphere: far past the 32-entry
    # scratch rows, and 32 subspheres x ~3,400 candidates per chunk span
    # several 16,384-candidate windows
    assert n / len(sc["sub"]["radius"]) > 100


def test_flat_search_cfg1_contact_rich_state(golden_dir):
    sc = sg.tetra_state_from_npz(os.path.join(golden_dir, "cfg1_settled.npz"))
    assert len(sc["levels"]["cell"]) >= 3
    _list_vs_oracle(sc, precision="mixed")


def test_flat_search_radius_ratio_10():
    sc = nbc.with_levels(sg.make_test_poly(n_clumps=300, seed=11, rmin=0.5e-3, rmax=5e-3, max_members=3,
                                           dt=1e-7, bl=256))
    _list_vs_oracle(sc)


@pytest.mark.parametrize("precision", ["mixed", "f64"])
def test_flat_search_matches_lane_groups_over_rebuilds(precision):
    sc = nbc.with_levels(sg.make_test_poly(n_clumps=150, seed=5))
    out = []
    for lanes in (8, 1):
        e = nbc.Engine([sc], precision=precision, tuned={"search_lanes": lanes})
        e.step(24)
        e.sync()
        out.append((e.clumps(), e.pairs(), e.stats()["rebuilds"]))
        e.close()
    (ca, pa, ra), (cb, pb, rb) = out
    assert ra == rb >= 3
    for k in ("pos", "vel", "angvel", "quat"):
        assert np.array_equal(ca[k], cb[k]), k
    assert np.array_equal(pa[0], pb[0]) and np.array_equal(pa[1], pb[1])

"""Long list rows: a dense lattice (spacing 0.6 r, about 160 listed partners
per subsphere) whose rows far exceed the search's 32-entry scratch rows, so
the compaction searches them again straight into the list; pair list
bit-exact against the FP64 oracle.
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
    e = nbc.Engine([sc], precision=precision, use_graph=False, tuned=None)
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


def test_dense_lattice_long_rows():
    sc = _dense_lattice()
    n = _list_vs_oracle(sc)
    # far past the 32-entry scratch rows of the search
    assert n / len(sc["sub"]["radius"]) > 100

"""The autotuner (nbc_autotune): the launch shapes it chooses among change
no result, and its choice is a valid shape that is cached by scene shape."""
import os
import tempfile

import numpy as np
import pytest

import nbc
import scenegen as sg

pytestmark = pytest.mark.gpu


def test_every_launch_shape_gives_the_same_results():
    """Lanes of the neighbour search, members per lane of the clump pass and
    blocks per SM of the pair kernel: 24 steps with rebuilds, bitwise equal
    clump states and lists for every value the autotuner tries."""
    sc = nbc.with_levels(sg.make_test_poly(n_clumps=150, seed=5))
    ref = None
    for shape in ({}, {"search_lanes": 16}, {"search_lanes": 32}, {"clump_batch": 2}, {"clump_batch": 4},
                  {"pair_blocks": 4}, {"pair_blocks": 16}):
        e = nbc.Engine([sc], precision="mixed", tuned=shape)
        e.step(24)
        e.sync()
        out = (e.clumps(), e.pairs(), e.stats()["rebuilds"])
        e.close()
        if ref is None:
            ref = out
            assert ref[2] >= 3
            continue
        for k in ("pos", "vel", "angvel", "quat"):
            assert np.array_equal(out[0][k], ref[0][k]), (shape, k)
        assert np.array_equal(out[1][0], ref[1][0]) and np.array_equal(out[1][1], ref[1][1]), shape


def test_autotune_returns_a_valid_cached_choice():
    sc = sg.make_test_tetra(n_clumps=200, seed=7, intruder=None, steps=100)
    with tempfile.TemporaryDirectory() as d:
        cache = os.path.join(d, "tune.json")
        a = nbc.autotune([sc], trial_steps=60, cache=cache)
        assert a["search_lanes"] in (8, 16, 32) and a["clump_batch"] in (1, 2, 4)
        assert a["pair_blocks"] in (4, 8, 12, 16) and a["ms_per_step"] > 0 and not a["cached"]
        b = nbc.autotune([sc], trial_steps=60, cache=cache)
        assert b["cached"] and {k: b[k] for k in nbc.TUNED_KEYS} == {k: a[k] for k in nbc.TUNED_KEYS}
    e = nbc.Engine([sc], tuned=a)
    e.step(10)
    e.sync()
    assert e.stats()["err"] == 0
    e.close()

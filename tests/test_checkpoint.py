"""Exact checkpoint and resume (nbc_checkpoint_write / nbc_checkpoint_read).

The reference restarts from StartStep (src/world.par:28, the loop of
src/dem_simulation_clump.cu:110) by re-reading ph/ch snapshots, which drops
the tangential, rolling and twisting spring histories, so its resume is not
the continuous run.  The engine's checkpoint holds everything the next step
needs; a run saved after N steps, loaded into a fresh engine and stepped M
more steps must equal the continuous N + M step run bit for bit: clump
states, the pair list, the intruder record, and the step and rebuild counts.
"""
import os
import tempfile

import numpy as np
import pytest

import nbc
import scenegen as sg

pytestmark = pytest.mark.gpu


def _same(a, b):
    ca, cb = a.clumps(), b.clumps()
    for k in ("pos", "vel", "angvel", "quat", "force", "torque"):
        assert np.array_equal(ca[k], cb[k]), k
    pa, pb = a.pairs(), b.pairs()
    assert np.array_equal(pa[0], pb[0]) and np.array_equal(pa[1], pb[1])
    sa, sb = a.stats(), b.stats()
    assert (sa["steps"], sa["rebuilds"], sa["npairs"]) == (sb["steps"], sb["rebuilds"], sb["npairs"])


@pytest.mark.parametrize("precision", ["mixed", "f64"])
@pytest.mark.parametrize("name", ["tetra_gravity", "spheres_cube_sphere"])
def test_resume_equals_continuous(golden_dir, precision, name):
    sc = sg.scene_from_npz(os.path.join(golden_dir, f"{name}.scene.npz"))
    cont = nbc.Engine([sc], precision=precision)
    cont.step(37)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "ck.bin")
        cont.checkpoint(path)
        cont.step(40)
        cont.sync()
        res = nbc.Engine([sc], precision=precision)
        res.restore(path)
        res.step(40)
        res.sync()
    _same(cont, res)
    assert cont.stats()["rebuilds"] >= 10
    if sc.get("intruder") is not None:
        assert np.array_equal(cont.intruder()["reaction"], res.intruder()["reaction"])
        assert np.array_equal(cont.intruder_history(count=40), res.intruder_history(count=40))
    cont.close()
    res.close()


def test_resume_of_a_batch_and_a_cylinder(golden_dir):
    """Three scenes in one engine (cube wall with a sphere intruder, a
    cylinder wall, a hierarchical grid), saved at a step where only some of
    them rebuild; each scene resumes bitwise."""
    a = sg.scene_from_npz(os.path.join(golden_dir, "spheres_cube_sphere.scene.npz"))
    b = sg.make_test_cyl("tetra", seed=32, squeeze=0.9, dt=5e-7, thresh_ratio=1e-3)
    c = nbc.with_levels(sg.make_test_poly(n_clumps=60, seed=9))
    cont = nbc.Engine([a, b, c], precision="mixed")
    cont.step(23)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "ck.bin")
        cont.checkpoint(path)
        cont.step(30)
        cont.sync()
        res = nbc.Engine([a, b, c], precision="mixed")
        res.restore(path)
        res.step(30)
        res.sync()
    for s in range(3):
        ca, cb = cont.clumps(s), res.clumps(s)
        for k in ("pos", "vel", "angvel", "quat"):
            assert np.array_equal(ca[k], cb[k]), (s, k)
        assert cont.stats(s)["rebuilds"] == res.stats(s)["rebuilds"]


def test_checkpoint_refuses_other_scenes_and_precision(golden_dir):
    sc = sg.scene_from_npz(os.path.join(golden_dir, "tetra_gravity.scene.npz"))
    other = sg.scene_from_npz(os.path.join(golden_dir, "spheres_gac.scene.npz"))
    e = nbc.Engine([sc], precision="mixed")
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "ck.bin")
        with pytest.raises(nbc.NbcError) as err:
            e.checkpoint(path)          # no step yet: nothing to save
        assert err.value.code == -7
        e.step(5)
        e.checkpoint(path)
        for eng in (nbc.Engine([sc], precision="f64"), nbc.Engine([other], precision="mixed")):
            with pytest.raises(nbc.NbcError) as err:
                eng.restore(path)
            assert err.value.code == -1
            eng.close()
    e.close()

"""The drop-in executable and the device-side failure path.

  * `nbody-clump_b200/nbody_clump_b200` is the reference's main()
    (src/main.cpp:4-16) on the engine: run in a reference working directory
    (world.par, ph/ch .bt, Rocks/), it must write the OutPart, OutClump,
    OutForce and OutCnt files the reference writes there
    (tests/golden/spheres_cube_sphere.ref.npz, from the reference build).
  * ERR_NONFINITE: the reference aborts when a wall force is not finite
    (src/dem_force_cube_wall_clump.cu:295-331).  A scene whose inputs are
    all finite but whose Young's modulus (1e300) overflows the FP32 contact
    law -- and, in FP64, the positions after a few steps -- must come back as
    NBC_ERR_NONFINITE from the device's own check, with the context still
    usable (no trap, no fault) and a healthy engine unaffected.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import nbc
import refbin
import scenegen as sg

pytestmark = pytest.mark.gpu

EXE = os.path.join(os.path.dirname(nbc.__file__), "nbody_clump_b200")


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_dropin_executable_writes_reference_outputs(golden_dir):
    name = "spheres_cube_sphere"
    sc = sg.scene_from_npz(os.path.join(golden_dir, f"{name}.scene.npz"))
    g = np.load(os.path.join(golden_dir, f"{name}.ref.npz"))
    with tempfile.TemporaryDirectory() as d:
        sg.write_reference_inputs(sc, d)
        r = subprocess.run([EXE], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, timeout=300)
        out = r.stdout.decode(errors="replace")
        assert r.returncode == 0, out[-2000:]
        assert "Final!!" in out
        for s in (1, 12, 24):
            ph = refbin.read_ph(os.path.join(d, "OutPart", "ph.%08d.bin" % s))
            ch = refbin.read_ch(os.path.join(d, "OutClump", "ch.%08d.bin" % s))
            assert np.array_equal(ph["part_fix"], g[f"s{s}/part_fix"]), s
            assert _rel(ph["pos"], g[f"s{s}/pos"]) < 1e-12
            assert _rel(ch["pos"], g[f"s{s}/clump_pos"]) < 1e-12
            assert _rel(ch["vel"], g[f"s{s}/clump_vel"]) < 1e-8
            fc = refbin.read_fc(os.path.join(d, "OutForce", "fc.%08d.bin" % s))
            ref = g[f"s{s}/intr_force"]
            assert np.abs(fc["force"] - ref).max() <= 1e-8 * max(1e-3, np.abs(ref).max())
        for s in (2, 12, 24):
            nei = refbin.read_cnt(os.path.join(d, "OutCnt", "Nei.%08d.bin" % s), np.int32)
            rows, slots = np.nonzero(nei >= 0)
            assert np.array_equal(rows, g[f"c{s}/rows"]) and np.array_equal(nei[rows, slots], g[f"c{s}/nei"])


def test_dropin_executable_reports_missing_inputs():
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([EXE], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, timeout=120)
        assert r.returncode != 0
        assert "DEMClumpMain" in r.stdout.decode(errors="replace")


@pytest.mark.parametrize("precision", ["mixed", "f64"])
def test_device_nonfinite_flag(precision):
    bad = sg.make_test_tetra(n_clumps=60, seed=41, intruder=None, steps=40)
    bad["params"]["Ymod"] = 1e300          # finite, but no force law survives it
    good = sg.make_test_tetra(n_clumps=60, seed=42, intruder=None, steps=40)
    e_bad = nbc.Engine([bad], precision=precision, use_graph=True)
    e_good = nbc.Engine([good], precision=precision, use_graph=True)
    with pytest.raises(nbc.NbcError) as err:
        for _ in range(40):
            e_bad.step(1)
    assert err.value.code == -4, err.value
    assert e_bad.stats()["err"] & 2
    # the context is intact: the healthy engine on the same GPU steps on
    e_good.step(40)
    e_good.sync()
    assert e_good.stats()["err"] == 0 and e_good.stats()["steps"] == 40
    assert np.isfinite(e_good.clumps()["pos"]).all()
    e_bad.close()
    e_good.close()

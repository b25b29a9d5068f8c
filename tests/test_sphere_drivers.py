"""The sphere-only drivers of the reference (class DEMmain, src/dem.h:31-99)
on the engine: `nbody-clump_b200/nbody_sphere_b200 <driver>` (DEMmain on the
C ABI, nbc_open_sphere + nbc_run) in a sphere-format working directory must
write the OutPart/ph.N.bin files the reference's own driver writes there
(tests/golden/<case>.ref.npz, made by tests/golden/make_ref_golden.py with
the reference build's oracle/_ref/nbody_sphere_ref):

  * sph_cube   RunSimulation2 (src/dem_simulation_cube.cu): compressed
               spheres in the cube with a sphere intruder and cohesion; the
               cube wall without history or moments, the penetrator law with
               cohesion, the first half-kick without the intruder, OutCnt;
  * sph_cyl    RunSimulation (src/dem_simulation_cylind.cu): compressed
               spheres in the closed cylinder with a cylinder intruder, a
               rebuild every few steps: pair histories restart from zero at
               every rebuild (the driver's second pointer exchange);
  * sph_hgrid  RunSimulation_HGrid (src/dem_simulation_hgrid.cu): two sphere
               sizes on two grid levels from grid.bt;
  * sph_split  RunSimulation_Split (src/dem_simulation_split.cu): free,
               driven and fixed spheres (src/dem_integrate_withglue.cu);
  * cyl_spheres RunSimulation with wall contacts only.

Sort order bit-exact, positions to 1e-12 and velocities to 1e-8 of their
scale at every step, the intruder's force history to 1e-8.  The hgrid case is
pinned to the oracle instead: the reference's hgrid list build races and its
run breaks action-reaction (test_reference_hgrid_driver_breaks_action_reaction).
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import nbc
import refbin
import scenegen as sg

EXE = os.path.join(os.path.dirname(nbc.__file__), "nbody_sphere_b200")
CASES = {"sph_cube": "cube", "sph_cyl": "cylinder", "sph_hgrid": "hgrid", "sph_split": "split",
         "cyl_spheres": "cylinder"}
# cases pinned to the reference's own run (the hgrid driver's list build
# races, see test_reference_hgrid_driver_breaks_action_reaction)
REF_PINNED = sorted(set(CASES) - {"sph_hgrid"})


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _by_original(part_fix, a):
    out = np.empty_like(a)
    out[part_fix] = a
    return out


def _scene(golden_dir, name):
    return sg.scene_from_npz(os.path.join(golden_dir, f"{name}.scene.npz"))


# --------------------------------------------------------------------------
# CPU: the fixtures and the input writer
# --------------------------------------------------------------------------

@pytest.mark.parametrize("name", sorted(CASES))
def test_sphere_fixtures_are_one_sphere_clumps(golden_dir, name):
    sc = _scene(golden_dir, name)
    K = len(sc["clump"]["pos"])
    assert len(sc["sub"]["radius"]) == K and np.array_equal(sc["sub"]["clump_id"], np.arange(K))
    assert np.abs(sc["sub"]["local"]).max() == 0.0
    g = np.load(os.path.join(golden_dir, f"{name}.ref.npz"))
    assert int(g["steps"]) == 24 and g["s24/pos"].shape == (K, 3)


def test_sphere_fixtures_exercise_their_driver(golden_dir):
    """Each case reaches what its driver does differently: the intruder in
    contact and cohesion on (cube), rebuilds with touching pairs (cylinder),
    two levels (hgrid), all three body kinds (split)."""
    cube = _scene(golden_dir, "sph_cube")
    assert cube["params"]["Cohesion"] > 0 and cube["params"]["isIntruder"] == 1 and cube["cube"] is not None
    cyl = _scene(golden_dir, "sph_cyl")
    assert cyl["cylinder"] is not None and cyl["params"]["isIntruder"] == 1
    hg = _scene(golden_dir, "sph_hgrid")
    assert set(np.unique(hg["levels"]["level"])) == {0, 1}
    r = hg["sub"]["radius"]
    assert r.max() / r.min() >= 2.4
    sp = _scene(golden_dir, "sph_split")
    assert set(np.unique(sp["body_kind"])) == {0, 1, 2}
    # The reference's split driver passes the original index where its first
    # half-kick expects Type (src/dem_simulation_split.cu:84-85 against
    # src/dem_integrate_withglue.cu:113-114): sphere 0 moves freely, sphere 1
    # is driven at (-0.2 y, -0.2 x, 0) (src/dem_integrate_withglue.cu:47-54),
    # every other sphere stays where it is, whatever its Type
    g = np.load(os.path.join(golden_dir, "sph_split.ref.npz"))
    pos = _by_original(g["s24/part_fix"], g["s24/pos"])
    p0 = sp["clump"]["pos"]
    assert np.array_equal(pos[2:], p0[2:])
    assert np.abs(pos[0] - p0[0]).max() > 0
    dt = sp["params"]["StepSize"]
    pred = p0[1].copy()
    for _ in range(24):
        pred = pred + dt * np.array([-0.2 * pred[1], -0.2 * pred[0], 0.0])
    assert np.array_equal(pos[1], pred)
    # its closing half-kick goes by Type (src/dem_integrate_withglue.cu:140):
    # the velocities of Type 0 spheres change, the others' do not
    vel = _by_original(g["s24/part_fix"], g["s24/vel"])
    v0 = sp["clump"]["vel"]
    k = sp["body_kind"]
    rest = np.arange(len(k)) >= 2
    assert np.array_equal(vel[rest & (k != 0)], v0[rest & (k != 0)])
    assert (np.abs(vel[rest & (k == 0)] - v0[rest & (k == 0)]).max(1) > 0).all()


@pytest.mark.parametrize("name", REF_PINNED)
def test_oracle_matches_reference_sphere_driver(golden_dir, name):
    """The oracle's restatement of the sphere drivers (integrator, sphere
    laws, memoryless cube wall, penetrator cohesion, history reset, the split
    driver's kinds) against the reference's own run of the driver, every one
    of 24 steps (CPU): sort order bit-exact, states to 1e-13, the intruder's
    position exact and its reaction to 1e-13 of its scale."""
    import oracle
    driver = CASES[name]
    sc = _scene(golden_dir, name)
    g = np.load(os.path.join(golden_dir, f"{name}.ref.npz"))
    o = oracle.OracleScene(sg.as_sphere_driver(sc, driver))
    for s in range(1, int(g["steps"]) + 1):
        o.step(1)
        pf = g[f"s{s}/part_fix"]
        assert np.array_equal(o.sub()["part_fix"], pf), f"step {s}: sort order"
        c = o.clumps()
        for k in ("pos", "vel", "angvel", "quat"):
            assert _rel(c[k], _by_original(pf, g[f"s{s}/{k}"])) < 1e-13, (s, k)
        if f"s{s}/intr_force" in g:
            it = o.intruder()
            assert np.array_equal(it["pos"], g[f"s{s}/intr_pos"]), s
            ref = g[f"s{s}/intr_force"][0]
            assert np.abs(it["reaction"] - ref).max() <= 1e-13 * max(1e-3, np.abs(ref).max()), s
    assert o.rebuilds >= 2


def test_reference_hgrid_driver_breaks_action_reaction(golden_dir):
    """The reference's hgrid list build races: a large sphere's thread
    appends its same-level partners with a plain read-modify-write of its
    front count (src/dem_hgrid_contlist.cu:124-127) while small spheres'
    threads append cross-level entries to the same row with atomicAdd
    (:149-152), so entries are lost and the back references of the lost
    pairs are never written.  Its step-1 forces therefore do not cancel in
    pairs: the internal forces sum to newtons where the wall forces sum to
    a tenth of one.  The engine's hgrid driver is pinned to the oracle (the
    race-free list) instead of this run."""
    sc = _scene(golden_dir, "sph_hgrid")
    g = np.load(os.path.join(golden_dir, "sph_hgrid.ref.npz"))
    v1 = _by_original(g["s1/part_fix"], g["s1/vel"])
    m = sc["clump"]["prop"][:, 3]
    dt = sc["params"]["StepSize"]
    gz = np.array([0.0, 0.0, sc["params"]["Gravity"]])
    F = (v1 - sc["clump"]["vel"] - dt * gz) * m[:, None] / (0.5 * dt)
    assert np.abs(F.sum(0)).max() > 1.0
    # the oracle's race-free list on the same scene: the pair forces cancel,
    # what is left is the wall's force
    import oracle
    o = oracle.OracleScene(sg.as_sphere_driver(sc, "hgrid"))
    o.step(1)
    Fo = (o.clumps()["vel"] - sc["clump"]["vel"] - dt * gz) * m[:, None] / (0.5 * dt)
    fw = o.sub_forces()["fw"].sum(0)
    assert np.abs(Fo.sum(0) - fw).max() < 1e-9 * np.abs(Fo).max()


@pytest.mark.parametrize("driver", ["cylinder", "cube", "split", "hgrid"])
def test_write_sphere_inputs_layout(golden_dir, driver):
    name = {"cylinder": "sph_cyl", "cube": "sph_cube", "split": "sph_split", "hgrid": "sph_hgrid"}[driver]
    sc = _scene(golden_dir, name)
    with tempfile.TemporaryDirectory() as d:
        sg.write_sphere_inputs(sc, d, driver)
        rows = np.loadtxt(os.path.join(d, sc["params"]["IniConFile"]))
        assert rows.shape == (len(sc["clump"]["pos"]), 21)
        assert np.array_equal(rows[:, 3:6], sc["clump"]["pos"])
        assert np.array_equal(rows[:, 20], sc["sub"]["radius"])
        wall = "CubeWall.bt" if driver == "cube" else "CylindWall.bt"
        assert os.path.exists(os.path.join(d, "Rocks", wall))
        assert os.path.exists(os.path.join(d, "Rocks", "Penetrator.bt"))
        if driver == "split":
            assert np.array_equal(rows[:, 2], sc["body_kind"])
        if driver == "hgrid":
            grid = np.loadtxt(os.path.join(d, "grid.bt"))
            assert grid.shape == (2, 7) and np.array_equal(rows[:, 2], sc["levels"]["level"])
            n = grid[:, 2] * grid[:, 3] * grid[:, 4]
            assert grid[1, 5] == n[0]


def _open_sphere_status(d, driver):
    import ctypes as C
    h = C.c_void_p()
    rc = nbc.lib().nbc_open_sphere(d.encode(), nbc.SPHERE_DRIVERS[driver] if isinstance(driver, str) else driver,
                                   None, C.byref(h))
    if rc == 0:
        nbc.lib().nbc_destroy(h)
    return rc, nbc.lib().nbc_last_error().decode()


@pytest.mark.parametrize("name", sorted(CASES))
def test_open_sphere_parses_every_driver(golden_dir, name):
    """nbc_open_sphere reads each driver's working directory (world.par, the
    21-column ph, the driver's wall, Penetrator.bt, grid.bt); the engine then
    needs a CUDA device (no CPU fallback)."""
    from conftest import cuda_available
    sc = _scene(golden_dir, name)
    with tempfile.TemporaryDirectory() as d:
        sg.write_sphere_inputs(sc, d, CASES[name])
        rc, msg = _open_sphere_status(d, CASES[name])
        assert rc == (0 if cuda_available() else -5), msg


def _remove(rel):
    def f(d):
        os.remove(os.path.join(d, rel))
    return f


def _edit(rel, fn):
    def f(d):
        p = os.path.join(d, rel)
        open(p, "w").write(fn(open(p).read()))
    return f


def _ph_type(value):
    def f(d):
        p = os.path.join(d, "ph.00000000.bt")
        lines = open(p).read().splitlines()
        cols = lines[3].split()
        cols[2] = str(value)
        lines[3] = " ".join(cols)
        open(p, "w").write("\n".join(lines) + "\n")
    return f


@pytest.mark.parametrize("name,driver,mutate,needle", [
    ("sph_cube", "cube", _remove("Rocks/CubeWall.bt"), "CubeWall.bt"),
    ("sph_cyl", "cylinder", _remove("Rocks/CylindWall.bt"), "CylindWall.bt"),
    ("sph_cyl", "cylinder", _remove("Rocks/Penetrator.bt"), "Penetrator.bt"),
    ("sph_hgrid", "hgrid", _remove("grid.bt"), "grid.bt"),
    ("sph_hgrid", "hgrid", _ph_type(2), "not a grid level"),
    ("sph_split", "split", _ph_type(5), "Type must be 0, 1 or 2"),
    ("sph_cube", "cube", _edit("ph.00000000.bt", lambda t: "\n".join(t.splitlines()[:-3]) + "\n"),
     "short or malformed"),
])
def test_open_sphere_rejects_bad_inputs(golden_dir, name, driver, mutate, needle):
    """Missing or malformed inputs come back as NBC_ERR_IO with the file
    named (the reference exits, src/dem_io.cu:196-199,
    src/dem_penetrator_io.cu:21-27), before any device work."""
    sc = _scene(golden_dir, name)
    with tempfile.TemporaryDirectory() as d:
        sg.write_sphere_inputs(sc, d, driver)
        mutate(d)
        rc, msg = _open_sphere_status(d, driver)
        assert rc == -3 and needle in msg, (rc, msg)


def test_open_sphere_rejects_unknown_driver(golden_dir):
    sc = _scene(golden_dir, "sph_cyl")
    with tempfile.TemporaryDirectory() as d:
        sg.write_sphere_inputs(sc, d, "cylinder")
        rc, msg = _open_sphere_status(d, 7)
        assert rc == -1 and "driver" in msg


# --------------------------------------------------------------------------
# GPU: the drop-in executable against the reference's drivers
# --------------------------------------------------------------------------

def _run(sc, driver, d):
    sg.write_sphere_inputs(sc, d, driver)
    r = subprocess.run([EXE, driver], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, timeout=300)
    out = r.stdout.decode(errors="replace")
    assert r.returncode == 0, out[-2000:]
    assert "Final!!" in out


@pytest.mark.gpu
@pytest.mark.parametrize("name", REF_PINNED)
def test_dropin_sphere_driver_matches_reference(golden_dir, name):
    driver = CASES[name]
    sc = _scene(golden_dir, name)
    g = np.load(os.path.join(golden_dir, f"{name}.ref.npz"))
    with tempfile.TemporaryDirectory() as d:
        _run(sc, driver, d)
        for s in range(1, int(g["steps"]) + 1):
            ph = refbin.read_sphere_ph(os.path.join(d, "OutPart", "ph.%08d.bin" % s))
            pf = g[f"s{s}/part_fix"]
            assert np.array_equal(ph["sorted_id"], np.arange(len(pf)))
            if driver != "hgrid":
                assert np.array_equal(ph["part_fix"], pf), f"step {s}: sort order"
            for k, tol in (("pos", 1e-12), ("vel", 1e-8), ("angvel", 1e-8), ("quat", 1e-12)):
                mine = _by_original(ph["part_fix"], ph[k])
                ref = _by_original(pf, g[f"s{s}/{k}"])
                assert _rel(mine, ref) < tol, (s, k, _rel(mine, ref))
            if f"s{s}/intr_force" in g:
                it = refbin.read_ch(os.path.join(d, "OutPart", "intruder.%08d.bin" % s))
                assert it["id"][0] == -1 and len(it["id"]) == 1
                assert _rel(it["pos"][0], g[f"s{s}/intr_pos"]) < 1e-12
                fc = refbin.read_fc(os.path.join(d, "OutForce", "fc.%08d.bin" % s))
                ref = g[f"s{s}/intr_force"]
                assert np.abs(fc["force"] - ref).max() <= 1e-8 * max(1e-3, np.abs(ref).max()), s
            if f"c{s}/rows" in g:
                nei = refbin.read_cnt(os.path.join(d, "OutCnt", "Nei.%08d.bin" % s), np.int32)
                rows, slots = np.nonzero(nei >= 0)
                assert np.array_equal(rows, g[f"c{s}/rows"]) and np.array_equal(nei[rows, slots], g[f"c{s}/nei"])


@pytest.mark.gpu
def test_dropin_hgrid_driver_matches_oracle(golden_dir):
    """RunSimulation_HGrid on two sphere sizes and two levels of grid.bt
    against the oracle's race-free hierarchical grid, every step: sort order
    and states to rounding (no intruder, so the driver's kinematics are the
    clump path's except for the sphere laws' lever arms, which the oracle
    restates too)."""
    import oracle
    sc = _scene(golden_dir, "sph_hgrid")
    orc = oracle.OracleScene(sg.as_sphere_driver(sc, "hgrid"))
    with tempfile.TemporaryDirectory() as d:
        _run(sc, "hgrid", d)
        for s in range(1, 25):
            orc.step(1)
            ph = refbin.read_sphere_ph(os.path.join(d, "OutPart", "ph.%08d.bin" % s))
            assert np.array_equal(ph["part_fix"], orc.sub()["part_fix"]), f"step {s}: sort order"
            co = orc.clumps()
            for k, tol in (("pos", 1e-12), ("vel", 1e-9), ("angvel", 1e-9), ("quat", 1e-12)):
                mine = _by_original(ph["part_fix"], ph[k])
                assert _rel(mine, co[k]) < tol, (s, k, _rel(mine, co[k]))
    assert orc.rebuilds >= 5


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sph_cyl", "sph_cube"])
def test_sphere_behaviour_is_needed(golden_dir, name):
    """Without the driver's own behaviour (pair histories carried by pair in
    the cylinder driver; the clump path's cube wall with history and
    moments) the engine leaves the reference's results: the golden cases
    tell the behaviours apart."""
    sc = dict(_scene(golden_dir, name))
    sc["sphere_mode"] = nbc.SPHERE_KINEMATICS
    sc["params"] = dict(sc["params"], isWallForce=1)
    g = np.load(os.path.join(golden_dir, f"{name}.ref.npz"))
    eng = nbc.Engine([sc], precision="f64", use_graph=False)
    eng.step(24)
    eng.sync()
    ce = eng.clumps()
    ref = _by_original(g["s24/part_fix"], g["s24/vel"])
    assert _rel(ce["vel"], ref) > 1e-6
    eng.close()


@pytest.mark.gpu
def test_sphere_engine_in_memory_matches_dropin(golden_dir):
    """The same sphere-driver behaviour through nbc.Engine (scene in memory,
    scenegen.as_sphere_driver) gives the drop-in's states bit for bit."""
    sc = _scene(golden_dir, "sph_cyl")
    eng = nbc.Engine([sg.as_sphere_driver(sc, "cylinder")], precision="f64", use_graph=True)
    eng.step(24)
    eng.sync()
    ce, se = eng.clumps(), eng.subspheres()
    eng.close()
    with tempfile.TemporaryDirectory() as d:
        _run(sc, "cylinder", d)
        ph = refbin.read_sphere_ph(os.path.join(d, "OutPart", "ph.%08d.bin" % 24))
    assert np.array_equal(ph["part_fix"], se["part_fix"])
    assert np.array_equal(_by_original(ph["part_fix"], ph["pos"]), ce["pos"])
    assert np.array_equal(_by_original(ph["part_fix"], ph["vel"]), ce["vel"])


@pytest.mark.gpu
def test_dropin_sphere_driver_reports_missing_inputs():
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([EXE, "cube"], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, timeout=120)
        assert r.returncode != 0
        assert "DEMmain" in r.stdout.decode(errors="replace")

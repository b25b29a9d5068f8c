"""The closed cylinder wall (the wall of the cfg1 scene).

The reference's clump path has only a cube wall; its closed cylinder wall
lives on the sphere-only driver (CylindWallInteraction_cuk + ForceWall_cuk,
src/dem_force_cylind_wall.cu:3-237, driven by DEMmain::RunSimulation,
src/dem_simulation_cylind.cu:3-211).  A scene of one-sphere clumps with
LocalPos = 0 makes the clump kinematics the sphere kinematics, so:

  * the oracle is pinned against the reference's sphere driver run on the
    `cyl_spheres` scene (tests/golden/cyl_spheres.ref.npz, made by
    tests/golden/make_ref_golden.py): every sphere presses on the bottom
    cap, the top cap, the side or a cap edge, spheres never touch each
    other, and the list is rebuilt every few steps;
  * the engine is checked against the sphere driver's outputs and against
    the oracle on that scene and on tetrahedral clumps pressed into the
    caps, the side and the edges (`make_test_cyl("tetra")`, inter-clump
    contacts as well): sort order and pair lists bit-exact, FP64 states to
    rounding, FP64 wall forces to 1e-10 of the force scale, FP32 law per
    contact within 1e-5 of the FP64 oracle;
  * the oracle's wall law matches the Hertz formula on a static overlap.
"""
import os

import numpy as np
import pytest

import oracle
import scenegen as sg


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _cyl_spheres(golden_dir):
    return sg.scene_from_npz(os.path.join(golden_dir, "cyl_spheres.scene.npz"))


def _cyl_tetra():
    return sg.make_test_cyl("tetra", seed=32, squeeze=0.9, dt=5e-7, thresh_ratio=1e-3)


def _regions(sc):
    """Subspheres overlapping the bottom cap, the top cap, the side, and
    both a cap and the side (an edge), at the scene's start."""
    cy = sc["cylinder"]
    rel = sc["sub"]["pos"] - cy["centre"]
    r = sc["sub"]["radius"]
    side = np.hypot(rel[:, 0], rel[:, 1]) + r - cy["radius"] > 0
    bot = -rel[:, 2] + r - cy["half_height"] > 0
    top = rel[:, 2] + r - cy["half_height"] > 0
    return bot, top, side, side & (bot | top)


def _by_original(part_fix, a):
    out = np.empty_like(a)
    out[part_fix] = a
    return out


@pytest.mark.parametrize("which", ["spheres", "tetra"])
def test_scenes_touch_every_region(golden_dir, which):
    sc = _cyl_spheres(golden_dir) if which == "spheres" else _cyl_tetra()
    bot, top, side, edge = _regions(sc)
    assert bot.sum() >= 3 and top.sum() >= 3 and side.sum() >= 3 and edge.sum() >= 2, \
        (bot.sum(), top.sum(), side.sum(), edge.sum())


def test_oracle_matches_reference_sphere_driver(golden_dir):
    """The oracle's clump-kinematics cylinder wall against the reference's
    sphere driver, every step of 24 (CPU)."""
    sc = _cyl_spheres(golden_dir)
    g = np.load(os.path.join(golden_dir, "cyl_spheres.ref.npz"))
    o = oracle.OracleScene(sc)
    for s in range(1, int(g["steps"]) + 1):
        o.step(1)
        c = o.clumps()
        pf = g[f"s{s}/part_fix"]
        # the sphere driver's arrays are in its sorted order; sphere k is clump k
        for k, tol in (("pos", 1e-12), ("vel", 1e-10), ("angvel", 1e-10)):
            ref = _by_original(pf, g[f"s{s}/{k}"])
            assert _rel(c[k], ref) < tol, (s, k, _rel(c[k], ref))
        assert np.abs(c["quat"] - _by_original(pf, g[f"s{s}/quat"])).max() < 1e-12
        assert np.array_equal(o.sub()["part_fix"], pf), f"step {s}: sort order"
    assert o.rebuilds >= 5


@pytest.mark.parametrize("where", ["bottom", "top", "side"])
def test_oracle_cylinder_hertz_static(where):
    """One sphere at rest pressed into the wall by delta, no gravity: the
    wall force after one step is the Hertz force (2/3) E/(1-nu^2) sqrt(R)
    delta^1.5 along the wall normal (Kn of src/dem_force_cylind_wall.cu:43
    times Dn), with no tangential part."""
    r, Rc, H, delta = 1e-3, 10e-3, 8e-3, 2e-5
    c = np.array([0.02, 0.02, 0.02])
    p = {"bottom": (0, 0, -(H - r + delta)), "top": (0, 0, H - r + delta), "side": (Rc - r + delta, 0, 0)}[where]
    pos = c + np.array([p])
    m = 2650 * 4 / 3 * np.pi * r ** 3
    params = sg.default_params(StepSize=1e-7, EndStep=1, Thresh=1e-4, Gravity=0.0, BranchLmtLen=16)
    sg.set_world_box(params, np.zeros(3), 2 * c)
    sc = sg.assemble(params, pos, np.array([[0, 0, 0, 1.0]]), np.zeros((1, 3)), np.zeros((1, 3)),
                     np.array([[0.4 * m * r * r] * 3 + [m]]), [np.zeros((1, 3))], [np.array([r])],
                     [np.array([m])], cylinder=sg.make_cylinder(Rc, H, c))
    o = oracle.OracleScene(sc)
    o.step(1)
    fw = o.sub_forces()["fw"][0]
    E, nu = params["Ymod"], params["Prat"]
    F = 2.0 / 3.0 * E / (1 - nu * nu) * np.sqrt(r) * delta ** 1.5
    n = {"bottom": (0, 0, 1.0), "top": (0, 0, -1.0), "side": (-1.0, 0, 0)}[where]
    assert np.abs(fw - F * np.array(n)).max() <= 1e-12 * F


# --------------------------------------------------------------------------
# engine (GPU) against the sphere driver and the oracle
# --------------------------------------------------------------------------

@pytest.mark.gpu
def test_engine_matches_reference_sphere_driver(golden_dir):
    """The engine (FP64) directly against the reference sphere driver's
    outputs on the cyl_spheres scene, every step."""
    import nbc
    sc = _cyl_spheres(golden_dir)
    g = np.load(os.path.join(golden_dir, "cyl_spheres.ref.npz"))
    eng = nbc.Engine([sc], precision="f64", use_graph=True)
    for s in range(1, int(g["steps"]) + 1):
        eng.step(1)
        eng.sync()
        c = eng.clumps()
        pf = g[f"s{s}/part_fix"]
        assert np.array_equal(eng.subspheres()["part_fix"], pf), f"step {s}: sort order"
        for k, tol in (("pos", 1e-12), ("vel", 1e-9), ("angvel", 1e-9)):
            assert _rel(c[k], _by_original(pf, g[f"s{s}/{k}"])) < tol, (s, k)
        assert np.abs(c["quat"] - _by_original(pf, g[f"s{s}/quat"])).max() < 1e-12
    assert eng.stats()["rebuilds"] >= 5 and eng.stats()["err"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["spheres", "tetra"])
def test_engine_matches_oracle_every_step_f64(golden_dir, which):
    """24 steps in FP64: sort order and pair lists bit-exact at every step,
    wall forces per subsphere within 1e-10 of the force scale, clump states
    to rounding; at least 5 list rebuilds."""
    import nbc
    sc = _cyl_spheres(golden_dir) if which == "spheres" else _cyl_tetra()
    eng = nbc.Engine([sc], precision="f64", use_graph=False)
    orc = oracle.OracleScene(sc)
    for s in range(24):
        eng.step_export(1)
        eng.sync()        # the closing half-kick, as the oracle's step ends with it
        orc.step(1)
        assert np.array_equal(eng.subspheres()["part_fix"], orc.sub()["part_fix"]), f"step {s + 1}: order"
        la, lb = eng.pairs()
        oa, ob = orc.pairs()
        assert np.array_equal(la, oa) and np.array_equal(lb, ob), f"step {s + 1}: pairs"
        parts, of = eng.force_parts(), orc.sub_forces()
        scale = np.abs(of["fw"]).max() + np.abs(of["fc"]).max()
        assert scale > 0
        for k in ("fw", "tw", "fc"):
            assert np.abs(parts[k] - of[k]).max() <= 1e-10 * max(scale, np.abs(of[k]).max()), (s + 1, k)
        ce, co = eng.clumps(), orc.clumps()
        for k in ("pos", "quat"):
            assert _rel(ce[k], co[k]) < 1e-12, (s + 1, k)
        for k in ("vel", "angvel"):
            assert _rel(ce[k], co[k]) < 1e-10, (s + 1, k)
    assert eng.stats()["rebuilds"] >= 5 and orc.rebuilds == eng.stats()["rebuilds"]
    assert (np.abs(orc.sub_forces()["fw"]).sum(1) > 0).sum() >= 5


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["spheres", "tetra"])
def test_engine_mixed_per_contact_1e5(golden_dir, which):
    """FP32 contact law: the wall force on every touching subsphere and the
    pair forces within 1e-5 (relative to the force on it) of the FP64 oracle
    after the first step."""
    import nbc
    sc = _cyl_spheres(golden_dir) if which == "spheres" else _cyl_tetra()
    eng = nbc.Engine([sc], precision="mixed", use_graph=False)
    orc = oracle.OracleScene(sc)
    eng.step_export(1)
    orc.step(1)
    parts, of = eng.force_parts(), orc.sub_forces()
    fmax = np.abs(of["fw"]).max() + np.abs(of["fc"]).max()
    for k in ("fw", "fc"):
        mag = np.linalg.norm(of[k], axis=1)
        on = mag > 1e-6 * fmax
        err = np.linalg.norm(parts[k] - of[k], axis=1)
        if on.any():
            assert (err[on] / mag[on]).max() <= 1e-5, (k, (err[on] / mag[on]).max())
        assert err.max() <= 1e-5 * fmax

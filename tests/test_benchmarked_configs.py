"""Parity at the configurations the benchmark runs, and long-horizon checks of
the mixed-precision law.

  * cfg1 in its contact-rich state (the benchmark's start state,
    tests/golden/cfg1_settled.npz: 200,000 subspheres of lognormal tetra
    clumps, the closed cylinder wall, 5 grid levels from the level chooser):
    one step on the engine and on the FP64 oracle from that state -- sort
    order and pair list bit-exact, every contact's normal force within 1e-5
    (mixed law) or 1e-9 (FP64) of the oracle;
  * a cfg2-like polydisperse bed (radii 0.5-5 mm, a radius ratio of 10, the
    level chooser's grid levels), settled on the engine and then checked the
    same way;
  * cfg0 (2,000 spheres settling for 10,000 steps) in both precisions
    against the reference's own FP64 run: bed heights and the bulk packing
    fraction within 0.01 (the benchmark's long-run acceptance);
  * a penetration force-depth curve under the mixed law against the FP64
    engine on the same bed: RMS relative difference below 5% once the
    intruder is R_I/2 deep.
"""
import os

import numpy as np
import pytest

import oracle
import scenegen as sg

pytestmark = pytest.mark.gpu

SNAP = "cfg1_settled.npz"


def _per_contact(fe, fo, floor=1e-6):
    mag = np.linalg.norm(fo, axis=1)
    big = mag > floor * mag.max()
    err = np.linalg.norm(fe - fo, axis=1)
    return (err[big] / mag[big]).max(), int(big.sum())


def _one_step_vs_oracle(scene, precision, tol, min_contacts=1000):
    import nbc
    eng = nbc.Engine([scene], precision=precision, use_graph=False)
    eng.step_export(1)
    orc = oracle.OracleScene(scene, threads=os.cpu_count() or 1)
    orc.step(1)
    assert np.array_equal(eng.subspheres()["part_fix"], orc.sub()["part_fix"]), "sort order"
    la, lb = eng.pairs()
    oa, ob = orc.pairs()
    assert np.array_equal(la, oa) and np.array_equal(lb, ob), "pair list"
    fo = orc.pair_caches()["cfcn"]
    rel, n = _per_contact(eng.pair_forces(), fo)
    assert n > min_contacts, f"only {n} contacts: not a contact-rich state"
    assert rel <= tol, f"per-contact normal force error {rel:.2e} over {n} contacts"
    parts, of = eng.force_parts(), orc.sub_forces()
    scale = np.abs(fo).max()
    for k in ("fc", "fw"):
        assert np.abs(parts[k] - of[k]).max() <= 10 * tol * scale, k
    eng.close()
    return n


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-5), ("f64", 1e-9)])
def test_cfg1_contact_rich_state_first_step(golden_dir, precision, tol):
    scene = sg.tetra_state_from_npz(os.path.join(golden_dir, SNAP))
    assert scene["cylinder"] is not None and len(scene["levels"]["cell"]) >= 3
    _one_step_vs_oracle(scene, precision, tol)


def test_cfg1_contact_rich_state_ten_steps_f64(golden_dir):
    """Ten steps from the snapshot in FP64: the list stays bit-exact with the
    oracle across the rebuilds in between, states to rounding."""
    import nbc
    scene = sg.tetra_state_from_npz(os.path.join(golden_dir, SNAP))
    eng = nbc.Engine([scene], precision="f64", use_graph=True)
    orc = oracle.OracleScene(scene, threads=os.cpu_count() or 1)
    eng.step(10)
    eng.sync()        # the closing half-kick, as the oracle's step ends with it
    orc.step(10)
    assert eng.stats()["rebuilds"] == orc.rebuilds >= 2
    la, lb = eng.pairs()
    oa, ob = orc.pairs()
    assert np.array_equal(la, oa) and np.array_equal(lb, ob)
    ce, co = eng.clumps(), orc.clumps()
    for k in ("pos", "quat"):
        assert np.abs(ce[k] - co[k]).max() <= 1e-12 * np.abs(co[k]).max(), k
    for k in ("vel", "angvel"):
        assert np.abs(ce[k] - co[k]).max() <= 1e-8 * np.abs(co[k]).max(), k


_SETTLED = {}


def _poly_bed_settled(n_sub=6000, steps=50000):
    """A cfg2-style bed (clumps of 1-8 subspheres, radii 0.5-5 mm) in a 12 x 12
    cm cube wall, settled on the engine from its seeded layers (0.36 s: the
    9 cm tall seeding falls and comes to rest)."""
    import nbc
    key = (n_sub, steps)
    if key not in _SETTLED:
        bed = nbc.with_levels(sg.make_poly_bed(n_sub, 20260901, 0.06))
        e = nbc.Engine([bed], precision="mixed")
        e.step(steps)
        _SETTLED[key] = e.restart_scene(bed)
        e.close()
    return _SETTLED[key]


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-5), ("f64", 1e-9)])
def test_cfg2_radius_ratio_10_first_step(precision, tol):
    """Polydisperse clumps with radii 0.5-5 mm (a radius ratio of 10, as in
    cfg2) on the level chooser's grid (5 levels), packed closer than their
    extent: the hierarchical-grid list bit-exact and per-contact forces
    within tol of the FP64 oracle.  (A settled cfg2 bed cannot be checked
    this way: its 5 mm spheres touch hundreds of small ones, more than the
    oracle's fixed-width rows of the reference's layout hold.)"""
    import nbc
    sc = nbc.with_levels(sg.make_test_poly(n_clumps=300, seed=11, rmin=0.5e-3, rmax=5e-3, max_members=3,
                                           dt=1e-7, bl=256))
    r = sc["sub"]["radius"]
    assert r.max() / r.min() > 8.0
    assert len(sc["levels"]["cell"]) >= 3
    _one_step_vs_oracle(sc, precision, tol, min_contacts=500)


def _packing_fraction(pos, r, lo, hi, n=400_000, seed=3):
    """Solid fraction of the box [lo, hi] by seeded Monte Carlo (spheres of
    one radius r)."""
    from scipy.spatial import cKDTree
    pts = np.random.default_rng(seed).uniform(lo, hi, (n, 3))
    d, _ = cKDTree(pos).query(pts, k=1)
    return float((d <= r).mean())


@pytest.mark.parametrize("precision", ["mixed", "f64"])
def test_cfg0_settled_bed_matches_reference_run(golden_dir, precision):
    """10,000 steps of cfg0 (the reference's FP64 CUDA run is the golden):
    mean and top height within 0.05 r and 0.5 r, and the bulk packing
    fraction (at least 3 r from every wall and 3 r below the top) within
    0.01.  The trajectories decorrelate after a few thousand steps (chaos),
    so the settled bed, not the particles, is compared."""
    import nbc
    sc = sg.scene_from_npz(os.path.join(golden_dir, "cfg0_settle.scene.npz"))
    g = np.load(os.path.join(golden_dir, "cfg0_settle.ref.npz"))
    eng = nbc.Engine([sc], precision=precision)
    eng.step(10000)
    eng.sync()
    pos = eng.clumps()["pos"]
    ref = g["s10000/clump_pos"]
    r = float(sc["sub"]["radius"][0])
    assert abs(pos[:, 2].mean() - ref[:, 2].mean()) < 0.05 * r
    assert abs(pos[:, 2].max() - ref[:, 2].max()) < 0.5 * r
    cube = sc["cube"]
    lo = cube["centre"] - cube["half"] + 3 * r
    hi = cube["centre"] + cube["half"] - 3 * r
    hi[2] = min(pos[:, 2].max(), ref[:, 2].max()) - 3 * r
    phi_e, phi_r = _packing_fraction(pos, r, lo, hi), _packing_fraction(ref, r, lo, hi)
    assert 0.45 < phi_r < 0.7
    assert abs(phi_e - phi_r) <= 0.01, (phi_e, phi_r)
    assert eng.stats()["err"] == 0


def test_force_depth_curve_mixed_against_f64():
    """A sphere intruder (R_I = 8 mm, 0.2 m/s) pushed into a settled
    polydisperse bed: the reaction-force curve of the mixed law against the
    FP64 engine on the same bed, RMS relative difference below 5% over the
    samples at least R_I/2 past the first contact (the FP64 run goes on until
    it is 3 R_I/4 past its first contact, the mixed run takes as many steps)."""
    import nbc
    st = _poly_bed_settled()
    Ri, v = 8e-3, 0.2
    # on the bed's surface, not on the few subspheres its fall threw up
    sc = sg.with_sphere_intruder(st, Ri, v, surface=98)
    dt = float(sc["params"]["StepSize"])
    sample = max(1, int(round(0.02 * Ri / (v * dt))))
    max_samples = 200   # 4 R_I of travel at most
    z0 = float(sc["intruder"]["pos"][2])
    curves = {}
    n_samples = None
    for prec in ("f64", "mixed"):
        e = nbc.Engine([sc], precision=prec)
        c = []
        first = None
        while True:
            e.step(sample)
            it = e.intruder()
            c.append((z0 - float(it["pos"][2]), float(it["reaction"][2])))
            if n_samples is not None:
                if len(c) == n_samples:
                    break
                continue
            if first is None and abs(c[-1][1]) > 1e-3:
                first = c[-1][0]
            if (first is not None and c[-1][0] - first >= 0.75 * Ri) or len(c) == max_samples:
                n_samples = len(c)
                break
        assert e.stats()["err"] == 0
        e.close()
        curves[prec] = np.array(c)
    dm, fm = curves["mixed"].T
    df, ff = curves["f64"].T
    assert np.allclose(dm, df)
    first = np.argmax(np.abs(ff) > 1e-3 * np.abs(ff).max())
    deep = dm - dm[first] >= 0.5 * Ri
    assert deep.sum() >= 10 and np.abs(ff[deep]).max() > 0.1
    rms = np.sqrt(np.mean((fm[deep] - ff[deep]) ** 2)) / np.sqrt(np.mean(ff[deep] ** 2))
    assert rms < 0.05, rms

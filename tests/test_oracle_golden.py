"""The CPU oracle against the reference's own outputs (CPU only).

The golden vectors (tests/golden/*.ref.npz) were produced by running the
unmodified reference solver (built by oracle/Makefile.ref) on a B200 with the
inputs in tests/golden/*.scene.npz; see tests/golden/make_ref_golden.py.
They pin the oracle, which in turn is the checker for the GPU engine.
"""
import os

import numpy as np
import pytest

import oracle
import scenegen as sg

SHORT = ["ref_fixture", "spheres_cube_sphere", "tetra_cube_cyl", "tetra_gravity", "spheres_gac"]


def _load(golden_dir, name):
    sc = sg.scene_from_npz(os.path.join(golden_dir, f"{name}.scene.npz"))
    g = np.load(os.path.join(golden_dir, f"{name}.ref.npz"))
    return sc, g


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", SHORT)
def test_oracle_matches_reference_every_step(golden_dir, name):
    sc, g = _load(golden_dir, name)
    p = sc["params"]
    o = oracle.OracleScene(sc)
    off = 1 if p["isIntruder"] else 0
    steps = int(g["steps"])
    rebuilds_seen = 0
    for s in range(1, steps + 1):
        o.step(1)
        sub, c = o.sub(), o.clumps()
        # sort order (ParticleID in sorted order) is bit-exact
        assert np.array_equal(sub["part_fix"], g[f"s{s}/part_fix"]), f"step {s}: sort order"
        assert _rel(sub["pos"], g[f"s{s}/pos"]) < 1e-12
        assert _rel(c["pos"], g[f"s{s}/clump_pos"][off:]) < 1e-12
        assert _rel(c["vel"], g[f"s{s}/clump_vel"][off:]) < 1e-10
        assert _rel(c["angvel"], g[f"s{s}/clump_angvel"][off:]) < 1e-10
        assert np.abs(c["quat"] - g[f"s{s}/clump_quat"][off:]).max() < 1e-12
        if p["isIntruder"]:
            it = o.intruder()
            ref_f = g[f"s{s}/intr_force"][0]
            assert np.abs(it["reaction"] - ref_f).max() <= 1e-10 * max(1.0, np.abs(ref_f).max())
            assert np.abs(it["pos"] - g[f"s{s}/clump_pos"][0]).max() < 1e-14
        if f"c{s}/rows" in g:
            anei, ng, ni = o.rows()
            rows, slots = np.nonzero(anei >= 0)
            assert np.array_equal(rows, g[f"c{s}/rows"]), f"step {s}: list rows"
            assert np.array_equal(slots, g[f"c{s}/slots"]), f"step {s}: list slots"
            assert np.array_equal(anei[rows, slots], g[f"c{s}/nei"]), f"step {s}: list partners"
            if f"c{s}/fcn" in g:
                f, cp = o.chain()
                ref = g[f"c{s}/fcn"]
                assert np.abs(f[rows, slots] - ref).max() <= 1e-11 * np.abs(ref).max()
                assert np.abs(cp[rows, slots] - g[f"c{s}/cpt"]).max() < 1e-14
        rebuilds_seen = o.rebuilds
    if name != "ref_fixture":
        assert rebuilds_seen >= 5, "the case is meant to exercise the history carry"


def test_oracle_cfg0_settling_prefix(golden_dir):
    """2,000 spheres settling: exact agreement while the trajectories are
    still correlated (the first 2,000 steps, with two list comparisons)."""
    sc, g = _load(golden_dir, "cfg0_settle")
    o = oracle.OracleScene(sc, threads=4)
    o.step(1000)
    sub, c = o.sub(), o.clumps()
    assert np.array_equal(sub["part_fix"], g["s1000/part_fix"])
    assert _rel(c["pos"], g["s1000/clump_pos"]) < 1e-12
    o.step(1000)
    anei, ng, ni = o.rows()
    rows, slots = np.nonzero(anei >= 0)
    assert np.array_equal(rows, g["c2000/rows"]) and np.array_equal(anei[rows, slots], g["c2000/nei"])


def test_oracle_damping_matches_restitution_formula():
    # LoadParameters (src/dem_subsphere_io.cu:143-145)
    e = 0.2
    ln = np.log(e)
    ref = 2.0 * np.sqrt(5.0 / 6.0) * ln / np.sqrt(ln * ln + 3.14159265359 ** 2)
    assert abs(sg.damping_from_restitution(e) - ref) < 1e-15


def test_oracle_threads_do_not_change_results():
    """The reference arm of the benchmark runs the oracle on every host
    thread, the parity tests mostly on one: its lists and states are the
    same bit for bit on 1 and 4 threads (each subsphere's sums run in a
    fixed order whatever the thread that owns it)."""
    import nbc
    sc = nbc.with_levels(sg.make_test_poly(n_clumps=120, seed=5))
    a, b = oracle.OracleScene(sc, threads=1), oracle.OracleScene(sc, threads=4)
    a.step(60)
    b.step(60)
    assert a.rebuilds == b.rebuilds and a.rebuilds > 5
    ca, cb = a.clumps(), b.clumps()
    for k in ca:
        assert np.array_equal(ca[k], cb[k]), k
    for x, y in zip(a.pairs(), b.pairs()):
        assert np.array_equal(x, y)

"""The B200 engine against the CPU oracle and the reference's own outputs.

Bars (from the engine's contract):
  * cell sort order and contact pair lists bit-exact;
  * FP64 engine: states and per-contact forces within 1e-9 relative of the
    oracle (rounding only: the GPU evaluates the same expressions with FMA);
  * mixed precision (FP32 contact law): per-contact forces within 1e-5
    relative of the FP64 oracle after one step;
  * graph and eager execution, and repeated runs, bitwise identical.
"""
import os
import tempfile

import numpy as np
import pytest

import nbc
import oracle
import refbin
import scenegen as sg

pytestmark = pytest.mark.gpu

CASES = ["ref_fixture", "spheres_cube_sphere", "tetra_cube_cyl", "tetra_gravity", "spheres_gac"]


def _scene(golden_dir, name):
    return sg.scene_from_npz(os.path.join(golden_dir, f"{name}.scene.npz"))


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _contact_rel_err(f_eng, f_ref, floor=1e-6):
    """max relative error over contacts whose force exceeds floor * max."""
    mag = np.linalg.norm(f_ref, axis=-1)
    big = mag > floor * mag.max()
    err = np.linalg.norm(f_eng - f_ref, axis=-1)
    return (err[big] / mag[big]).max(), np.abs(err[~big]).max() if (~big).any() else 0.0


@pytest.mark.parametrize("name", CASES)
def test_first_step_f64(golden_dir, name):
    sc = _scene(golden_dir, name)
    eng = nbc.Engine([sc], precision="f64", use_graph=False)
    orc = oracle.OracleScene(sc)
    eng.step_export(1)
    eng.sync()
    orc.step(1)
    so, se = orc.sub(), eng.subspheres()
    assert np.array_equal(se["part_fix"], so["part_fix"])
    la, lb = eng.pairs()
    oa, ob = orc.pairs()
    assert np.array_equal(la, oa) and np.array_equal(lb, ob)
    anei_e, ng_e, ni_e = eng.rows()
    anei_o, ng_o, ni_o = orc.rows()
    assert np.array_equal(anei_e, anei_o)
    fe, ce = eng.chain()
    fo, co = orc.chain()
    assert _rel(fe, fo) < 1e-9
    assert np.abs(ce - co).max() < 1e-14
    parts = eng.force_parts()
    of = orc.sub_forces()
    scale = np.abs(of["fc"]).max() + np.abs(of["fw"]).max() + np.abs(of["fi"]).max()
    for k in ("fc", "fw", "fi"):
        assert np.abs(parts[k] - of[k]).max() <= 1e-10 * scale, k
    ce_, co_ = eng.clumps(), orc.clumps()
    for k in ("pos", "vel", "angvel", "quat"):
        assert _rel(ce_[k], co_[k]) < 1e-12, k
    if sc["params"]["isIntruder"]:
        ie, io = eng.intruder(), orc.intruder()
        assert np.abs(ie["reaction"] - io["reaction"]).max() <= 1e-10 * max(1e-3, np.abs(io["reaction"]).max())
        assert np.abs(ie["pos"] - io["pos"]).max() < 1e-15


@pytest.mark.parametrize("name", CASES)
def test_24_steps_f64_against_reference(golden_dir, name):
    """Engine (FP64) directly against the reference build's outputs at every
    step: sort order and lists bit-exact, states to rounding."""
    sc = _scene(golden_dir, name)
    g = np.load(os.path.join(golden_dir, f"{name}.ref.npz"))
    eng = nbc.Engine([sc], precision="f64", use_graph=True)
    off = 1 if sc["params"]["isIntruder"] else 0
    for s in range(1, int(g["steps"]) + 1):
        if f"c{s}/fcn" in g:
            eng.step_export(1)
        else:
            eng.step(1)
        eng.sync()
        se, ce = eng.subspheres(), eng.clumps()
        assert np.array_equal(se["part_fix"], g[f"s{s}/part_fix"]), f"step {s}"
        assert _rel(ce["pos"], g[f"s{s}/clump_pos"][off:]) < 1e-11
        assert _rel(ce["vel"], g[f"s{s}/clump_vel"][off:]) < 1e-8
        assert _rel(ce["angvel"], g[f"s{s}/clump_angvel"][off:]) < 1e-8
        if f"c{s}/rows" in g:
            anei, _, _ = eng.rows()
            rows, slots = np.nonzero(anei >= 0)
            assert np.array_equal(rows, g[f"c{s}/rows"]) and np.array_equal(slots, g[f"c{s}/slots"])
            assert np.array_equal(anei[rows, slots], g[f"c{s}/nei"])
            if f"c{s}/fcn" in g:
                f, cp = eng.chain()
                ref = g[f"c{s}/fcn"]
                assert np.abs(f[rows, slots] - ref).max() <= 1e-8 * np.abs(ref).max()
        if off:
            ie = eng.intruder()
            ref_f = g[f"s{s}/intr_force"][0]
            assert np.abs(ie["reaction"] - ref_f).max() <= 1e-8 * max(1e-3, np.abs(ref_f).max())
    st = eng.stats()
    assert st["err"] == 0
    if name != "ref_fixture":
        assert st["rebuilds"] >= 5


@pytest.mark.parametrize("name", CASES)
def test_mixed_precision_per_contact_1e5(golden_dir, name):
    sc = _scene(golden_dir, name)
    eng = nbc.Engine([sc], precision="mixed", use_graph=False)
    orc = oracle.OracleScene(sc)
    eng.step_export(1)
    orc.step(1)
    anei_e, _, _ = eng.rows()
    anei_o, _, _ = orc.rows()
    assert np.array_equal(anei_e, anei_o)
    fe, _ = eng.chain()
    fo, _ = orc.chain()
    rel, small = _contact_rel_err(fe.reshape(-1, 3), fo.reshape(-1, 3))
    assert rel <= 1e-5, f"per-contact normal force error {rel:.2e}"
    parts = eng.force_parts()
    of = orc.sub_forces()
    # per-subsphere totals: error relative to the largest contact force on it
    scale = np.abs(fo).max()
    for k in ("fc", "fw", "fi"):
        assert np.abs(parts[k] - of[k]).max() <= 1e-5 * scale, k


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_graph_equals_eager_bitwise(golden_dir, precision):
    sc = _scene(golden_dir, "tetra_cube_cyl")
    a = nbc.Engine([sc], precision=precision, use_graph=False)
    b = nbc.Engine([sc], precision=precision, use_graph=True)
    a.step(24)
    b.step(24)
    a.sync()
    b.sync()
    ca, cb = a.clumps(), b.clumps()
    for k in ("pos", "vel", "angvel", "quat", "force", "torque"):
        assert np.array_equal(ca[k], cb[k]), k
    assert a.stats()["rebuilds"] == b.stats()["rebuilds"] >= 5


def test_runs_are_deterministic(golden_dir):
    sc = _scene(golden_dir, "spheres_cube_sphere")
    out = []
    for _ in range(2):
        e = nbc.Engine([sc], precision="mixed")
        e.step(24)
        e.sync()
        out.append((e.clumps(), e.intruder()))
    for k in ("pos", "vel", "angvel", "quat"):
        assert np.array_equal(out[0][0][k], out[1][0][k])
    assert np.array_equal(out[0][1]["reaction"], out[1][1]["reaction"])


def test_step_split_equals_single_call(golden_dir):
    """nbc_step(12) twice with a sync between equals nbc_step(24)."""
    sc = _scene(golden_dir, "tetra_gravity")
    a = nbc.Engine([sc], precision="f64")
    b = nbc.Engine([sc], precision="f64")
    a.step(24)
    a.sync()
    b.step(12)
    b.sync()
    b.step(12)
    b.sync()
    for k in ("pos", "vel", "angvel", "quat"):
        assert np.array_equal(a.clumps()[k], b.clumps()[k]), k


def test_dropin_open_run_writes_reference_files(golden_dir):
    """nbc_open/nbc_run on a reference working directory: the OutPart,
    OutClump, OutForce and OutCnt files it writes match the reference's."""
    name = "spheres_cube_sphere"
    sc = _scene(golden_dir, name)
    g = np.load(os.path.join(golden_dir, f"{name}.ref.npz"))
    with tempfile.TemporaryDirectory() as d:
        sg.write_reference_inputs(sc, d)
        eng = nbc.Engine.open(d, precision="f64")
        eng.run()
        eng.close()
        for s in (1, 2, 12, 24):
            ph = refbin.read_ph(os.path.join(d, "OutPart", "ph.%08d.bin" % s))
            ch = refbin.read_ch(os.path.join(d, "OutClump", "ch.%08d.bin" % s))
            assert np.array_equal(ph["part_fix"], g[f"s{s}/part_fix"])
            assert np.array_equal(ph["sorted_id"], np.arange(len(ph["part_fix"])))
            assert _rel(ph["pos"], g[f"s{s}/pos"]) < 1e-12
            assert ch["id"][0] == -1 and len(ch["id"]) == sc["params"]["ClumpNum"] + 1
            assert _rel(ch["pos"], g[f"s{s}/clump_pos"]) < 1e-12
            fc = refbin.read_fc(os.path.join(d, "OutForce", "fc.%08d.bin" % s))
            assert np.abs(fc["force"] - g[f"s{s}/intr_force"]).max() <= 1e-8 * max(1e-3, np.abs(g[f"s{s}/intr_force"]).max())
            assert os.path.exists(os.path.join(d, "OutForce", "yi.%08d.bin" % s))
        for s in (2, 12, 24):
            nei = refbin.read_cnt(os.path.join(d, "OutCnt", "Nei.%08d.bin" % s), np.int32)
            rows, slots = np.nonzero(nei >= 0)
            assert np.array_equal(rows, g[f"c{s}/rows"]) and np.array_equal(nei[rows, slots], g[f"c{s}/nei"])
            fcn = refbin.read_cnt(os.path.join(d, "OutCnt", "Fcn.%08d.bin" % s), "3f8")
            ref = g[f"c{s}/fcn"]
            assert np.abs(fcn[rows, slots] - ref).max() <= 1e-8 * np.abs(ref).max()
        assert open(os.path.join(d, "OutClump", "PenetratorShape.bt")).read().startswith("sphere")


def test_cfg0_settling_statistics(golden_dir):
    """10,000 steps of 2,000 settling spheres against the reference's final
    state: the trajectories decorrelate (chaos), the bed must not."""
    sc = _scene(golden_dir, "cfg0_settle")
    g = np.load(os.path.join(golden_dir, "cfg0_settle.ref.npz"))
    eng = nbc.Engine([sc], precision="f64")
    eng.step(10000)
    eng.sync()
    z = eng.clumps()["pos"][:, 2]
    zr = g["s10000/clump_pos"][:, 2]
    r = sc["sub"]["radius"][0]
    assert abs(np.mean(z) - np.mean(zr)) < 0.05 * r
    assert abs(np.max(z) - np.max(zr)) < 0.5 * r
    assert np.abs(np.sort(z) - np.sort(zr)).max() < 0.5 * r
    assert eng.stats()["err"] == 0


@pytest.mark.parametrize("precision,tol", [("f64", 1e-9), ("mixed", 1e-5)])
def test_hierarchical_grid_matches_oracle(precision, tol):
    """Polydisperse clumps (radius ratio 5) on the level table chosen by
    nbc_choose_levels: rows (same-level in discovery order, cross-level after
    them in ascending order of the finer partner) bit-exact with the oracle's
    hierarchical search, per-contact forces within tol."""
    sc = nbc.with_levels(sg.make_test_poly(n_clumps=150, seed=5))
    assert sc["levels"] is not None and len(sc["levels"]["cell"]) >= 2
    eng = nbc.Engine([sc], precision=precision, use_graph=True)
    orc = oracle.OracleScene(sc)
    eng.step_export(1)
    orc.step(1)
    for k in range(2):
        ae, _, _ = eng.rows()
        ao, _, _ = orc.rows()
        assert np.array_equal(ae, ao), f"rows differ (check {k})"
        assert np.array_equal(eng.subspheres()["part_fix"], orc.sub()["part_fix"])
        fe, _ = eng.chain()
        fo, _ = orc.chain()
        rel, _ = _contact_rel_err(fe.reshape(-1, 3), fo.reshape(-1, 3))
        assert rel <= tol, rel
        if k == 0:
            eng.step(10)
            eng.step_export(1)
            orc.step(11)
    assert eng.stats()["rebuilds"] >= 3


def test_batch_results_equal_alone(golden_dir):
    """Scenes batched in one engine give bitwise the results they give alone
    (per-scene rebuild decisions, scene-uniform blocks, no cross-scene sums)."""
    a = _scene(golden_dir, "spheres_cube_sphere")
    b = _scene(golden_dir, "tetra_cube_cyl")
    c = nbc.with_levels(sg.make_test_poly(n_clumps=60, seed=9))
    both = nbc.Engine([a, b, c], precision="mixed")
    alone = [nbc.Engine([x], precision="mixed") for x in (a, b, c)]
    both.step(24)
    both.sync()
    for e in alone:
        e.step(24)
        e.sync()
    for s, e in enumerate(alone):
        cb, ca = both.clumps(s), e.clumps(0)
        for k in ("pos", "vel", "angvel", "quat"):
            assert np.array_equal(cb[k], ca[k]), (s, k)
        assert both.stats(s)["rebuilds"] == e.stats(0)["rebuilds"]
        ib, ia = both.intruder(s), e.intruder(0)
        assert np.array_equal(ib["reaction"], ia["reaction"])


def test_pair_capacity_overflow_recovers_identically(golden_dir):
    """Pair buffers sized exactly to the first list (slack 1.0): a later,
    longer list overflows inside a graph launch, the kernels stand still, the
    host grows the buffers and replays that step's rebuild.  The result equals
    a run that never overflowed."""
    sc = _scene(golden_dir, "tetra_gravity")      # its list grows from 2963 to 2966 pairs
    tight = nbc.Engine([sc], precision="mixed", use_graph=True, pair_slack=1.0)
    roomy = nbc.Engine([sc], precision="mixed", use_graph=True, pair_slack=3.0)
    tight.step(1)
    bytes_first = tight.info()["device_bytes"]
    tight.step(23)
    assert tight.info()["device_bytes"] > bytes_first, "the capacity overflow path was not taken"
    roomy.step(24)
    tight.sync()
    roomy.sync()
    for k in ("pos", "vel", "angvel", "quat"):
        assert np.array_equal(tight.clumps()[k], roomy.clumps()[k]), k
    st = tight.stats()
    assert st["err"] == 0 and st["steps"] == 24


def test_list_growth_inside_graph_keeps_history():
    """Clumps converging from a loose lattice: the list grows from 3,099 to
    ~17,000 pairs after the step graph was captured with buffers sized for
    the first list (slack 1.0), so the pair buffers grow several times while
    graph launches run.  Every kernel of the captured rebuild must cover the
    grown list: the graph run equals the eager run bitwise and matches the
    FP64 oracle's pair list and states."""
    sc = sg.make_test_converging(steps=1500)
    graph = nbc.Engine([sc], precision="f64", use_graph=True, pair_slack=1.0)
    eager = nbc.Engine([sc], precision="f64", use_graph=False, pair_slack=1.0)
    graph.step(1)
    bytes_first = graph.info()["device_bytes"]
    graph.step(1499)
    eager.step(1500)
    assert graph.info()["device_bytes"] > bytes_first, "the pair buffers never grew"
    st = graph.stats()
    assert st["err"] == 0 and st["npairs"] > 4 * 3099, st
    graph.sync()
    eager.sync()
    for k in ("pos", "vel", "angvel", "quat"):
        assert np.array_equal(graph.clumps()[k], eager.clumps()[k]), k
    o = oracle.OracleScene(sc, threads=4)
    o.step(1500)
    lp_e, lpb_e = graph.pairs()
    lp_o, lpb_o = o.pairs()
    assert np.array_equal(lp_e, lp_o) and np.array_equal(lpb_e, lpb_o), "pair list differs from the oracle"
    ce, co = graph.clumps(), o.clumps()
    for k in ("pos", "quat"):
        assert _rel(ce[k], co[k]) < 1e-9, (k, _rel(ce[k], co[k]))
    for k in ("vel", "angvel"):
        assert _rel(ce[k], co[k]) < 1e-6, (k, _rel(ce[k], co[k]))


def test_restart_scene_carries_the_state(golden_dir):
    """Engine.restart_scene: a new engine created from another engine's
    state starts with that state (subsphere positions, clump poses and
    velocities, intruder) and steps from it."""
    sc = _scene(golden_dir, "tetra_gravity")
    a = nbc.Engine([sc], precision="f64", use_graph=True)
    a.step(12)
    sc2 = a.restart_scene(sc)
    b = nbc.Engine([sc2], precision="f64", use_graph=True)
    ca, cb = a.clumps(), b.clumps()
    for k in ("pos", "vel", "angvel", "quat"):
        assert np.array_equal(ca[k], cb[k]), k
    sa, sb = a.subspheres(), b.subspheres()
    pa = np.empty_like(sa["pos"]); pa[sa["part_fix"]] = sa["pos"]
    pb = np.empty_like(sb["pos"]); pb[sb["part_fix"]] = sb["pos"]
    assert np.array_equal(pa, pb)
    if sc.get("intruder") is not None:
        assert np.array_equal(a.intruder()["pos"], b.intruder()["pos"])
    b.step(5)
    b.sync()
    assert b.stats()["err"] == 0 and b.stats()["steps"] == 5

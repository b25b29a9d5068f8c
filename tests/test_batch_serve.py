"""Batches of independent scenes and the request server (continuous
batching): every scene's result in a batch or in the server's mix equals the
same scene run alone, bitwise (a batch is one engine over its scenes, each
with its own rebuild schedule and pair region; the requests admitted together
share one engine, each standing still at its own step count), and admission
respects the slot limit and the device-memory budget."""
import os

import numpy as np
import pytest

import nbc
import scenegen as sg

pytestmark = pytest.mark.gpu


def _scenes():
    return [sg.make_test_tetra(n_clumps=60, seed=11, intruder=None),
            sg.make_test_tetra(n_clumps=140, seed=12, intruder="sphere"),
            sg.make_test_spheres(n=300, seed=13, intruder="cylinder")]


def test_batch_equals_alone():
    scenes = _scenes()
    b = nbc.Batch(scenes, precision="mixed")
    b.step(150)          # several chunks of 64 steps, uneven tail
    b.step(17)
    for sc, e in zip(scenes, b.engines):
        a = nbc.Engine([sc], precision="mixed")
        a.step(167)
        a.sync()
        e.sync()
        ca, cb = a.clumps(), e.clumps()
        for k in ("pos", "vel", "angvel", "quat"):
            assert np.array_equal(ca[k], cb[k]), k
        assert a.stats()["rebuilds"] == e.stats()["rebuilds"]
        assert e.stats()["steps"] == 167
        a.close()
    b.close()


def test_scene_step_limits_equal_alone():
    """Scenes of one engine with their own step limits: each stands still at
    its limit (inside graph launches) while the others go on, with the state
    and intruder record of the scene run alone for that many steps."""
    scenes = _scenes()
    stops = [40, 95, 0]
    b = nbc.Batch(scenes, precision="mixed")
    for v, n in zip(b.engines, stops):
        if n:
            v.set_steps(n)
    b.step(70)
    b.step(60)
    b.sync()
    with pytest.raises(nbc.NbcError):
        b.engines[0].set_steps(100)   # 130 steps have started
    for sc, v, n in zip(scenes, b.engines, stops):
        n = n or 130
        a = nbc.Engine([sc], precision="mixed")
        a.step(n)
        a.sync()
        ca, cb = a.clumps(), v.clumps()
        for k in ("pos", "vel", "angvel", "quat"):
            assert np.array_equal(ca[k], cb[k]), (n, k)
        assert v.stats()["steps"] == n and a.stats()["rebuilds"] == v.stats()["rebuilds"]
        if sc.get("intruder") is not None:
            ia, ib = a.intruder(), v.intruder()
            assert np.array_equal(ia["pos"], ib["pos"]) and np.array_equal(ia["reaction"], ib["reaction"])
            assert np.array_equal(a.intruder_history(count=n), v.intruder_history(count=n))
        a.close()
    b.close()


def _requests():
    out = []
    for i, (n, r_i, v, mu) in enumerate([(1500, 4e-3, 0.3, 0.3), (4000, 6e-3, 0.5, 0.6),
                                          (2500, 5e-3, 0.2, 0.45), (800, 3e-3, 0.4, 0.7)]):
        bed = sg.make_poly_bed(n, 100 + i, 0.02, rmin=0.5e-3, rmax=1.5e-3)
        out.append(sg.with_sphere_intruder(bed, r_i, v, mu=mu))
    return out


def _alone_curve(scene, nsteps, every):
    e = nbc.Engine([scene], precision="mixed", pair_slack=1.6)
    e.step(nsteps)
    e.sync()
    h = e.intruder_history(count=nsteps)
    steps = np.arange(1, nsteps + 1)
    keep = (steps % every == 0) | (steps == nsteps)
    pos = e.intruder()["pos"].copy()
    e.close()
    return h[keep], pos


def test_server_results_equal_alone_and_respect_slots():
    reqs = _requests()
    nsteps, every = [300, 410, 250, 333], 50
    srv = nbc.Server(budget_bytes=64e9, max_active=2, cohort=2, precision="mixed")
    ids = [srv.submit(sc, n, every) for sc, n in zip(reqs, nsteps)]
    seen_running, results = 0, {}
    for _ in range(1000):
        st = srv.advance(chunk=37)
        seen_running = max(seen_running, st["running"])
        assert st["running"] <= 2
        # results are taken and released as soon as they are ready, while
        # requests admitted with them may still run
        for rid in ids:
            if rid not in results and srv.state(rid)[0] == 2:
                results[rid] = srv.result(rid)
                srv.release(rid)
        if len(results) == len(ids):
            break
    assert seen_running == 2
    for rid, sc, n in zip(ids, reqs, nsteps):
        res = results[rid]
        assert res is not None and res["steps"] == n
        curve, pos = _alone_curve(sc, n, every)
        assert np.array_equal(res["curve"], curve), rid
        assert np.array_equal(res["intr_pos"], pos), rid
    assert srv.memory()[0] == 0.0
    srv.close()


def test_server_admits_by_memory_budget():
    reqs = _requests()[:3]
    srv = nbc.Server(budget_bytes=1.0, max_active=8, precision="mixed")   # room for one request at a time
    ids = [srv.submit(sc, 40, 10) for sc in reqs]
    st = srv.advance(chunk=10)
    assert st["running"] == 1 and st["queued"] == 2
    for _ in range(100):
        st = srv.advance(chunk=10)
        assert st["running"] <= 1
        if st["finished"] == 3:
            break
    assert all(srv.state(i)[0] == 2 for i in ids)
    srv.close()


def test_server_retires_a_bad_request_and_serves_the_others():
    """A request whose scene fails the engine's input checks (here a radius
    of zero) is retired with its error at admission; the requests around it
    run and give the results they give alone."""
    reqs = _requests()[:3]
    bad = dict(reqs[1])
    bad["sub"] = {k: np.array(v, copy=True) for k, v in reqs[1]["sub"].items()}
    bad["sub"]["radius"][0] = 0.0
    srv = nbc.Server(budget_bytes=64e9, max_active=3, precision="mixed")
    ids = [srv.submit(sc, 60, 20) for sc in (reqs[0], bad, reqs[2])]
    for _ in range(100):
        st = srv.advance(chunk=30)
        if st["finished"] == 3:
            break
    assert srv.state(ids[1])[0] == 3
    with pytest.raises(nbc.NbcError, match="radius or mass not positive"):
        srv.result(ids[1])
    for rid, sc in ((ids[0], reqs[0]), (ids[2], reqs[2])):
        res = srv.result(rid)
        curve, pos = _alone_curve(sc, 60, 20)
        assert np.array_equal(res["curve"], curve) and np.array_equal(res["intr_pos"], pos)
    srv.close()

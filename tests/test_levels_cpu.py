"""The hierarchical-grid level chooser (nbc_choose_levels) and the oracle's
hierarchical broad phase (CPU only)."""
import numpy as np

import nbc
import oracle
import scenegen as sg


def test_monodisperse_keeps_one_level():
    lv, cell = nbc.choose_levels(np.full(1000, 1e-3))
    assert len(cell) == 1 and np.all(lv == 0) and abs(cell[0] - 3e-3) < 1e-15


def test_levels_are_nested_bands():
    rng = np.random.default_rng(0)
    r = np.exp(rng.uniform(np.log(0.5e-3), np.log(5e-3), 20000))
    lv, cell = nbc.choose_levels(r, 4)
    assert len(cell) >= 2
    assert np.all(np.diff(cell) < 0), "level 0 is the coarsest"
    for l in range(len(cell)):
        assert np.all(3.0 * r[lv == l] <= cell[l] + 1e-15)
    # a larger radius never sits on a finer level than a smaller one
    order = np.argsort(r)
    assert np.all(np.diff(lv[order]) <= 0)


def test_oracle_hgrid_pairs_equal_single_level_set():
    """The hierarchical search finds exactly the pairs of the single-level
    search (same cutoff); only ownership and order differ."""
    sc = sg.make_test_poly(n_clumps=120, seed=5)
    one = oracle.OracleScene(sc)
    one.step(1)
    multi = oracle.OracleScene(nbc.with_levels(sc))
    assert sc["sub"]["radius"].max() / sc["sub"]["radius"].min() > 3
    multi.step(1)
    fa, fb = one.sub()["part_fix"], multi.sub()["part_fix"]
    pa = {tuple(sorted((fa[a], fa[b]))) for a, b in zip(*one.pairs())}
    pb = {tuple(sorted((fb[a], fb[b]))) for a, b in zip(*multi.pairs())}
    assert pa == pb and len(pa) > 100
    # same physics: clump states after the step agree to rounding
    ca, cb = one.clumps(), multi.clumps()
    assert np.abs(ca["vel"] - cb["vel"]).max() <= 1e-9 * np.abs(ca["vel"]).max()


def test_owner_rows_are_two_ascending_runs():
    """The order the back references rely on (binary search in k_backref):
    an owner row lists its same-level partners first, in ascending index
    order (the stencil's cells are visited in ascending cell order and the
    subspheres are sorted by cell), then its cross-level partners in
    ascending order.  Checked on the oracle's lists, which follow the
    reference's order, after several rebuilds."""
    sc = nbc.with_levels(sg.make_test_poly(n_clumps=120, seed=5))
    assert sc["levels"] is not None and len(sc["levels"]["cell"]) > 1
    o = oracle.OracleScene(sc)
    o.step(40)
    assert o.rebuilds >= 2
    lv = np.asarray(sc["levels"]["level"])[o.sub()["part_fix"]]
    anei, ng, _ = o.rows()
    runs = 0
    for i in range(len(ng)):
        row = anei[i, :ng[i]]
        same = lv[row] == lv[i]
        k = int(np.argmin(same)) if not same.all() else len(row)
        assert same[:k].all() and not same[k:].any(), i      # same-level entries form a prefix
        assert np.all(np.diff(row[:k]) > 0) and np.all(np.diff(row[k:]) > 0), i
        runs += k < len(row)
    assert runs > 10

"""nbc_cell_sort_noalloc: the allocation-free cell sort, for callers that
cannot call cudaMalloc (device memory owned by another framework's pool, or a
memory budget fixed at start-up).  Checked through the C ABI against the
engine's own sort (nbc_step + nbc_get_subspheres) on the same positions, on
two calls in a row (the second call reuses the library's scratch array as
the first left it).  Integer outputs: bit-exact.

Collected last on purpose: it shares nothing with the other tests and runs
in a fresh process too.
"""
import math

import numpy as np
import pytest

import nbc
import scenegen as sg

pytestmark = pytest.mark.gpu


def engine_grid(scene):
    """The padded grid the engine hashes with (SetMeshSize,
    src/dem_subsphere_io.cu:195-230)."""
    p = scene["params"]
    c = 3.0 * float(scene["sub"]["radius"].max())
    g = nbc.GridDesc()
    g.cell = c
    for a, ax in enumerate("xyz"):
        g.origin[a] = p["WorldOrigin_" + ax] - c
        g.dims[a] = int(math.ceil((p["WorldSize_" + ax] + 2 * c) / c))
        g.box_lo[a] = p["BoxLowLmt_" + ax]
        g.box_hi[a] = p["BoxUpLmt_" + ax]
    return g


def test_noalloc_sort_matches_engine_sort_twice():
    import torch

    scene = sg.make_cfg1(n_clumps=5000, seed=7, steps=2)     # 20,000 subspheres, 10 radix tiles
    eng = nbc.Engine([scene], precision="f64", use_graph=False)
    eng.step(1)       # the first step builds the list: hash + sort of the posed positions
    eng.sync()
    sub = eng.subspheres()
    fix, pos_sorted = sub["part_fix"], sub["pos"]
    n = len(fix)
    pos = np.empty_like(pos_sorted)
    pos[fix] = pos_sorted                 # back to input order: the order the engine sorted from
    grid = engine_grid(scene)

    dpos = torch.from_numpy(pos).cuda()
    for call in range(2):
        perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        key = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        nbc.cell_sort_noalloc(dpos.data_ptr(), n, grid, perm.data_ptr(), key.data_ptr(), 0)
        torch.cuda.synchronize()
        p, k = perm.cpu().numpy(), key.cpu().numpy()
        assert np.array_equal(p, fix), f"call {call}: permutation differs from the engine's sort"
        assert np.all(np.diff(k) >= 0), f"call {call}: keys not ascending"
    eng.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    grid = nbc.GridDesc()
    grid.cell = 1.0
    for a in range(3):
        grid.dims[a] = 4
        grid.box_hi[a] = 4.0
    with pytest.raises(nbc.NbcError) as e:
        nbc.cell_sort_noalloc(1, nbc.NOALLOC_MAX_N + 1, grid, 1, 1, 0)
    assert e.value.code == -1 and "scratch array" in str(e.value)

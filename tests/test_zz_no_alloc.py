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


def numpy_cell_sort(pos, g):
    """The cell hash of GetParticleCellIndex_cuk (src/dem_grid.cu:155-202,
    the engine's padded grid: positions outside the box go to the last
    cell, cell coordinates clamped to the grid) and a stable sort by cell."""
    dims = np.array(g.dims[:], np.int64)
    cellnum = int(np.prod(dims))
    lo, hi = np.array(g.box_lo[:]), np.array(g.box_hi[:])
    out = np.any((pos >= hi) | (pos < lo), axis=1)
    c = np.floor((pos - np.array(g.origin[:])) / g.cell).astype(np.int64)
    c = np.clip(c, 0, dims - 1)
    key = np.clip(c[:, 2] * dims[1] * dims[0] + c[:, 1] * dims[0] + c[:, 0], 0, cellnum - 1)
    key[out] = cellnum - 1
    perm = np.argsort(key, kind="stable")
    return perm.astype(np.int32), key[perm].astype(np.int32)


@pytest.mark.parametrize("dims,n", [((6, 6, 6), 3001), ((20, 20, 91), 20000 + 777), ((50, 50, 40), 70001)])
def test_noalloc_sort_matches_numpy_for_one_two_three_passes(dims, n):
    """216 cells (one 8-bit radix pass: the hash lands in the library's
    scratch array and the pass in the caller's buffers), 36,400 cells (two
    passes) and 100,000 cells (three passes), n not a multiple of the radix
    tile, some positions outside the box and some on cell faces: permutation
    and keys bit-exact with a numpy hash and stable sort, on two calls in a
    row."""
    import torch

    rng = np.random.default_rng(n)
    g = nbc.GridDesc()
    g.cell = 1e-3
    for a in range(3):
        g.origin[a] = -g.cell
        g.dims[a] = dims[a]
        g.box_lo[a] = 0.0
        g.box_hi[a] = (dims[a] - 2) * g.cell
    span = np.array([(d - 2) * g.cell for d in dims])
    pos = rng.uniform(-0.05, 1.05, (n, 3)) * span           # about 15% outside the box
    pos[: n // 10] = np.round(pos[: n // 10] / g.cell) * g.cell   # some exactly on cell faces
    want_p, want_k = numpy_cell_sort(pos, g)
    bits = int(np.ceil(np.log2(np.prod(dims))))
    assert (bits + 7) // 8 == {216: 1, 36400: 2, 100000: 3}[int(np.prod(dims))]
    dpos = torch.from_numpy(pos).cuda()
    for call in range(2):
        perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        key = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        nbc.cell_sort_noalloc(dpos.data_ptr(), n, g, perm.data_ptr(), key.data_ptr(), 0)
        torch.cuda.synchronize()
        assert np.array_equal(perm.cpu().numpy(), want_p), f"call {call}: permutation"
        assert np.array_equal(key.cpu().numpy(), want_k), f"call {call}: keys"


def test_noalloc_rejects_sizes_beyond_its_scratch():
    grid = nbc.GridDesc()
    grid.cell = 1.0
    for a in range(3):
        grid.dims[a] = 4
        grid.box_hi[a] = 4.0
    with pytest.raises(nbc.NbcError) as e:
        nbc.cell_sort_noalloc(1, nbc.NOALLOC_MAX_N + 1, grid, 1, 1, 0)
    assert e.value.code == -1 and "scratch array" in str(e.value)

"""The drop-in boundary on CPU: the C ABI library, its input parsing and the
binary output layout (no GPU needed)."""
import ctypes as C
import os
import re
import tempfile

import numpy as np
import pytest

import nbc
import refbin
import scenegen as sg

from conftest import REPO, cuda_available

HEADER = os.path.join(REPO, "include", "nbc.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(nbc_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = nbc.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(nbc.EXPORTED)


def test_scene_desc_layout_matches_header():
    # every field of nbc_scene_desc, in order, is mirrored by the ctypes struct
    src = open(HEADER).read()
    body = src[src.index("typedef struct {\n    int n_sub"):src.index("} nbc_scene_desc;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl or decl.startswith("typedef"):
            decl = decl.replace("typedef struct {", "").strip()
            if not decl:
                continue
        decl = re.sub(r"^(const\s+)?\w+\s*\*?\s*", "", decl)
        for name in decl.split(","):
            fields.append(re.sub(r"\[.*\]", "", name).replace("*", "").strip())
    assert fields == [f for f, _ in nbc.SceneDesc._fields_]


def test_create_rejects_bad_arguments():
    L = nbc.lib()
    h = C.c_void_p()
    assert L.nbc_create(None, 0, None, C.byref(h)) == -1
    assert b"no scenes" in L.nbc_last_error()
    assert L.nbc_step(None, 1) == -1


def _copy_scene(sc):
    out = dict(sc)
    for k in ("sub", "clump"):
        out[k] = {kk: np.array(vv, copy=True) for kk, vv in sc[k].items()}
    return out


@pytest.mark.parametrize("where,index,value,needle", [
    ("sub.pos", (0, 0), float("nan"), "non-finite position"),
    ("sub.radius", 1, 0.0, "radius or mass not positive"),
    ("sub.mass", 2, -1.0, "radius or mass not positive"),
    ("clump.prop", (2, 3), -1.0, "clump inertia or mass not positive"),
    ("clump.vel", (3, 1), float("inf"), "non-finite or zero clump state"),
])
def test_create_rejects_invalid_values_before_the_device(where, index, value, needle):
    """A scene's values are checked on the host before any device call, so
    a bad scene is an argument error (on a machine without a GPU too) and
    never reaches a kernel."""
    sc = _copy_scene(sg.make_test_spheres(n=64, seed=3))
    part, key = where.split(".")
    sc[part][key][index] = value
    d, keep = nbc.scene_desc(sc)
    arr = (C.POINTER(nbc.SceneDesc) * 1)(C.pointer(d))
    h = C.c_void_p()
    rc = nbc.lib().nbc_create(arr, 1, None, C.byref(h))
    assert nbc.STATUS[rc] == "ERR_ARG"
    assert needle in nbc.lib().nbc_last_error().decode()


def _workdir(scene, d):
    sg.write_reference_inputs(scene, d)
    return d


def _open_status(d):
    h = C.c_void_p()
    rc = nbc.lib().nbc_open(d.encode(), None, C.byref(h))
    if rc == 0:
        nbc.lib().nbc_destroy(h)
    return rc, nbc.lib().nbc_last_error().decode()


def test_open_parses_reference_inputs():
    sc = sg.make_test_spheres(n=64, seed=3)
    with tempfile.TemporaryDirectory() as d:
        _workdir(sc, d)
        rc, msg = _open_status(d)
        # inputs parsed; the engine then needs a CUDA device (no CPU fallback)
        assert rc == (0 if cuda_available() else -5), msg


@pytest.mark.parametrize("mutate,needle", [
    (lambda t: t.replace("Ymod =", "Ymodd ="), "Unrecoganized item Ymodd"),
    (lambda t: "\n".join(l for l in t.splitlines() if not l.startswith("Beta")), "missing"),
])
def test_open_rejects_bad_world_par(mutate, needle):
    sc = sg.make_test_spheres(n=64, seed=3)
    with tempfile.TemporaryDirectory() as d:
        _workdir(sc, d)
        p = os.path.join(d, "world.par")
        text = open(p).read()
        open(p, "w").write(mutate(text))
        rc, msg = _open_status(d)
        assert rc == -3 and needle in msg, msg


def test_open_rejects_short_ph_and_bad_penetrator():
    sc = sg.make_test_spheres(n=64, seed=3)
    with tempfile.TemporaryDirectory() as d:
        _workdir(sc, d)
        p = os.path.join(d, "ph.00000000.bt")
        lines = open(p).read().splitlines()
        with open(p, "w") as f:
            f.write("\n".join(lines[:-5]) + "\n")
        rc, msg = _open_status(d)
        assert rc == -3 and "short or malformed" in msg
    with tempfile.TemporaryDirectory() as d:
        _workdir(sc, d)
        p = os.path.join(d, "Rocks", "Penetrator.bt")
        text = open(p).read()
        open(p, "w").write(text.replace("sphere", "cone"))
        rc, msg = _open_status(d)
        assert rc == -3 and "Unknown penetrator shape" in msg
    with tempfile.TemporaryDirectory() as d:
        _workdir(sc, d)
        p = os.path.join(d, "Rocks", "Penetrator.bt")
        text = open(p).read()
        open(p, "w").write(text.replace("gravity_after_contact", "warp").replace("constant_velocity", "warp"))
        rc, msg = _open_status(d)
        assert rc == -3 and "motion mode" in msg


def test_reference_fixture_reads_back(golden_dir):
    # scenegen's reader of the reference's text files against the stored npz
    sc = sg.scene_from_npz(os.path.join(golden_dir, "ref_fixture.scene.npz"))
    with tempfile.TemporaryDirectory() as d:
        sg.write_reference_inputs(sc, d)
        back = sg.read_reference_inputs(d)
        for k in ("pos", "local", "mass", "radius"):
            assert np.array_equal(back["sub"][k], sc["sub"][k])
        assert np.array_equal(back["sub"]["clump_id"], sc["sub"]["clump_id"])
        for k in ("pos", "vel", "quat", "angvel", "prop"):
            assert np.array_equal(back["clump"][k], sc["clump"][k])
        assert back["intruder"]["motion"] == sc["intruder"]["motion"]


def test_binary_layout_round_trip():
    rng = np.random.default_rng(0)
    n, k = 17, 5
    with tempfile.TemporaryDirectory() as d:
        p = refbin.file_name(d, "ph", 1000)
        assert p.endswith("ph.00001000.bin")
        arrs = dict(sorted_id=np.arange(n), part_fix=rng.permutation(n), clump_id=rng.integers(0, k, n),
                    pos=rng.random((n, 3)), local=rng.random((n, 3)), mass=rng.random(n), radius=rng.random(n))
        refbin.write_ph(p, **arrs)
        assert os.path.getsize(p) == 4 + 3 * 4 * n + 2 * 24 * n + 2 * 8 * n
        back = refbin.read_ph(p)
        for key, v in arrs.items():
            assert np.array_equal(back[key], v)
        q = refbin.file_name(d, "ch", 1)
        intr = {"pos": rng.random(3), "vel": rng.random(3), "quat": rng.random(4), "angvel": rng.random(3)}
        c = {x: rng.random((k, 3)) for x in ("pos", "vel", "angvel")}
        c["quat"], c["prop"] = rng.random((k, 4)), rng.random((k, 4))
        refbin.write_ch(q, c["pos"], c["vel"], c["quat"], c["angvel"], c["prop"], intruder=intr)
        back = refbin.read_ch(q)
        assert back["id"][0] == -1 and np.array_equal(back["id"][1:], np.arange(k))
        assert np.array_equal(back["pos"][0], intr["pos"]) and np.array_equal(back["pos"][1:], c["pos"])
        assert np.array_equal(back["prop"][0], np.zeros(4))


def test_generators_are_seeded_and_consistent():
    a = sg.make_test_tetra(n_clumps=30, seed=5)
    b = sg.make_test_tetra(n_clumps=30, seed=5)
    assert np.array_equal(a["sub"]["pos"], b["sub"]["pos"])
    # subsphere positions are the clump pose applied to the body offsets
    R = sg.quat_to_body2world(a["clump"]["quat"])
    cid = a["sub"]["clump_id"]
    pos = a["clump"]["pos"][cid] + np.einsum("nij,nj->ni", R[cid], a["sub"]["local"])
    assert np.abs(pos - a["sub"]["pos"]).max() < 1e-15
    # principal-frame template: tetrahedron inertia is isotropic
    I = a["clump"]["prop"][0, :3]
    assert np.ptp(I) / I.mean() < 0.02
    c1 = sg.make_cfg1(n_clumps=2000, seed=1, steps=10)
    assert c1["params"]["NumberBody"] == 8000 and c1["cylinder"] is not None
    r = c1["sub"]["radius"]
    xy = np.linalg.norm(c1["sub"]["pos"][:, :2], axis=1)
    assert (xy + r).max() < c1["cylinder"]["radius"]

"""ctypes binding of libnbc.so (include/nbc.h) for Python callers.

Mirrors the engine's C ABI one call per method; the engine itself is C++ and
sm_100a CUDA.  There is no fallback: if libnbc.so is missing or no CUDA device
is present, Engine() raises.

    import nbc, scenegen
    eng = nbc.Engine([scenegen.make_cfg0()], precision="f64")
    eng.step(100); eng.sync()
    state = eng.clumps(0)
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnbc.so")

NBC_OK = 0
STATUS = {-1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_IO", -4: "ERR_NONFINITE", -5: "ERR_NO_DEVICE",
          -6: "ERR_MEMORY", -7: "ERR_STATE"}
PREC = {"f64": 0, "mixed": 1}
WALL = {None: 0, "cube": 1, "cylinder": 2}
# DEMmain drivers of nbc_open_sphere (NBC_DRIVER_*) and the NBC_SPHERE_* bits
SPHERE_DRIVERS = {"cylinder": 0, "cube": 1, "split": 2, "hgrid": 3}
SPHERE_KINEMATICS, SPHERE_CUBE_WALL, SPHERE_RESET_HISTORY = 1, 2, 4
MOTION = {"constant_velocity": 0, "gravity": 1, "gravity_after_contact": 2}

D3 = C.c_double * 3
D4 = C.c_double * 4
P_D = C.POINTER(C.c_double)
P_I = C.POINTER(C.c_int)


class SceneDesc(C.Structure):
    _fields_ = [
        ("n_sub", C.c_int), ("n_clump", C.c_int), ("branch_len", C.c_int),
        ("start_step", C.c_int), ("end_step", C.c_int), ("output_interval", C.c_int),
        ("dt", C.c_double), ("ymod", C.c_double), ("prat", C.c_double), ("frcoe", C.c_double),
        ("normres", C.c_double), ("beta", C.c_double), ("cohesion", C.c_double),
        ("gravity", C.c_double), ("thresh", C.c_double),
        ("world_origin", D3), ("world_size", D3), ("box_lo", D3), ("box_hi", D3),
        ("is_wall_force", C.c_int),
        ("clump_id", P_I), ("pos", P_D), ("local", P_D), ("mass", P_D), ("radius", P_D),
        ("clump_pos", P_D), ("clump_vel", P_D), ("clump_quat", P_D), ("clump_angvel", P_D),
        ("clump_prop", P_D),
        ("wall", C.c_int),
        ("cube_half", D3), ("cube_centre", D3), ("cube_vel", D3), ("cube_angvel", D3),
        ("cyl_radius", C.c_double), ("cyl_half_height", C.c_double), ("cyl_axis", D3),
        ("cyl_centre", D3), ("cyl_vel", D3), ("cyl_angvel", D3),
        ("intruder", C.c_int), ("intr_motion", C.c_int),
        ("intr_radius", C.c_double), ("intr_half_height", C.c_double), ("intr_axis", D3),
        ("intr_prop", D4), ("intr_pos", D3), ("intr_vel", D3), ("intr_angvel", D3),
        ("levels", C.c_int), ("level", P_I), ("level_cell", P_D),
        ("sphere_mode", C.c_int), ("body_kind", P_I),
    ]


class GridDesc(C.Structure):
    _fields_ = [("origin", D3), ("cell", C.c_double), ("dims", C.c_int * 3), ("box_lo", D3), ("box_hi", D3)]


NOALLOC_MAX_N = 262144


def cell_sort_noalloc(pos_ptr: int, n: int, grid: GridDesc, perm_ptr: int, key_ptr: int, stream: int = 0):
    """nbc_cell_sort_noalloc on caller-owned device buffers (raw addresses)."""
    _check(lib().nbc_cell_sort_noalloc(C.c_void_p(pos_ptr), int(n), C.byref(grid), C.c_void_p(perm_ptr),
                                       C.c_void_p(key_ptr), C.c_void_p(stream)))


def choose_levels(radius, max_levels=6):
    """Hierarchical-grid levels for these radii: (level[n], level_cell[L])."""
    r = np.ascontiguousarray(radius, dtype=np.float64)
    lv = np.zeros(len(r), np.int32)
    cell = np.zeros(max(8, int(max_levels)))
    L = lib().nbc_choose_levels(_p(r), len(r), int(max_levels), _p(lv, P_I), _p(cell))
    return lv, cell[:L].copy()


def union_mass(centres, radii, clump_start, samples=1 << 18, device=0):
    """Union volume, centroid and second central moments of clump templates
    (nbc_union_mass): centres [M][3] and radii [M] of all members, clump k
    owning members clump_start[k] .. clump_start[k+1]-1.  Returns
    (volume[K], centroid[K][3], moments[K][3][3])."""
    c = np.ascontiguousarray(centres, dtype=np.float64).reshape(-1, 3)
    r = np.ascontiguousarray(radii, dtype=np.float64)
    st = np.ascontiguousarray(clump_start, dtype=np.int32)
    K = len(st) - 1
    out = np.zeros((max(K, 1), 10))
    _check(lib().nbc_union_mass(_p(c), _p(r), _p(st, P_I), K, int(samples), _p(out), int(device)))
    out = out[:K]
    m = np.empty((K, 3, 3))
    m[:, 0, 0], m[:, 1, 1], m[:, 2, 2] = out[:, 4], out[:, 5], out[:, 6]
    m[:, 0, 1] = m[:, 1, 0] = out[:, 7]
    m[:, 0, 2] = m[:, 2, 0] = out[:, 8]
    m[:, 1, 2] = m[:, 2, 1] = out[:, 9]
    return out[:, 0].copy(), out[:, 1:4].copy(), m


def with_levels(scene: dict, max_levels=6) -> dict:
    """The scene with a hierarchical grid chosen by nbc_choose_levels (or
    unchanged when one level is best)."""
    lv, cell = choose_levels(scene["sub"]["radius"], max_levels)
    out = dict(scene)
    out["levels"] = {"level": lv, "cell": cell} if len(cell) > 1 else None
    return out


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("lanes", C.c_int), ("use_graph", C.c_int),
                ("device", C.c_int), ("pair_slack", C.c_double), ("search_lanes", C.c_int),
                ("clump_batch", C.c_int), ("pair_blocks", C.c_int)]


EXPORTED = [
    "nbc_last_error", "nbc_default_options", "nbc_open", "nbc_open_sphere", "nbc_run", "nbc_create", "nbc_destroy",
    "nbc_step", "nbc_step_export", "nbc_sync", "nbc_num_scenes", "nbc_scene_stats", "nbc_contact_counts",
    "nbc_get_subspheres", "nbc_get_subsphere_body", "nbc_get_clumps", "nbc_get_sub_forces",
    "nbc_get_force_parts", "nbc_get_pairs", "nbc_get_rows", "nbc_get_chain", "nbc_get_pair_forces",
    "nbc_get_intruder",
    "nbc_get_intruder_diag", "nbc_get_intruder_history", "nbc_timing_enable", "nbc_timing_read",
    "nbc_timing_phases",
    "nbc_engine_info", "nbc_set_scene_steps", "nbc_cell_sort_noalloc", "nbc_choose_levels", "nbc_union_mass",
    "nbc_checkpoint_write", "nbc_checkpoint_read", "nbc_autotune", "nbc_launch_info",
    "nbc_batch_create", "nbc_batch_step", "nbc_batch_engine", "nbc_batch_destroy",
    "nbc_server_create", "nbc_server_submit", "nbc_server_advance", "nbc_server_result",
    "nbc_server_release", "nbc_server_memory", "nbc_server_destroy", "nbc_server_set_cohort",
]

_lib = None


class NbcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Load libnbc.so (building it first if this tree has not built it)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            import build as _b  # noqa: PLC0415  (the in-tree build script)
            _b.build()
        L = C.CDLL(LIB_PATH)
        L.nbc_last_error.restype = C.c_char_p
        L.nbc_default_options.argtypes = [C.POINTER(Options)]
        L.nbc_default_options.restype = None
        for f in EXPORTED:
            if f not in ("nbc_last_error", "nbc_default_options"):
                getattr(L, f).restype = C.c_int
        _lib = L
    return _lib


def _check(rc):
    if rc != NBC_OK:
        raise NbcError(rc, lib().nbc_last_error().decode(errors="replace"))


def _p(a, t=P_D):
    return a.ctypes.data_as(t) if a is not None else None


def _set(arr, vals):
    for i, v in enumerate(vals):
        arr[i] = float(v)


def scene_desc(scene: dict):
    """Build a SceneDesc (and the arrays it points to) from a scenegen scene."""
    p, s, c = scene["params"], scene["sub"], scene["clump"]
    keep = {
        "cid": np.ascontiguousarray(s["clump_id"], dtype=np.int32),
        "pos": np.ascontiguousarray(s["pos"], dtype=np.float64),
        "local": np.ascontiguousarray(s["local"], dtype=np.float64),
        "mass": np.ascontiguousarray(s["mass"], dtype=np.float64),
        "radius": np.ascontiguousarray(s["radius"], dtype=np.float64),
    }
    for k in ("pos", "vel", "quat", "angvel", "prop"):
        keep["c" + k] = np.ascontiguousarray(c[k], dtype=np.float64)
    d = SceneDesc()
    d.n_sub, d.n_clump = int(p["NumberBody"]), int(p["ClumpNum"])
    d.branch_len = int(p["BranchLmtLen"])
    d.start_step, d.end_step = int(p["StartStep"]), int(p["EndStep"])
    d.output_interval = int(p["OutputInterval"])
    d.dt, d.ymod, d.prat, d.frcoe = p["StepSize"], p["Ymod"], p["Prat"], p["Frcoe"]
    d.normres, d.beta, d.cohesion = p["NormRes"], p["Beta"], p["Cohesion"]
    d.gravity, d.thresh = p["Gravity"], p["Thresh"]
    _set(d.world_origin, [p["WorldOrigin_" + a] for a in "xyz"])
    _set(d.world_size, [p["WorldSize_" + a] for a in "xyz"])
    _set(d.box_lo, [p["BoxLowLmt_" + a] for a in "xyz"])
    _set(d.box_hi, [p["BoxUpLmt_" + a] for a in "xyz"])
    d.is_wall_force = int(p["isWallForce"])
    d.clump_id = _p(keep["cid"], P_I)
    d.pos, d.local, d.mass, d.radius = _p(keep["pos"]), _p(keep["local"]), _p(keep["mass"]), _p(keep["radius"])
    d.clump_pos, d.clump_vel, d.clump_quat = _p(keep["cpos"]), _p(keep["cvel"]), _p(keep["cquat"])
    d.clump_angvel, d.clump_prop = _p(keep["cangvel"]), _p(keep["cprop"])
    cube, cyl = scene.get("cube"), scene.get("cylinder")
    if cube is not None:
        d.wall = 1
        _set(d.cube_half, cube["half"]); _set(d.cube_centre, cube["centre"])
        _set(d.cube_vel, cube["vel"]); _set(d.cube_angvel, cube["angvel"])
    elif cyl is not None:
        d.wall = 2
        d.cyl_radius, d.cyl_half_height = cyl["radius"], cyl["half_height"]
        _set(d.cyl_axis, cyl["axis"]); _set(d.cyl_centre, cyl["centre"])
        _set(d.cyl_vel, cyl["vel"]); _set(d.cyl_angvel, cyl["angvel"])
    it = scene.get("intruder")
    d.intruder = -1
    if it is not None and int(p["isIntruder"]):
        d.intruder = 1 if it["shape"] == "sphere" else 0
        d.intr_motion = MOTION[it["motion"]]
        d.intr_radius, d.intr_half_height = it["radius"], it["half_height"]
        _set(d.intr_axis, it["axis"]); _set(d.intr_prop, it["prop"])
        _set(d.intr_pos, it["pos"]); _set(d.intr_vel, it["vel"]); _set(d.intr_angvel, it["angvel"])
    lv = scene.get("levels")
    d.levels = 1
    if lv is not None:
        keep["level"] = np.ascontiguousarray(lv["level"], dtype=np.int32)
        keep["level_cell"] = np.ascontiguousarray(lv["cell"], dtype=np.float64)
        d.levels = len(keep["level_cell"])
        d.level, d.level_cell = _p(keep["level"], P_I), _p(keep["level_cell"])
    # the sphere-only drivers' behaviour (NBC_SPHERE_* bits) and split-driver body kinds
    d.sphere_mode = int(scene.get("sphere_mode", 0))
    if scene.get("body_kind") is not None:
        keep["body_kind"] = np.ascontiguousarray(scene["body_kind"], dtype=np.int32)
        d.body_kind = _p(keep["body_kind"], P_I)
    return d, keep


class Engine:
    """A batch of scenes resident on one GPU."""

    def __init__(self, scenes, precision="mixed", use_graph=True, device=0, pair_slack=0.0,
                 search_lanes=0, clump_batch=0, pair_blocks=0, tuned=None):
        L = lib()
        self._descs = [scene_desc(s) for s in scenes]
        self.N = [int(s["params"]["NumberBody"]) for s in scenes]
        self.K = [int(s["params"]["ClumpNum"]) for s in scenes]
        self.BL = [int(s["params"]["BranchLmtLen"]) for s in scenes]
        arr = (C.POINTER(SceneDesc) * len(scenes))(*[C.pointer(d) for d, _ in self._descs])
        o = _options(precision, use_graph, device, pair_slack, search_lanes, clump_batch, pair_blocks, tuned)
        h = C.c_void_p()
        _check(L.nbc_create(arr, len(scenes), C.byref(o), C.byref(h)))
        self.h = h

    @classmethod
    def open(cls, workdir: str, precision="f64", use_graph=True):
        """The drop-in path: read a reference working directory."""
        self = cls.__new__(cls)
        L = lib()
        o = Options()
        L.nbc_default_options(C.byref(o))
        o.precision, o.use_graph = PREC[precision], int(use_graph)
        h = C.c_void_p()
        _check(L.nbc_open(workdir.encode(), C.byref(o), C.byref(h)))
        self.h = h
        self._descs = []
        return self

    @classmethod
    def open_sphere(cls, workdir: str, driver: str, precision="f64", use_graph=True):
        """The sphere-only drivers' drop-in path (DEMmain): driver is one of
        SPHERE_DRIVERS."""
        self = cls.__new__(cls)
        L = lib()
        o = Options()
        L.nbc_default_options(C.byref(o))
        o.precision, o.use_graph = PREC[precision], int(use_graph)
        h = C.c_void_p()
        _check(L.nbc_open_sphere(workdir.encode(), SPHERE_DRIVERS[driver], C.byref(o), C.byref(h)))
        self.h = h
        self._descs = []
        return self

    def run(self):
        _check(lib().nbc_run(self.h))

    @classmethod
    def borrowed(cls, handle, scenes):
        """A view of an engine owned by a Batch or a Server (not destroyed by close)."""
        self = cls.__new__(cls)
        self._descs = []
        self.N = [int(sc["params"]["NumberBody"]) for sc in scenes]
        self.K = [int(sc["params"]["ClumpNum"]) for sc in scenes]
        self.BL = [int(sc["params"]["BranchLmtLen"]) for sc in scenes]
        self.h = handle
        self._owner = False
        return self

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value and getattr(self, "_owner", True):
            lib().nbc_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1):
        _check(lib().nbc_step(self.h, int(n)))

    def step_export(self, n=1):
        _check(lib().nbc_step_export(self.h, int(n)))

    def sync(self):
        _check(lib().nbc_sync(self.h))

    def stats(self, s=0):
        v = [C.c_int() for _ in range(4)]
        _check(lib().nbc_scene_stats(self.h, s, *[C.byref(x) for x in v]))
        return {"steps": v[0].value, "rebuilds": v[1].value, "npairs": v[2].value, "err": v[3].value}

    def subspheres(self, s=0):
        n = self.N[s]
        fix, cid = np.zeros(n, np.int32), np.zeros(n, np.int32)
        pos, rad = np.zeros((n, 3)), np.zeros(n)
        _check(lib().nbc_get_subspheres(self.h, s, _p(fix, P_I), _p(cid, P_I), _p(pos), _p(rad)))
        return {"part_fix": fix, "clump_id": cid, "pos": pos, "radius": rad}

    def clumps(self, s=0):
        k = self.K[s]
        o = {x: np.zeros((k, 3)) for x in ("pos", "vel", "angvel", "force", "torque")}
        o["quat"] = np.zeros((k, 4))
        _check(lib().nbc_get_clumps(self.h, s, _p(o["pos"]), _p(o["vel"]), _p(o["quat"]),
                                    _p(o["angvel"]), _p(o["force"]), _p(o["torque"])))
        return o

    def contact_counts(self):
        """(near pairs of the current list, those that touched at the last step)."""
        a, b = C.c_longlong(), C.c_longlong()
        _check(lib().nbc_contact_counts(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def restart_scene(self, base, s=0):
        """A scene that starts from scene s's current state: subsphere
        positions, clump poses and velocities, intruder position and velocity
        (spring histories start from zero, as in a reference run restarted
        from its OutPart/OutClump snapshot)."""
        self.sync()
        sub, cl = self.subspheres(s), self.clumps(s)
        out = dict(base)
        out["sub"] = dict(base["sub"])
        out["clump"] = dict(base["clump"])
        pos = np.empty_like(sub["pos"])
        pos[sub["part_fix"]] = sub["pos"]
        out["sub"]["pos"] = pos
        for k in ("pos", "vel", "quat", "angvel"):
            out["clump"][k] = cl[k].copy()
        if base.get("intruder") is not None:
            it = self.intruder(s)
            out["intruder"] = dict(base["intruder"], pos=it["pos"].copy(), vel=it["vel"].copy())
        return out

    def sub_forces(self, s=0):
        n = self.N[s]
        f, t = np.zeros((n, 3)), np.zeros((n, 3))
        _check(lib().nbc_get_sub_forces(self.h, s, _p(f), _p(t)))
        return f, t

    def force_parts(self, s=0):
        n = self.N[s]
        parts = np.zeros((6, n, 3))
        _check(lib().nbc_get_force_parts(self.h, s, _p(parts)))
        return {k: parts[i] for i, k in enumerate(("fc", "tc", "fw", "tw", "fi", "ti"))}

    def pairs(self, s=0):
        n = C.c_int(0)
        _check(lib().nbc_get_pairs(self.h, s, C.byref(n), None, None))
        a, b = np.zeros(n.value, np.int32), np.zeros(n.value, np.int32)
        _check(lib().nbc_get_pairs(self.h, s, C.byref(n), _p(a, P_I), _p(b, P_I)))
        return a, b

    def rows(self, s=0, bl=None):
        bl = bl or self.BL[s]
        n = self.N[s]
        anei = np.zeros((n, bl), np.int32)
        ng, ni = np.zeros(n, np.int32), np.zeros(n, np.int32)
        _check(lib().nbc_get_rows(self.h, s, bl, _p(anei, P_I), _p(ng, P_I), _p(ni, P_I)))
        return anei, ng, ni

    def chain(self, s=0, bl=None):
        bl = bl or self.BL[s]
        n = self.N[s]
        f, c = np.zeros((n, bl, 3)), np.zeros((n, bl, 3))
        _check(lib().nbc_get_chain(self.h, s, bl, _p(f), _p(c)))
        return f, c

    def launch_info(self):
        """nbc_launch_info: the launch shapes in use and whether untimed steps
        run in a device-side loop."""
        v = [C.c_int() for _ in range(4)]
        _check(lib().nbc_launch_info(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("step_loop",) + TUNED_KEYS, [x.value for x in v]))

    def checkpoint(self, path):
        """nbc_checkpoint_write: the exact state after the last step."""
        _check(lib().nbc_checkpoint_write(self.h, os.fsencode(path)))

    def restore(self, path):
        """nbc_checkpoint_read into this engine (made from the same scenes and
        precision); stepping on continues the saved run bit for bit."""
        _check(lib().nbc_checkpoint_read(self.h, os.fsencode(path)))

    def pair_forces(self, s=0):
        """After step_export: the normal force on the owner of every listed
        pair, in list order (zero where the pair does not touch)."""
        n = C.c_int(0)
        _check(lib().nbc_get_pair_forces(self.h, s, C.byref(n), None))
        f = np.zeros((n.value, 3))
        _check(lib().nbc_get_pair_forces(self.h, s, C.byref(n), _p(f)))
        return f

    def intruder(self, s=0):
        o = {k: np.zeros(3) for k in ("pos", "vel", "reaction", "torque")}
        st = C.c_int()
        _check(lib().nbc_get_intruder(self.h, s, _p(o["pos"]), _p(o["vel"]), _p(o["reaction"]),
                                      _p(o["torque"]), C.byref(st)))
        o["state"] = st.value
        return o

    def intruder_diag(self, s=0):
        n = self.N[s]
        d = np.zeros((4, n, 3))
        _check(lib().nbc_get_intruder_diag(self.h, s, _p(d)))
        return d

    def intruder_history(self, s=0, count=1):
        out = np.zeros((count, 6))
        _check(lib().nbc_get_intruder_history(self.h, s, int(count), _p(out)))
        return out

    def timing_enable(self, on=True):
        _check(lib().nbc_timing_enable(self.h, int(on)))

    def timing_read(self):
        ms, nc, nk, nr = C.c_double(), C.c_int(), C.c_longlong(), C.c_int()
        _check(lib().nbc_timing_read(self.h, C.byref(ms), C.byref(nc), C.byref(nk), C.byref(nr)))
        return {"contact_ms": ms.value, "contact_launches": nc.value, "kernel_launches": nk.value,
                "rebuilds": nr.value}

    def timing_phases(self):
        """Mean ms per timed step (timing level 2): clump, rebuild node, boundary, contact, step."""
        a = np.zeros(5)
        _check(lib().nbc_timing_phases(self.h, _p(a, P_D)))
        return dict(zip(("clump", "rebuild", "boundary", "contact", "step"), a.tolist()))

    def set_steps(self, nsteps, s=0):
        """Scene s stands still after nsteps steps from the engine's creation (0: no limit)."""
        _check(lib().nbc_set_scene_steps(self.h, int(s), int(nsteps)))

    def info(self):
        b, ms = C.c_double(), C.c_double()
        _check(lib().nbc_engine_info(self.h, C.byref(b), C.byref(ms)))
        return {"device_bytes": b.value, "last_step_ms": ms.value}


TUNED_KEYS = ("search_lanes", "clump_batch", "pair_blocks")


def _options(precision="mixed", use_graph=True, device=0, pair_slack=0.0, search_lanes=0, clump_batch=0,
             pair_blocks=0, tuned=None):
    """nbc_options; `tuned` (a dict from autotune) overrides the launch shapes."""
    o = Options()
    lib().nbc_default_options(C.byref(o))
    o.precision, o.use_graph, o.device = PREC[precision], int(use_graph), device
    o.pair_slack = pair_slack
    o.search_lanes, o.clump_batch, o.pair_blocks = search_lanes, clump_batch, pair_blocks
    for k in TUNED_KEYS:
        if tuned and k in tuned:
            setattr(o, k, int(tuned[k]))
    return o


def autotune(scenes, precision="mixed", device=0, trial_steps=200, cache=None):
    """nbc_autotune: the fastest launch shapes for these scenes (a dict of
    TUNED_KEYS plus ms_per_step).  `cache`, a JSON file, keeps the choice by
    scene shape across processes, so a shape is measured once."""
    import json
    key = "|".join(str(x) for x in (len(scenes), sum(int(s["params"]["NumberBody"]) for s in scenes),
                                    sum(int(s["params"]["ClumpNum"]) for s in scenes),
                                    max(len(s["levels"]["cell"]) if s.get("levels") else 1 for s in scenes),
                                    precision, trial_steps))
    book = {}
    if cache and os.path.exists(cache):
        with open(cache) as f:
            book = json.load(f)
        if key in book:
            return dict(book[key], cached=True)
    descs = [scene_desc(s) for s in scenes]
    arr = (C.POINTER(SceneDesc) * len(scenes))(*[C.pointer(d) for d, _ in descs])
    o = _options(precision, True, device)
    ms = C.c_double(0.0)
    _check(lib().nbc_autotune(arr, len(scenes), C.byref(o), int(trial_steps), C.byref(ms)))
    out = {k: int(getattr(o, k)) for k in TUNED_KEYS}
    out["ms_per_step"] = ms.value
    if cache:
        book[key] = out
        with open(cache, "w") as f:
            json.dump(book, f, indent=1, sort_keys=True)
    return dict(out, cached=False)


class SceneView:
    """Scene s of a multi-scene engine: the per-scene getters of Engine with
    the scene index bound."""

    _PER_SCENE = ("stats", "subspheres", "clumps", "sub_forces", "force_parts", "pairs", "rows", "chain", "pair_forces",
                  "intruder", "intruder_diag", "intruder_history", "restart_scene", "set_steps")

    def __init__(self, engine, s):
        self.engine, self.s = engine, s

    def sync(self):
        self.engine.sync()

    def __getattr__(self, name):
        if name in SceneView._PER_SCENE:
            f = getattr(self.engine, name)
            return lambda *a, **k: f(*a, s=self.s, **k)
        raise AttributeError(name)


class Batch:
    """Independent scenes advanced together (nbc_batch_*): one engine over
    all of them, one launch per kernel and step; each scene's results equal
    those of the scene run alone.  engines[i] is scene i's view."""

    def __init__(self, scenes, **opts):
        self._descs = [scene_desc(s) for s in scenes]
        arr = (C.POINTER(SceneDesc) * len(scenes))(*[C.pointer(d) for d, _ in self._descs])
        o = _options(**opts)
        h = C.c_void_p()
        _check(lib().nbc_batch_create(arr, len(scenes), C.byref(o), C.byref(h)))
        self.h = h
        e = C.c_void_p()
        _check(lib().nbc_batch_engine(self.h, C.byref(e)))
        self.engine = Engine.borrowed(e, scenes)
        self.engines = [SceneView(self.engine, i) for i in range(len(scenes))]

    def step(self, n=1):
        _check(lib().nbc_batch_step(self.h, int(n)))

    def sync(self):
        self.engine.sync()

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.engine.h = None
            lib().nbc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous batching of requests (nbc_server_*): a request is a scene
    and a step count; its result is the intruder reaction sampled every
    sample_every steps and the intruder's final position."""

    def __init__(self, budget_bytes, max_active=64, cohort=1, **opts):
        o = _options(**opts)
        h = C.c_void_p()
        _check(lib().nbc_server_create(C.byref(o), C.c_double(budget_bytes), int(max_active), C.byref(h)))
        self.h = h
        _check(lib().nbc_server_set_cohort(self.h, int(cohort)))

    def submit(self, scene, nsteps, sample_every=100):
        d, keep = scene_desc(scene)
        rid = C.c_int()
        _check(lib().nbc_server_submit(self.h, C.byref(d), int(nsteps), int(sample_every), C.byref(rid)))
        return rid.value

    def advance(self, chunk=200):
        a, q, f = C.c_int(), C.c_int(), C.c_int()
        _check(lib().nbc_server_advance(self.h, int(chunk), C.byref(a), C.byref(q), C.byref(f)))
        return {"running": a.value, "queued": q.value, "finished": f.value}

    def state(self, rid):
        st, done, ns = C.c_int(), C.c_int(), C.c_int()
        _check(lib().nbc_server_result(self.h, int(rid), C.byref(st), C.byref(done), C.byref(ns), None, None))
        return st.value, done.value, ns.value

    def result(self, rid):
        st, done, ns = self.state(rid)
        if st not in (2, 3):
            return None
        curve, pos = np.zeros((ns, 6)), np.zeros(3)
        _check(lib().nbc_server_result(self.h, int(rid), None, None, None, _p(curve), _p(pos)))
        return {"curve": curve, "intr_pos": pos, "steps": done}

    def release(self, rid):
        _check(lib().nbc_server_release(self.h, int(rid)))

    def memory(self):
        u, b = C.c_double(), C.c_double()
        _check(lib().nbc_server_memory(self.h, C.byref(u), C.byref(b)))
        return u.value, b.value

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().nbc_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""ctypes binding of the FP64 CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and
bench.py's CPU baseline to check or time against the reference algorithm;
the engine never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

D3 = C.c_double * 3
D4 = C.c_double * 4
P_D = C.POINTER(C.c_double)
P_I = C.POINTER(C.c_int)


class Desc(C.Structure):
    _fields_ = [
        ("N", C.c_int), ("K", C.c_int), ("BL", C.c_int),
        ("start_step", C.c_int), ("end_step", C.c_int), ("output_interval", C.c_int),
        ("dt", C.c_double), ("E", C.c_double), ("nu", C.c_double), ("mu", C.c_double),
        ("e_rest", C.c_double), ("beta", C.c_double), ("cohesion", C.c_double),
        ("gravity", C.c_double), ("thresh", C.c_double),
        ("world_origin", D3), ("world_size", D3), ("box_lo", D3), ("box_hi", D3),
        ("is_wall", C.c_int), ("is_intruder", C.c_int),
        ("clump_id", P_I), ("pos", P_D), ("local", P_D), ("mass", P_D), ("radius", P_D),
        ("cpos", P_D), ("cvel", P_D), ("cquat", P_D), ("cangvel", P_D), ("cprop", P_D),
        ("has_cube", C.c_int),
        ("cube_half", D3), ("cube_centre", D3), ("cube_vel", D3), ("cube_quat", D4),
        ("cube_angvel", D3),
        ("has_cyl", C.c_int),
        ("cyl_radius", C.c_double), ("cyl_half_height", C.c_double), ("cyl_axis", D3),
        ("cyl_centre", D3), ("cyl_vel", D3), ("cyl_angvel", D3),
        ("intr_shape", C.c_int), ("intr_motion", C.c_int), ("intr_wait", C.c_int),
        ("intr_radius", C.c_double), ("intr_half_height", C.c_double), ("intr_axis", D3),
        ("intr_prop", D4), ("intr_pos", D3), ("intr_vel", D3), ("intr_quat", D4),
        ("intr_angvel", D3),
        ("levels", C.c_int), ("level", P_I), ("level_cell", P_D),
        ("sphere_mode", C.c_int), ("body_kind", P_I),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.nbo_create.restype = C.c_void_p
        L.nbo_create.argtypes = [C.POINTER(Desc)]
        L.nbo_destroy.argtypes = [C.c_void_p]
        L.nbo_step.argtypes = [C.c_void_p, C.c_int]
        L.nbo_step.restype = C.c_int
        L.nbo_set_threads.argtypes = [C.c_int]
        for f in ("nbo_num_pairs", "nbo_step_count", "nbo_rebuild_count"):
            getattr(L, f).argtypes = [C.c_void_p]
            getattr(L, f).restype = C.c_int
        for f in ("nbo_get_sub", "nbo_get_clumps", "nbo_get_sub_forces", "nbo_get_pairs",
                  "nbo_get_rows", "nbo_get_pair_caches", "nbo_get_chain", "nbo_get_intruder",
                  "nbo_get_intruder_diag"):
            getattr(L, f).restype = None
        _lib = L
    return _lib


def _p(a, t=P_D):
    return a.ctypes.data_as(t) if a is not None else None


def _set(arr, vals):
    for i, v in enumerate(vals):
        arr[i] = float(v)


class OracleScene:
    """One scene advanced by the CPU oracle.  `scene` is a scenegen dict."""

    def __init__(self, scene: dict, threads: int = 1):
        L = lib()
        L.nbo_set_threads(int(threads))
        p = scene["params"]
        s, c = scene["sub"], scene["clump"]
        self.N, self.K, self.BL = int(p["NumberBody"]), int(p["ClumpNum"]), int(p["BranchLmtLen"])
        keep = self._keep = {}
        keep["cid"] = np.ascontiguousarray(s["clump_id"], dtype=np.int32)
        for k in ("pos", "local", "mass", "radius"):
            keep[k] = np.ascontiguousarray(s[k], dtype=np.float64)
        for k in ("pos", "vel", "quat", "angvel", "prop"):
            keep["c" + k] = np.ascontiguousarray(c[k], dtype=np.float64)
        d = Desc()
        d.N, d.K, d.BL = self.N, self.K, self.BL
        d.start_step, d.end_step = int(p["StartStep"]), int(p["EndStep"])
        d.output_interval = int(p["OutputInterval"])
        d.dt, d.E, d.nu, d.mu = p["StepSize"], p["Ymod"], p["Prat"], p["Frcoe"]
        d.e_rest, d.beta, d.cohesion = p["NormRes"], p["Beta"], p["Cohesion"]
        d.gravity, d.thresh = p["Gravity"], p["Thresh"]
        _set(d.world_origin, [p["WorldOrigin_" + a] for a in "xyz"])
        _set(d.world_size, [p["WorldSize_" + a] for a in "xyz"])
        _set(d.box_lo, [p["BoxLowLmt_" + a] for a in "xyz"])
        _set(d.box_hi, [p["BoxUpLmt_" + a] for a in "xyz"])
        d.is_wall, d.is_intruder = int(p["isWallForce"]), int(p["isIntruder"])
        d.clump_id = _p(keep["cid"], P_I)
        d.pos, d.local = _p(keep["pos"]), _p(keep["local"])
        d.mass, d.radius = _p(keep["mass"]), _p(keep["radius"])
        d.cpos, d.cvel, d.cquat = _p(keep["cpos"]), _p(keep["cvel"]), _p(keep["cquat"])
        d.cangvel, d.cprop = _p(keep["cangvel"]), _p(keep["cprop"])
        cube = scene.get("cube")
        if cube is not None:
            d.has_cube = 1
            _set(d.cube_half, cube["half"]); _set(d.cube_centre, cube["centre"])
            _set(d.cube_vel, cube["vel"]); _set(d.cube_quat, cube["quat"])
            _set(d.cube_angvel, cube["angvel"])
        cyl = scene.get("cylinder")
        if cyl is not None:
            d.has_cyl = 1
            d.cyl_radius, d.cyl_half_height = cyl["radius"], cyl["half_height"]
            _set(d.cyl_axis, cyl["axis"]); _set(d.cyl_centre, cyl["centre"])
            _set(d.cyl_vel, cyl["vel"]); _set(d.cyl_angvel, cyl["angvel"])
        it = scene.get("intruder")
        if it is not None:
            d.intr_shape = 1 if it["shape"] == "sphere" else 0
            d.intr_motion = 0 if it["motion"] == "constant_velocity" else 1
            d.intr_wait = 1 if it["motion"] == "gravity_after_contact" else 0
            d.intr_radius, d.intr_half_height = it["radius"], it["half_height"]
            _set(d.intr_axis, it["axis"]); _set(d.intr_prop, it["prop"])
            _set(d.intr_pos, it["pos"]); _set(d.intr_vel, it["vel"])
            _set(d.intr_quat, it["quat"]); _set(d.intr_angvel, it["angvel"])
        lv = scene.get("levels")
        if lv is not None:
            keep["level"] = np.ascontiguousarray(lv["level"], dtype=np.int32)
            keep["level_cell"] = np.ascontiguousarray(lv["cell"], dtype=np.float64)
            d.levels = len(keep["level_cell"])
            d.level = _p(keep["level"], P_I)
            d.level_cell = _p(keep["level_cell"])
        # the reference's sphere-only drivers (scenegen.as_sphere_driver)
        d.sphere_mode = int(scene.get("sphere_mode", 0))
        if scene.get("body_kind") is not None:
            keep["body_kind"] = np.ascontiguousarray(scene["body_kind"], dtype=np.int32)
            d.body_kind = _p(keep["body_kind"], P_I)
        self._desc = d
        self.h = L.nbo_create(C.byref(d))

    def __del__(self):
        if getattr(self, "h", None):
            lib().nbo_destroy(self.h)
            self.h = None

    def step(self, n=1):
        rc = lib().nbo_step(self.h, int(n))
        if rc:
            raise RuntimeError(f"oracle step failed: {rc}")

    @property
    def npairs(self):
        return lib().nbo_num_pairs(self.h)

    @property
    def rebuilds(self):
        return lib().nbo_rebuild_count(self.h)

    def sub(self):
        N = self.N
        fix, cid = np.zeros(N, np.int32), np.zeros(N, np.int32)
        pos, rad = np.zeros((N, 3)), np.zeros(N)
        lib().nbo_get_sub(self.h, _p(fix, P_I), _p(cid, P_I), _p(pos), _p(rad))
        return {"part_fix": fix, "clump_id": cid, "pos": pos, "radius": rad}

    def clumps(self):
        K = self.K
        o = {k: np.zeros((K, 3)) for k in ("pos", "vel", "angvel", "force", "torque")}
        o["quat"] = np.zeros((K, 4))
        lib().nbo_get_clumps(self.h, _p(o["pos"]), _p(o["vel"]), _p(o["quat"]),
                             _p(o["angvel"]), _p(o["force"]), _p(o["torque"]))
        return o

    def sub_forces(self):
        N = self.N
        o = {k: np.zeros((N, 3)) for k in ("fc", "tc", "fw", "tw", "fi", "ti")}
        lib().nbo_get_sub_forces(self.h, *[_p(o[k]) for k in ("fc", "tc", "fw", "tw", "fi", "ti")])
        return o

    def pairs(self):
        P = self.npairs
        a, b = np.zeros(P, np.int32), np.zeros(P, np.int32)
        lib().nbo_get_pairs(self.h, _p(a, P_I), _p(b, P_I))
        return a, b

    def rows(self):
        N, BL = self.N, self.BL
        anei = np.zeros((N, BL), np.int32)
        ng, ni = np.zeros(N, np.int32), np.zeros(N, np.int32)
        lib().nbo_get_rows(self.h, _p(anei, P_I), _p(ng, P_I), _p(ni, P_I))
        return anei, ng, ni

    def pair_caches(self):
        P = self.npairs
        o = {k: np.zeros((P, 3)) for k in ("cfc", "cfcn", "cpt", "dv", "dt", "dr")}
        lib().nbo_get_pair_caches(self.h, *[_p(o[k]) for k in ("cfc", "cfcn", "cpt", "dv", "dt", "dr")])
        return o

    def chain(self):
        N, BL = self.N, self.BL
        f, c = np.zeros((N, BL, 3)), np.zeros((N, BL, 3))
        lib().nbo_get_chain(self.h, _p(f), _p(c))
        return f, c

    def intruder(self):
        o = {k: np.zeros(3) for k in ("pos", "vel", "totf", "tott", "reaction")}
        st = C.c_int(0)
        lib().nbo_get_intruder(self.h, _p(o["pos"]), _p(o["vel"]), _p(o["totf"]), _p(o["tott"]),
                               _p(o["reaction"]), C.byref(st))
        o["state"] = st.value
        return o

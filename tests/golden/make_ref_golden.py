"""Generate the golden vectors that pin the CPU oracle to the reference.

Two phases:

``prepare`` (run where the scene generator runs; no GPU):
    writes each case's input scene as ``<case>.scene.npz`` in this folder.
    The ``ref_fixture`` case is the reference's own input set
    (``src/world.par``, ``src/ph.00000000.bt``, ``src/ch.00000000.bt``,
    ``src/Rocks/*.bt``) re-read with ``scenegen.read_reference_inputs`` and
    stored in the same npz layout; it needs the reference tree (``--ref``).

``run`` (run on a machine with a B200 and the reference build
``oracle/_ref/nbody_clump_ref`` made by ``oracle/Makefile.ref``):
    for each case, writes the reference's text inputs into a scratch
    directory, runs the unmodified reference solver there (its own ``main``,
    ``DEMClumpMain::RunSimulationClump``), reads the raw binary outputs it
    writes (``OutPart/ph.*.bin``, ``OutClump/ch.*.bin``, ``OutCnt/*.bin``,
    ``OutForce/*.bin``; layouts of ``src/dem_binary_io.h``) and stores a
    compact ``<case>.ref.npz`` in ``--out``.

Cases in SPHERE_PATH run one of the reference's sphere-only drivers instead
(``oracle/_ref/nbody_sphere_ref <driver>``: ``DEMmain::RunSimulation``
(cylinder), ``RunSimulation2`` (cube), ``RunSimulation_Split`` and
``RunSimulation_HGrid``, ``src/dem_simulation_{cylind,cube,split,hgrid}.cu``).
Their scenes are one-sphere clumps with LocalPos = 0, written by
``scenegen.write_sphere_inputs`` in the sphere format (``ph`` with 21
columns, ``src/dem_io.cu:155-193``, the driver's wall file, and ``grid.bt``
for the hgrid driver); the driver's ``OutPart/ph.*.bin``
(``src/dem_io.cu:313-329``) gives positions, velocities, quaternions and
angular velocities at every step, and with an intruder
``OutPart/intruder.*.bin`` and ``OutForce/fc.*.bin`` its position and force
history (and ``OutCnt`` for the cube driver).

The ``.ref.npz`` files are committed next to this script and read by
``tests/test_oracle_golden.py`` and the GPU parity tests.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "nbody-clump_b200"))
import scenegen as sg  # noqa: E402
import refbin  # noqa: E402

# case -> (builder, steps, contact-output steps kept with forces)
CASES = {
    "ref_fixture": None,
    "spheres_cube_sphere": lambda: sg.make_test_spheres(n=343, seed=11, intruder="sphere",
                                                        wall="cube", steps=24),
    "tetra_cube_cyl": lambda: sg.make_test_tetra(n_clumps=100, seed=12, intruder="cylinder",
                                                 wall="cube", steps=24),
    "tetra_gravity": lambda: sg.make_test_tetra(n_clumps=80, seed=13, intruder="sphere",
                                                motion="gravity", wall="cube", steps=24),
    "spheres_gac": lambda: sg.make_test_spheres(n=216, seed=14, intruder="sphere",
                                                motion="gravity_after_contact", wall="cube",
                                                steps=24),
    "cfg0_settle": None,
    "cyl_spheres": lambda: sg.make_test_cyl("spheres", seed=31, steps=24, thresh_ratio=1e-3),
    "sph_cube": lambda: _cohesive(sg.make_test_spheres(n=343, seed=41, intruder="sphere", wall="cube",
                                                       steps=24), 5e3),
    "sph_cyl": lambda: sg.make_test_spheres(n=343, seed=42, intruder="cylinder", wall="cylinder", steps=24),
    "sph_hgrid": lambda: sg.make_test_sphere_levels(seed=43, steps=24),
    "sph_split": lambda: sg.make_test_split(seed=44, steps=24),
}
# cases run by the reference's sphere-only driver (oracle/_ref/nbody_sphere_ref <driver>)
SPHERE_PATH = {"cyl_spheres": "cylinder", "sph_cube": "cube", "sph_cyl": "cylinder", "sph_hgrid": "hgrid",
               "sph_split": "split"}


def _cohesive(sc, c):
    sc["params"]["Cohesion"] = c
    return sc
STEPS = 24
FORCE_STEPS = (2, 12, 24)


def prepare(ref_dir: str | None, names):
    for name in names:
        build = CASES[name]
        path = os.path.join(HERE, f"{name}.scene.npz")
        if name == "ref_fixture":
            if ref_dir is None:
                print("skip ref_fixture (no --ref)")
                continue
            sc = sg.read_reference_inputs(os.path.join(ref_dir, "src"))
            sc.pop("cylinder_file", None)
            sc["params"]["EndStep"] = STEPS
            sc["params"]["OutputInterval"] = 1
        elif name == "cfg0_settle":
            sc = sg.make_cfg0(steps=10000)
            sc["params"]["OutputInterval"] = 1000
        else:
            sc = build()
            sc["params"]["EndStep"] = STEPS
            sc["params"]["OutputInterval"] = 1
        sg.scene_to_npz(sc, path)
        print("wrote", path, sc["params"]["NumberBody"], "subspheres")


def run_sphere_case(binary: str, name: str, out: str, keep: bool):
    sc = sg.scene_from_npz(os.path.join(HERE, f"{name}.scene.npz"))
    work = tempfile.mkdtemp(prefix=f"ref_{name}_")
    driver = SPHERE_PATH[name]
    sg.write_sphere_inputs(sc, work, driver)
    t0 = time.time()
    r = subprocess.run([binary, driver], cwd=work, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       timeout=900)
    wall = time.time() - t0
    if r.returncode != 0:
        print(r.stdout.decode(errors="replace")[-3000:])
        raise SystemExit(f"reference sphere driver failed on {name}: rc={r.returncode}")
    p = sc["params"]
    steps = p["EndStep"] - p["StartStep"]
    res = {"wall_s": np.array(wall), "steps": np.array(steps)}
    for s in range(p["OutputInterval"], steps + 1, p["OutputInterval"]):
        ph = refbin.read_sphere_ph(os.path.join(work, "OutPart", "ph.%08d.bin" % s))
        for k in ("part_fix", "pos", "vel", "quat", "angvel"):
            res[f"s{s}/{k}"] = ph[k]
        if p["isIntruder"]:
            it = refbin.read_ch(os.path.join(work, "OutPart", "intruder.%08d.bin" % s))
            fc = refbin.read_fc(os.path.join(work, "OutForce", "fc.%08d.bin" % s))
            res[f"s{s}/intr_pos"] = it["pos"][0]
            res[f"s{s}/intr_force"] = fc["force"]
    if p["isIntruder"] and driver == "cube":
        for s in range(2 * p["OutputInterval"], steps + 1, 2 * p["OutputInterval"]):
            nei = refbin.read_cnt(os.path.join(work, "OutCnt", "Nei.%08d.bin" % s), np.int32)
            rows, slots = np.nonzero(nei >= 0)
            res[f"c{s}/rows"] = rows.astype(np.int32)
            res[f"c{s}/slots"] = slots.astype(np.int16)
            res[f"c{s}/nei"] = nei[rows, slots].astype(np.int32)
    np.savez_compressed(os.path.join(out, f"{name}.ref.npz"), **res)
    print(f"{name}: {steps} steps in {wall:.2f} s wall (reference sphere driver, incl. file IO)")
    if not keep:
        shutil.rmtree(work, ignore_errors=True)


def run_case(binary: str, name: str, out: str, keep: bool):
    sc = sg.scene_from_npz(os.path.join(HERE, f"{name}.scene.npz"))
    work = tempfile.mkdtemp(prefix=f"ref_{name}_")
    sg.write_reference_inputs(sc, work)
    t0 = time.time()
    r = subprocess.run([binary], cwd=work, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       timeout=900)
    wall = time.time() - t0
    log = r.stdout.decode(errors="replace")
    if r.returncode != 0:
        print(log[-3000:])
        raise SystemExit(f"reference failed on {name}: rc={r.returncode}")
    p = sc["params"]
    steps = p["EndStep"] - p["StartStep"]
    interval = p["OutputInterval"]
    res = {"wall_s": np.array(wall), "steps": np.array(steps)}
    outs = list(range(interval, steps + 1, interval))
    for s in outs:
        ph = refbin.read_ph(os.path.join(work, "OutPart", "ph.%08d.bin" % s))
        ch = refbin.read_ch(os.path.join(work, "OutClump", "ch.%08d.bin" % s))
        res[f"s{s}/part_fix"] = ph["part_fix"]
        res[f"s{s}/pos"] = ph["pos"]
        for k in ("pos", "vel", "quat", "angvel"):
            res[f"s{s}/clump_{k}"] = ch[k]
        if p["isIntruder"]:
            fc = refbin.read_fc(os.path.join(work, "OutForce", "fc.%08d.bin" % s))
            res[f"s{s}/intr_force"] = fc["force"]
            res[f"s{s}/intr_torque"] = fc["torque"]
    for s in range(2 * interval, steps + 1, 2 * interval):
        nei = refbin.read_cnt(os.path.join(work, "OutCnt", "Nei.%08d.bin" % s), np.int32)
        rows, slots = np.nonzero(nei >= 0)
        res[f"c{s}/rows"] = rows.astype(np.int32)
        res[f"c{s}/slots"] = slots.astype(np.int16)
        res[f"c{s}/nei"] = nei[rows, slots].astype(np.int32)
        if s in FORCE_STEPS or (name == "cfg0_settle" and s == steps):
            fcn = refbin.read_cnt(os.path.join(work, "OutCnt", "Fcn.%08d.bin" % s), "3f8")
            cpt = refbin.read_cnt(os.path.join(work, "OutCnt", "Cpt.%08d.bin" % s), "3f8")
            res[f"c{s}/fcn"] = fcn[rows, slots]
            res[f"c{s}/cpt"] = cpt[rows, slots]
    np.savez_compressed(os.path.join(out, f"{name}.ref.npz"), **res)
    print(f"{name}: {steps} steps in {wall:.2f} s wall (reference, incl. file IO)")
    if not keep:
        shutil.rmtree(work, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("phase", choices=["prepare", "run"])
    ap.add_argument("--ref", default=None, help="reference tree (prepare)")
    ap.add_argument("--binary", default=os.path.join(REPO, "oracle", "_ref", "nbody_clump_ref"))
    ap.add_argument("--sphere-binary", default=os.path.join(REPO, "oracle", "_ref", "nbody_sphere_ref"))
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--cases", default=",".join(CASES))
    ap.add_argument("--keep", action="store_true")
    a = ap.parse_args()
    if a.phase == "prepare":
        prepare(a.ref, a.cases.split(","))
        return
    os.makedirs(a.out, exist_ok=True)
    for name in a.cases.split(","):
        if not os.path.exists(os.path.join(HERE, f"{name}.scene.npz")):
            continue
        if name in SPHERE_PATH:
            run_sphere_case(a.sphere_binary, name, a.out, a.keep)
        else:
            run_case(a.binary, name, a.out, a.keep)


if __name__ == "__main__":
    main()

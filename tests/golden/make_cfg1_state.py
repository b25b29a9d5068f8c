"""Make the contact-rich cfg1 state the benchmark and the cfg1 parity test
start from (needs a CUDA device).

The cfg1 bed (50,000 tetrahedral clumps, 200,000 subspheres, closed
cylinder R = 60 mm, half-height 150 mm, hierarchical grid chosen by
nbc_choose_levels) is generated with its default seed and settled by the
engine (mixed precision, as benchmarked) for --steps steps; the state reached
is written as a compact snapshot (scenegen.tetra_state_to_npz: clump poses,
velocities, size scales and grid levels).  Every --sample steps the script
prints the step, the rebuilds so far, the listed, near and touching pairs
and the mean clump speed, which is how the snapshot step was picked: late
enough that the bed is a dense packing with most subspheres in contact,
early enough that it still moves and rebuilds its list.

    python tests/golden/make_cfg1_state.py --steps 20000 --out tests/golden/cfg1_settled.npz
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "nbody-clump_b200"))
import nbc  # noqa: E402
import scenegen as sg  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--sample", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=20260828)
    ap.add_argument("--out", default=os.path.join(HERE, "cfg1_settled.npz"))
    ap.add_argument("--also", default="", help="extra snapshot steps, comma separated (written beside --out)")
    a = ap.parse_args()
    scene = nbc.with_levels(sg.make_cfg1(seed=a.seed))
    scales = sg.tetra_scales(seed=a.seed)
    extra = sorted(int(x) for x in a.also.split(",") if x)
    eng = nbc.Engine([scene], precision="mixed")
    done = 0
    marks = sorted(set(range(a.sample, a.steps + 1, a.sample)) | set(extra) | {a.steps})
    for m in marks:
        eng.step(m - done)
        done = m
        st = eng.stats()
        near, touch = eng.contact_counts()
        speed = np.linalg.norm(eng.clumps()["vel"], axis=1)
        print(json.dumps({"step": m, "rebuilds": st["rebuilds"], "pairs": st["npairs"], "near": near,
                          "touching": touch, "speed_mean": float(speed.mean()), "speed_max": float(speed.max())}),
              flush=True)
        if m in extra or m == a.steps:
            state = eng.restart_scene(scene)
            path = a.out if m == a.steps else a.out.replace(".npz", f".{m}.npz")
            sg.tetra_state_to_npz(state, scales, path, steps=m, seed=a.seed)
            print(json.dumps({"wrote": path, "bytes": os.path.getsize(path)}), flush=True)
    eng.close()


if __name__ == "__main__":
    main()

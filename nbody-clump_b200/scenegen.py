"""Scene generator and reader/writer for the reference's text input formats.

A *scene* is a plain dict of numpy arrays and scalars:

    params   dict of the 38 ``world.par`` keys (``src/dem_subsphere_io.cu:83-128``)
    sub      dict: clump_id int32[N], pos f64[N,3], local f64[N,3], mass f64[N],
             radius f64[N]                       (ph columns, ``src/dem_subsphere_io.cu:174-175``)
    clump    dict: pos, vel, angvel f64[K,3], quat f64[K,4] (x,y,z,w),
             prop f64[K,4] = (Ixx, Iyy, Izz, M)  (ch columns, ``src/dem_clumpsphere_io.cu:46-48``)
    cube     dict or None: half f64[3], centre, vel, angvel f64[3], quat f64[4]
             (``src/dem_cube_wall_io.cu:43-48``)
    cylinder dict or None: radius, half_height, axis f64[3], prop f64[4], centre, vel,
             angvel f64[3], quat f64[4]          (``src/dem_cylind_wall_io.cu:41-49``)
    intruder dict or None: shape 'sphere'|'cylinder', radius, half_height, axis f64[3],
             prop f64[4], pos, vel, angvel f64[3], quat f64[4],
             motion 'constant_velocity'|'gravity'|'gravity_after_contact'
             (``src/dem_penetrator_io.cu:42-115``)

The builders below produce the synthetic workloads the engine is measured on
(monodisperse spheres, tetrahedral clumps, polydisperse clumps) with seeded
numpy generators, so every scene is reproducible from its seed.
"""
from __future__ import annotations

import math
import os

import numpy as np

# Parameter keys in the order the reference's world.par lists them.
PAR_KEYS = [
    "NumberBody", "ClumpNum", "BranchLmtLen", "BodyFileDir", "IniConFile",
    "StepSize", "EndStep", "StartStep", "OutputInterval",
    "Ymod", "Prat", "Frcoe", "NormRes", "Frvel", "Beta", "MU_T", "MU_R", "Cohesion",
    "Gravity", "Thresh", "GridLevels", "Update",
    "WorldSize_x", "WorldSize_y", "WorldSize_z",
    "WorldOrigin_x", "WorldOrigin_y", "WorldOrigin_z",
    "BoxUpLmt_x", "BoxUpLmt_y", "BoxUpLmt_z",
    "BoxLowLmt_x", "BoxLowLmt_y", "BoxLowLmt_z",
    "isIntruder", "isSelfGravity", "isWallForce", "isQuaternion",
]
assert len(PAR_KEYS) == 38

PI_REF = 3.14159265359  # the reference's PI literal (src/dem_constant.h:14)


def damping_from_restitution(e: float) -> float:
    """Damping ratio derived from restitution, as the reference's
    LoadParameters computes it (src/dem_subsphere_io.cu:143-145)."""
    ln = math.log(e)
    return 2.0 * math.sqrt(5.0 / 6.0) * ln / math.sqrt(ln * ln + PI_REF * PI_REF)


def rayleigh_dt(r: float, rho: float, E: float, nu: float) -> float:
    """Rayleigh time step pi r sqrt(rho/G) / (0.1631 nu + 0.8766)."""
    G = E / (2.0 * (1.0 + nu))
    return math.pi * r * math.sqrt(rho / G) / (0.1631 * nu + 0.8766)


# ----------------------------------------------------------------------------
# quaternion helpers (x, y, z, w) with w the scalar, the reference convention
# ----------------------------------------------------------------------------

def quat_to_body2world(q: np.ndarray) -> np.ndarray:
    """Rotation matrices C_bn (body -> world) for quaternions q[...,4].

    Same matrix as the reference's Quat2IvDCM (src/type.h:238-250)."""
    x, y, z, w = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    m = np.empty(q.shape[:-1] + (3, 3))
    m[..., 0, 0] = x * x - y * y - z * z + w * w
    m[..., 1, 0] = 2.0 * (x * y + z * w)
    m[..., 2, 0] = 2.0 * (x * z - y * w)
    m[..., 0, 1] = 2.0 * (x * y - z * w)
    m[..., 1, 1] = -x * x + y * y - z * z + w * w
    m[..., 2, 1] = 2.0 * (y * z + x * w)
    m[..., 0, 2] = 2.0 * (x * z + y * w)
    m[..., 1, 2] = 2.0 * (y * z - x * w)
    m[..., 2, 2] = -x * x - y * y + z * z + w * w
    return m


def random_unit_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniformly distributed unit quaternions (Shoemake's method)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
    q = np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2),
                  b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)], axis=1)
    return q


# ----------------------------------------------------------------------------
# clump templates
# ----------------------------------------------------------------------------

def tetra_template(r: float = 1.0, offset_ratio: float = 0.6) -> np.ndarray:
    """Four subsphere centres on a regular tetrahedron at distance
    offset_ratio*r from the centroid (body frame)."""
    v = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=np.float64)
    v /= np.linalg.norm(v[0])
    return v * (offset_ratio * r)


def union_mass_properties(centres: np.ndarray, radii: np.ndarray, rho: float,
                          samples: int = 400_000, seed: int = 7):
    """Mass, centre of mass and inertia tensor of a union of spheres by
    seeded Monte Carlo over the bounding box."""
    rng = np.random.default_rng(seed)
    lo = (centres - radii[:, None]).min(0)
    hi = (centres + radii[:, None]).max(0)
    pts = lo + (hi - lo) * rng.random((samples, 3))
    inside = np.zeros(samples, dtype=bool)
    for c, rr in zip(centres, radii):
        inside |= ((pts - c) ** 2).sum(1) <= rr * rr
    vol = np.prod(hi - lo) * inside.mean()
    p = pts[inside]
    com = p.mean(0)
    d = p - com
    cov = (d[:, :, None] * d[:, None, :]).mean(0)
    inertia = rho * vol * (np.trace(cov) * np.eye(3) - cov)
    return rho * vol, com, inertia


def _principal_frame(centres, radii, rho):
    """Re-express a template in its principal frame; returns (centres', I_principal, M)."""
    M, com, I = union_mass_properties(centres, radii, rho)
    w, V = np.linalg.eigh(I)
    if np.linalg.det(V) < 0:
        V[:, 0] = -V[:, 0]
    return (centres - com) @ V, w, M


# ----------------------------------------------------------------------------
# scene assembly
# ----------------------------------------------------------------------------

def default_params(**kw) -> dict:
    p = {
        "NumberBody": 0, "ClumpNum": 0, "BranchLmtLen": 64,
        "BodyFileDir": "./Rocks/", "IniConFile": "ph.00000000.bt",
        "StepSize": 1e-5, "EndStep": 1, "StartStep": 0, "OutputInterval": 1,
        "Ymod": 1e7, "Prat": 0.3, "Frcoe": 0.5, "NormRes": 0.5, "Frvel": 5e-4,
        "Beta": 0.5, "MU_T": 0.5, "MU_R": 0.5, "Cohesion": 0.0,
        "Gravity": -9.81, "Thresh": 1e-4, "GridLevels": 1, "Update": 0,
        "WorldSize_x": 0.1, "WorldSize_y": 0.1, "WorldSize_z": 0.1,
        "WorldOrigin_x": 0.0, "WorldOrigin_y": 0.0, "WorldOrigin_z": 0.0,
        "BoxUpLmt_x": 0.1, "BoxUpLmt_y": 0.1, "BoxUpLmt_z": 0.1,
        "BoxLowLmt_x": 0.0, "BoxLowLmt_y": 0.0, "BoxLowLmt_z": 0.0,
        "isIntruder": 0, "isSelfGravity": 0, "isWallForce": 1, "isQuaternion": 1,
    }
    p.update(kw)
    return p


def set_world_box(params: dict, lo, hi):
    """World box = hashing box = [lo, hi] (the reference pads it by one cell itself)."""
    lo = np.asarray(lo, float)
    hi = np.asarray(hi, float)
    for a, k in enumerate("xyz"):
        params["WorldOrigin_" + k] = float(lo[a])
        params["WorldSize_" + k] = float(hi[a] - lo[a])
        params["BoxLowLmt_" + k] = float(lo[a])
        params["BoxUpLmt_" + k] = float(hi[a])


def assemble(params, clump_pos, clump_quat, clump_vel, clump_angvel, clump_prop,
             members_local, members_radius, members_mass, cube=None, cylinder=None,
             intruder=None) -> dict:
    """Build a scene from per-clump poses and per-clump member lists.

    members_local[k] is an (n_k, 3) array of body-frame offsets, members_radius[k]
    and members_mass[k] are (n_k,) arrays.  Subsphere world positions are
    X_c + C_bn(q) local, the pose the reference's UpdatePos computes."""
    K = len(clump_pos)
    counts = np.array([len(m) for m in members_local], dtype=np.int64)
    cid = np.repeat(np.arange(K, dtype=np.int32), counts)
    local = np.concatenate(members_local, axis=0)
    radius = np.concatenate(members_radius)
    mass = np.concatenate(members_mass)
    R = quat_to_body2world(clump_quat)
    pos = clump_pos[cid] + np.einsum("nij,nj->ni", R[cid], local)
    params = dict(params)
    params["NumberBody"] = int(len(cid))
    params["ClumpNum"] = int(K)
    params["isWallForce"] = 1 if (cube is not None or cylinder is not None) else 0
    params["isIntruder"] = 1 if intruder is not None else 0
    return {
        "params": params,
        "sub": {"clump_id": cid, "pos": pos, "local": local, "mass": mass, "radius": radius},
        "clump": {"pos": np.ascontiguousarray(clump_pos, dtype=np.float64),
                  "vel": np.ascontiguousarray(clump_vel, dtype=np.float64),
                  "quat": np.ascontiguousarray(clump_quat, dtype=np.float64),
                  "angvel": np.ascontiguousarray(clump_angvel, dtype=np.float64),
                  "prop": np.ascontiguousarray(clump_prop, dtype=np.float64)},
        "cube": cube, "cylinder": cylinder, "intruder": intruder,
    }


def make_cube(half, centre, vel=(0, 0, 0), angvel=(0, 0, 0), quat=(1.0, 0, 0, 0)):
    return {"half": np.array(half, float), "centre": np.array(centre, float),
            "vel": np.array(vel, float), "angvel": np.array(angvel, float),
            "quat": np.array(quat, float)}


def make_cylinder(radius, half_height, centre, axis=(0, 0, 1), prop=(1, 1, 1, 1),
                  vel=(0, 0, 0), angvel=(0, 0, 0), quat=(0, 0, 0, 1.0)):
    return {"radius": float(radius), "half_height": float(half_height),
            "axis": np.array(axis, float), "prop": np.array(prop, float),
            "centre": np.array(centre, float), "vel": np.array(vel, float),
            "angvel": np.array(angvel, float), "quat": np.array(quat, float)}


def make_intruder(shape, radius, pos, vel, half_height=None, axis=(0, 0, 1),
                  prop=(1, 1, 1, 1), angvel=(0, 0, 0), quat=(0, 0, 0, 1.0),
                  motion="constant_velocity"):
    if half_height is None:
        half_height = radius
    return {"shape": shape, "radius": float(radius), "half_height": float(half_height),
            "axis": np.array(axis, float), "prop": np.array(prop, float),
            "pos": np.array(pos, float), "vel": np.array(vel, float),
            "angvel": np.array(angvel, float), "quat": np.array(quat, float),
            "motion": motion}


def lattice_points(rng, n, spacing, lo, nx, ny, jitter):
    """n points on a cubic lattice filling x, then y, then z layers."""
    idx = np.arange(n)
    ix, iy, iz = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    pts = np.stack([ix, iy, iz], axis=1) * spacing + np.asarray(lo, float)
    if jitter > 0:
        pts = pts + rng.uniform(-jitter, jitter, size=pts.shape)
    return pts


# ----------------------------------------------------------------------------
# the measured workloads
# ----------------------------------------------------------------------------

MATERIAL = {"Ymod": 1e7, "Prat": 0.3, "Frcoe": 0.5, "NormRes": 0.5, "rho": 2650.0}


def make_cfg0(n: int = 2000, seed: int = 20260828, steps: int = 10000) -> dict:
    """2,000 monodisperse one-sphere clumps (r = 1 mm) on a 2.2 r lattice with
    +-0.1 r jitter settling in a 40 x 40 x 80 mm cube wall; dt = 0.2 dt_Rayleigh."""
    rng = np.random.default_rng(seed)
    r, rho = 1e-3, MATERIAL["rho"]
    m = rho * 4.0 / 3.0 * math.pi * r ** 3
    I = 0.4 * m * r * r
    dt = 0.2 * rayleigh_dt(r, rho, MATERIAL["Ymod"], MATERIAL["Prat"])
    sp = 2.2 * r
    pts = lattice_points(rng, n, sp, (1.1 * r, 1.1 * r, 1.1 * r), 18, 18, 0.1 * r)
    params = default_params(StepSize=dt, EndStep=steps, OutputInterval=steps,
                            Ymod=MATERIAL["Ymod"], Prat=MATERIAL["Prat"],
                            Frcoe=MATERIAL["Frcoe"], NormRes=MATERIAL["NormRes"],
                            Thresh=0.2 * r, BranchLmtLen=64)
    set_world_box(params, (0, 0, 0), (0.04, 0.04, 0.08))
    K = n
    return assemble(params, pts, np.tile([0, 0, 0, 1.0], (K, 1)), np.zeros((K, 3)),
                    np.zeros((K, 3)), np.tile([I, I, I, m], (K, 1)),
                    [np.zeros((1, 3))] * K, [np.array([r])] * K, [np.array([m])] * K,
                    cube=make_cube((0.02, 0.02, 0.04), (0.02, 0.02, 0.04)))


def _tetra_members(scales, r, offset_ratio, rho):
    base = tetra_template(1.0, offset_ratio)
    cen, Ip, M1 = _principal_frame(base, np.ones(4), rho)  # unit-size template
    locals_, radii, masses, props = [], [], [], []
    for s in scales:
        rr = r * s
        M = M1 * rr ** 3
        locals_.append(cen * rr)
        radii.append(np.full(4, rr))
        masses.append(np.full(4, M / 4.0))
        props.append([Ip[0] * rr ** 5, Ip[1] * rr ** 5, Ip[2] * rr ** 5, M])
    return locals_, radii, masses, np.array(props)


def layered_packing(rng, diam, R, z0, jitter=0.02):
    """Clump centres in horizontal square-lattice layers inside a circle of
    radius R: clumps sorted by size (largest first), each layer spaced by its
    largest member's diameter * 1.05, layer order shuffled within a layer."""
    order = np.argsort(-diam, kind="stable")
    pts = np.zeros((len(diam), 3))
    z = z0
    i = 0
    while i < len(order):
        d = 1.05 * diam[order[i]]
        n = int(2 * (R - 0.5 * d) / d) + 1
        g = (np.arange(n) - (n - 1) / 2.0) * d
        gx, gy = np.meshgrid(g, g, indexing="ij")
        inside = gx ** 2 + gy ** 2 <= (R - 0.5 * d) ** 2
        xy = np.stack([gx[inside], gy[inside]], axis=1)
        take = order[i:i + len(xy)]
        sel = rng.permutation(len(xy))[:len(take)]
        pts[take, 0:2] = xy[sel] + rng.uniform(-jitter * d, jitter * d, (len(take), 2))
        pts[take, 2] = z + 0.5 * d
        z += d
        i += len(take)
    return pts


def make_cfg1(n_clumps: int = 50_000, seed: int = 20260828, steps: int = 20000, mu: float = None,
              fit_box: bool = False) -> dict:
    """50,000 tetrahedral clumps (4 subspheres, r = 1 mm, centre offset 0.6 r,
    log-normal(0, 0.2) size scale, random orientation) seeded in layers inside
    a closed cylinder wall (R = 60 mm, height 300 mm = half-height 150 mm,
    axis z, floor at z = 0; the layers reach z = 0.19 m) and settling under
    gravity.  mu overrides the friction; fit_box
    ends the hashing box a few clump sizes above the seeded bed (the bed only
    falls) instead of at the cylinder top, so small beds get small grids."""
    rng = np.random.default_rng(seed)
    r, rho = 1e-3, MATERIAL["rho"]
    scales = rng.lognormal(0.0, 0.2, n_clumps)
    locals_, radii, masses, props = _tetra_members(scales, r, 0.6, rho)
    diam = 2.0 * np.array([np.linalg.norm(l, axis=1).max() + rr.max() for l, rr in zip(locals_, radii)])
    R, H = 0.06, 0.15
    pts = layered_packing(rng, diam, R, 0.0)
    q = random_unit_quaternions(rng, n_clumps)
    rmin = min(rr.min() for rr in radii)
    dt = 0.2 * rayleigh_dt(rmin, rho, MATERIAL["Ymod"], MATERIAL["Prat"])
    params = default_params(StepSize=dt, EndStep=steps, OutputInterval=steps,
                            Ymod=MATERIAL["Ymod"], Prat=MATERIAL["Prat"],
                            Frcoe=MATERIAL["Frcoe"] if mu is None else float(mu), NormRes=MATERIAL["NormRes"],
                            Thresh=0.2 * rmin, BranchLmtLen=96)
    top = min(2 * H, float(pts[:, 2].max() + 5 * diam.max())) if fit_box else 2 * H
    set_world_box(params, (-R, -R, 0.0), (R, R, top))
    K = n_clumps
    return assemble(params, pts, q, np.zeros((K, 3)), np.zeros((K, 3)), props,
                    locals_, radii, masses,
                    cylinder=make_cylinder(R, H, (0, 0, H)))


def tetra_scales(n_clumps: int = 50_000, seed: int = 20260828) -> np.ndarray:
    """The per-clump size scales make_cfg1 draws for (n_clumps, seed): the
    first draw of its generator."""
    return np.random.default_rng(seed).lognormal(0.0, 0.2, n_clumps)


def tetra_state_to_npz(scene: dict, scales: np.ndarray, path: str, **meta):
    """A compact snapshot of a scene of tetrahedral clumps (the cfg1 family):
    its parameters and walls, each clump's size scale, pose (FP64) and
    velocities (FP32), and the hierarchical-grid level of every subsphere.
    The members are rebuilt from the scales by the template, so the file
    stays a few MB for 50,000 clumps."""
    local, radius = _tetra_members(scales, 1e-3, 0.6, MATERIAL["rho"])[:2]
    if not (np.array_equal(np.concatenate(radius), scene["sub"]["radius"])
            and np.array_equal(np.concatenate(local), scene["sub"]["local"])):
        raise ValueError("scales do not rebuild the scene's members")
    flat = {}
    for k, v in scene["params"].items():
        flat["param/" + k] = np.array(v)
    for grp in ("cube", "cylinder"):
        if scene.get(grp) is not None:
            for k, v in scene[grp].items():
                flat[f"{grp}/{k}"] = np.array(v)
    c = scene["clump"]
    flat["clump/scale"] = np.asarray(scales, np.float64)
    flat["clump/pos"] = c["pos"]
    flat["clump/quat"] = c["quat"]
    flat["clump/vel"] = c["vel"].astype(np.float32)
    flat["clump/angvel"] = c["angvel"].astype(np.float32)
    lv = scene.get("levels")
    if lv is not None:
        flat["levels/level"] = np.asarray(lv["level"], np.uint8)
        flat["levels/cell"] = np.asarray(lv["cell"], np.float64)
    for k, v in meta.items():
        flat["meta/" + k] = np.array(v)
    np.savez_compressed(path, **flat)


def tetra_state_from_npz(path: str) -> dict:
    """The scene a tetra_state_to_npz snapshot holds: subsphere positions are
    the clump poses applied to the rebuilt members (X + C_bn(q) local)."""
    z = np.load(path)
    params = {}
    for k in z.files:
        if k.startswith("param/"):
            v = z[k]
            params[k[6:]] = v.item() if v.dtype.kind != "U" else str(v)
    scales = z["clump/scale"]
    locals_, radii, masses, props = _tetra_members(scales, 1e-3, 0.6, MATERIAL["rho"])
    grp = {}
    for g in ("cube", "cylinder"):
        keys = [k for k in z.files if k.startswith(g + "/")]
        if keys:
            grp[g] = {k.split("/", 1)[1]: (z[k].item() if z[k].ndim == 0 else z[k].copy()) for k in keys}
    sc = assemble(params, z["clump/pos"], z["clump/quat"], z["clump/vel"].astype(np.float64),
                  z["clump/angvel"].astype(np.float64), props, locals_, radii, masses,
                  cube=grp.get("cube"), cylinder=grp.get("cylinder"))
    if "levels/level" in z.files:
        sc["levels"] = {"level": z["levels/level"].astype(np.int32), "cell": z["levels/cell"].copy()}
    else:
        sc["levels"] = None
    sc["meta"] = {k[5:]: z[k].item() for k in z.files if k.startswith("meta/")}
    return sc


def make_cfg3(n_scenes: int = 256, seed: int = 20260828, steps: int = 20000, kmin: int = 500,
              kmax: int = 50_000) -> list:
    """The batched workload: n_scenes independent cfg1-style settling scenes,
    clump counts log-uniform in [kmin, kmax], friction uniform in [0.2, 0.8],
    scene s seeded with seed + s."""
    rng = np.random.default_rng(seed)
    ks = np.exp(rng.uniform(np.log(kmin), np.log(kmax), n_scenes)).astype(int)
    mus = rng.uniform(0.2, 0.8, n_scenes)
    return [make_cfg1(int(k), seed + s, steps, mu=float(m), fit_box=True) for s, (k, m) in enumerate(zip(ks, mus))]


def _poly_members(rng, n_clumps, rmin, rmax, max_members, rho):
    """Clumps of 1..max_members subspheres (uniform): a clump size r_c
    log-uniform in [rmin, rmax], member radii r_c x U(0.8, 1), centres at
    0.6 r_c in random directions; mass 0.8 x the spheres' and inertia
    0.4 M r_c^2 (a filled-clump approximation: the small test scenes use it,
    it needs no GPU)."""
    m = rng.integers(1, max_members + 1, n_clumps)
    rc = np.exp(rng.uniform(np.log(rmin), np.log(rmax), n_clumps))
    locals_, radii, masses, props, ext = [], [], [], [], np.zeros(n_clumps)
    for k in range(n_clumps):
        rr = rc[k] * rng.uniform(0.8, 1.0, m[k])
        if m[k] == 1:
            cen = np.zeros((1, 3))
        else:
            d = rng.normal(size=(m[k], 3))
            d /= np.linalg.norm(d, axis=1)[:, None]
            cen = d * (0.6 * rc[k])
            cen = cen - cen.mean(0)
        M = 0.8 * float(np.sum(rho * 4.0 / 3.0 * np.pi * rr ** 3))
        I = 0.4 * M * rc[k] ** 2
        locals_.append(cen)
        radii.append(rr)
        masses.append(np.full(m[k], M / m[k]))
        props.append([I, I, I, M])
        ext[k] = 2.0 * (np.linalg.norm(cen, axis=1).max() + rr.max())
    return locals_, radii, masses, np.array(props), ext



def _poly_templates(rng, n_clumps, rmin, rmax, max_members, rho, lam=0.5, samples=1 << 18):
    """The cfg2 / cfg4 clump templates: clumps of 1..max_members subspheres
    (uniform), every subsphere's radius log-uniform in [rmin, rmax]; the
    largest is the core and each other member sits on it in a uniformly
    random direction at centre distance |r_n - r_core| + 2 lam min(r_n,
    r_core): the reference's template builder (make_clump_template_lambda.m)
    places equal spheres at 2 r lambda, and for unequal ones this keeps the
    smaller sphere sticking out of the larger by the same fraction of its
    diameter (a compact clump, like the builder's ball and cross families,
    rather than a chain).  Mass, centre of mass
    and inertia of each union (overlap counted once) come from
    nbc.union_mass (the builder's Monte Carlo integration, on the GPU for all
    clumps at once); members are re-expressed in the clump's principal frame
    and the clump mass is split equally among them, as the builder does."""
    import nbc
    m = rng.integers(1, max_members + 1, n_clumps)
    start = np.concatenate([[0], np.cumsum(m)]).astype(np.int32)
    M = int(start[-1])
    r_all = np.exp(rng.uniform(np.log(rmin), np.log(rmax), M))
    d = rng.normal(size=(M, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    cen = np.zeros((M, 3))
    for k in range(n_clumps):
        b, e = start[k], start[k + 1]
        core = b + int(np.argmax(r_all[b:e]))
        rc, rr = r_all[core], r_all[b:e]
        dist = np.abs(rr - rc) + 2.0 * lam * np.minimum(rr, rc)
        cen[b:e] = dist[:, None] * d[b:e]
        cen[core] = 0.0
    vol, com, mom = nbc.union_mass(cen, r_all, start, samples=samples)
    mass = rho * vol
    inertia = (rho * vol)[:, None, None] * (np.trace(mom, axis1=1, axis2=2)[:, None, None] * np.eye(3) - mom)
    w, V = np.linalg.eigh(inertia)
    flip = np.linalg.det(V) < 0
    V[flip, :, 0] = -V[flip, :, 0]
    owner = np.repeat(np.arange(n_clumps), m)
    local = np.einsum("mi,mij->mj", cen - com[owner], V[owner])
    props = np.column_stack([w[:, 0], w[:, 1], w[:, 2], mass])
    locals_, radii, masses = [], [], []
    ext = np.zeros(n_clumps)
    for k in range(n_clumps):
        sl = slice(start[k], start[k + 1])
        locals_.append(local[sl])
        radii.append(r_all[sl])
        masses.append(np.full(m[k], mass[k] / m[k]))
        ext[k] = 2.0 * (np.linalg.norm(local[sl], axis=1) + r_all[sl]).max()
    return locals_, radii, masses, props, ext


def layered_packing_box(rng, diam, hx, hy, z0, jitter=0.02):
    """Clump centres in square-lattice layers inside [-hx, hx] x [-hy, hy],
    largest clumps first, each layer spaced by its largest diameter * 1.05."""
    order = np.argsort(-diam, kind="stable")
    pts = np.zeros((len(diam), 3))
    z, i = z0, 0
    while i < len(order):
        d = 1.05 * diam[order[i]]
        nx, ny = max(1, int(2 * hx / d)), max(1, int(2 * hy / d))
        gx = (np.arange(nx) - (nx - 1) / 2.0) * d
        gy = (np.arange(ny) - (ny - 1) / 2.0) * d
        X, Y = np.meshgrid(gx, gy, indexing="ij")
        xy = np.stack([X.ravel(), Y.ravel()], axis=1)
        take = order[i:i + len(xy)]
        sel = rng.permutation(len(xy))[:len(take)]
        pts[take, 0:2] = xy[sel] + rng.uniform(-jitter * d, jitter * d, (len(take), 2))
        pts[take, 2] = z + 0.5 * d
        z += d
        i += len(take)
    return pts


def make_poly_bed(n_sub, seed, half_xy, rmin=0.5e-3, rmax=5e-3, max_members=8, mu=0.5, steps=1000):
    """A polydisperse bed of about n_sub subspheres (clumps of 1..8, radii
    log-uniform in [rmin, rmax]) seeded in layers in a cube wall of half
    width half_xy, floor at z = 0, the wall and hashing box 1.5 x the seeded
    height tall; settling under gravity from rest."""
    rng = np.random.default_rng(seed)
    rho = MATERIAL["rho"]
    k = max(1, int(round(n_sub / (0.5 * (1 + max_members)))))
    locals_, radii, masses, props, ext = _poly_templates(rng, k, rmin, rmax, max_members, rho)
    pts = layered_packing_box(rng, ext, half_xy, half_xy, 0.0)
    top = float(pts[:, 2].max() + ext.max())
    H = 0.75 * top
    rs = np.concatenate(radii)
    dt = 0.2 * rayleigh_dt(float(rs.min()), rho, MATERIAL["Ymod"], MATERIAL["Prat"])
    params = default_params(StepSize=dt, EndStep=steps, OutputInterval=steps,
                            Ymod=MATERIAL["Ymod"], Prat=MATERIAL["Prat"], Frcoe=float(mu),
                            NormRes=MATERIAL["NormRes"], Thresh=0.2 * float(rs.min()), BranchLmtLen=96)
    set_world_box(params, (-half_xy, -half_xy, 0.0), (half_xy, half_xy, 2 * H))
    K = len(locals_)
    return assemble(params, pts, random_unit_quaternions(rng, K), np.zeros((K, 3)), np.zeros((K, 3)),
                    props, locals_, radii, masses, cube=make_cube((half_xy, half_xy, H), (0, 0, H)))


def with_sphere_intruder(scene, radius, speed, mu=None, xy=(0.0, 0.0), gap=0.0, mass=1.0, surface=None):
    """The scene with a sphere intruder of this radius above xy, its lowest
    point `gap` above the highest subsphere under it, driven down at a
    constant speed (the reference's constant_velocity motion).  With
    surface=q (a percentile) its lowest point rests that far above the q-th
    percentile of the subsphere tops under it instead: a settled bed keeps a
    few subspheres thrown up by the impacts of its fall, and the intruder
    should meet the bed, not them."""
    out = dict(scene)
    out["params"] = dict(scene["params"])
    if mu is not None:
        out["params"]["Frcoe"] = float(mu)
    pos, rad = scene["sub"]["pos"], scene["sub"]["radius"]
    if surface is None:
        z = _place_intruder_on_bed(pos, rad, xy, "sphere", radius, radius, -gap)
    else:
        under = np.hypot(pos[:, 0] - xy[0], pos[:, 1] - xy[1]) < radius + rad.max()
        z = float(np.percentile(pos[under, 2] + rad[under], surface)) + gap + radius
    I = 0.4 * mass * radius ** 2
    out["intruder"] = make_intruder("sphere", radius, (xy[0], xy[1], z), (0, 0, -float(speed)),
                                    prop=(I, I, I, mass), motion="constant_velocity")
    out["params"]["isIntruder"] = 1
    return out


def make_cfg2(n_sub: int = 1_000_000, seed: int = 20260828, steps: int = 56000, half_xy: float = 0.2) -> dict:
    """Polydisperse penetration bed: 1,000,000 subspheres in clumps of 1..8,
    radii log-uniform in [0.5, 5] mm, in a 0.4 x 0.4 m cube wall made tall
    enough for the seeded bed (the 0.3 m box of the configuration cannot hold
    these spheres); settle it, then add the 20 mm intruder with
    with_sphere_intruder(bed, 0.02, 0.1)."""
    return make_poly_bed(n_sub, seed, half_xy, steps=steps)


# ----------------------------------------------------------------------------
# small, contact-rich scenes for parity tests
# ----------------------------------------------------------------------------

def _place_intruder_on_bed(pos, radius, xy, shape, Ri, Hi, depth):
    """z of an intruder centred above xy whose lowest point overlaps the
    highest subsphere beneath it by `depth`."""
    d2 = (pos[:, 0] - xy[0]) ** 2 + (pos[:, 1] - xy[1]) ** 2
    if shape == "sphere":
        reach = np.sqrt(np.maximum((Ri + radius) ** 2 - d2, 0.0))
        cand = d2 < (Ri + radius) ** 2
        z = (pos[cand, 2] + reach[cand] - depth)
    else:
        cand = d2 < (Ri + radius) ** 2
        z = pos[cand, 2] + radius[cand] + Hi - depth
    return float(z.max())


def make_test_spheres(n=400, seed=1, r=1e-3, overlap=0.02, vel=0.5, angvel=200.0,
                      intruder="sphere", motion="constant_velocity", thresh_ratio=0.0003,
                      dt=2e-7, steps=30, wall="cube", bl=64):
    """Compressed lattice of one-sphere clumps: every neighbour pair overlaps by
    about `overlap`*r, random linear and angular velocities, walls and an
    intruder in contact from the first step, and a small Thresh so the
    contact list is rebuilt every few steps."""
    rng = np.random.default_rng(seed)
    rho = MATERIAL["rho"]
    nx = int(round(n ** (1 / 3))) + 1
    sp = 2 * r * (1 - overlap)
    lo = np.array([r * (1 - 2 * overlap)] * 3)
    pts = lattice_points(rng, n, sp, lo, nx, nx, 0.2 * overlap * r)
    hi = pts.max(0) + r * (1 - 2 * overlap)
    K = n
    m = rho * 4 / 3 * math.pi * r ** 3
    I = 0.4 * m * r * r
    params = default_params(StepSize=dt, EndStep=steps, OutputInterval=1,
                            Thresh=thresh_ratio * r, BranchLmtLen=bl)
    params["Cohesion"] = 0.0
    box_lo, box_hi = -0.5 * r * np.ones(3), hi + np.array([0.5 * r, 0.5 * r, 6 * r])
    set_world_box(params, box_lo, box_hi)
    cube = cyl = None
    if wall == "cube":
        cube = make_cube(0.5 * hi, 0.5 * hi)
    elif wall == "cylinder":
        c = 0.5 * hi
        cyl = make_cylinder(0.5 * max(hi[0], hi[1]) * 1.0, 0.5 * hi[2], c)
    intr = None
    if intruder is not None:
        xy = (0.5 * hi[0] + 0.3 * r, 0.5 * hi[1] - 0.2 * r)
        Ri, Hi = 3 * r, 2 * r
        rad = np.full(len(pts), r)
        z = _place_intruder_on_bed(pts, rad, xy, intruder, Ri, Hi, 0.25 * r)
        c = (xy[0], xy[1], z)
        if intruder == "sphere":
            intr = make_intruder("sphere", Ri, c, (0, 0, -0.5), prop=(1, 1, 1, 0.05),
                                 motion=motion)
        else:
            intr = make_intruder("cylinder", Ri, c, (0, 0, -0.5), half_height=Hi,
                                 prop=(1, 1, 1, 0.05), motion=motion)
    return assemble(params, pts, random_unit_quaternions(rng, K),
                    rng.uniform(-vel, vel, (K, 3)), rng.uniform(-angvel, angvel, (K, 3)),
                    np.tile([I, I, I, m], (K, 1)),
                    [np.zeros((1, 3))] * K, [np.array([r])] * K, [np.array([m])] * K,
                    cube=cube, cylinder=cyl, intruder=intr)


def make_test_sphere_levels(n_side=6, seed=43, R=1.5e-3, ratio=0.40, overlap=0.02, vel=0.5, angvel=200.0,
                            thresh_ratio=0.0003, dt=2e-7, steps=24, bl=64):
    """Spheres of two sizes on two grid levels, every sphere in contact: a
    compressed cubic lattice of radius-R spheres (neighbours overlap by about
    2 `overlap` R) and, in each lattice layer, a sphere of radius `ratio` R
    at the centre of every square of four, overlapping those four; a closed
    cylinder around the lattice whose caps and side press on the outer
    spheres.  The level table (coarse level 0 for the large spheres, cells
    of three radii) goes in scene["levels"]."""
    rng = np.random.default_rng(seed)
    rho = MATERIAL["rho"]
    a = 2 * R * (1 - overlap)
    g = np.arange(n_side) * a
    big = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    h = (g[:-1] + 0.5 * a)
    small = np.stack(np.meshgrid(h, h, g, indexing="ij"), -1).reshape(-1, 3)
    pts = np.concatenate([big, small]) + R
    rad = np.concatenate([np.full(len(big), R), np.full(len(small), ratio * R)])
    pts = pts + rng.uniform(-0.02 * overlap * R, 0.02 * overlap * R, pts.shape)
    K = len(pts)
    m = rho * 4 / 3 * math.pi * rad ** 3
    I = 0.4 * m * rad * rad
    centre = 0.5 * (pts.min(0) + pts.max(0))
    half_diag = math.sqrt(2) * 0.5 * (n_side - 1) * a
    cyl = make_cylinder(half_diag + R * (1 - overlap), 0.5 * (n_side - 1) * a + R * (1 - overlap), centre)
    params = default_params(StepSize=dt, EndStep=steps, OutputInterval=1, Thresh=thresh_ratio * ratio * R,
                            BranchLmtLen=bl)
    lo, hi = centre - (half_diag + 2 * R), centre + (half_diag + 2 * R)
    set_world_box(params, lo, hi)
    sc = assemble(params, pts, random_unit_quaternions(rng, K), rng.uniform(-vel, vel, (K, 3)),
                  rng.uniform(-angvel, angvel, (K, 3)), np.stack([I, I, I, m], 1),
                  [np.zeros((1, 3))] * K, [np.array([x]) for x in rad], [np.array([x]) for x in m],
                  cylinder=cyl)
    sc["levels"] = {"level": (rad < R).astype(np.int32), "cell": np.array([3 * R, 3 * ratio * R])}
    return sc


def make_test_split(n=343, seed=44, r=1e-3, offset=(0.05, 0.08), vel=3.0, angvel=200.0, dt=5e-6, steps=24,
                    kinds=(0.7, 0.15, 0.15), bl=64):
    """A compressed lattice of one-sphere clumps in a closed cylinder, away
    from the z axis (so that driven spheres move), with body kinds of the
    split driver drawn per sphere: free, driven at the prescribed velocity,
    fixed (scene["body_kind"]).  Free spheres move fast enough to pass a
    tenth of their radius within a few steps."""
    sc = make_test_spheres(n=n, seed=seed, r=r, vel=vel, angvel=angvel, intruder=None, dt=dt, steps=steps,
                           wall="cylinder", bl=bl)
    shift = np.array([offset[0], offset[1], 0.0])
    sc["sub"]["pos"] = sc["sub"]["pos"] + shift
    sc["clump"]["pos"] = sc["clump"]["pos"] + shift
    sc["cylinder"]["centre"] = sc["cylinder"]["centre"] + shift
    p = sc["params"]
    for a, k in enumerate("xyz"):
        p["WorldOrigin_" + k] += shift[a]
        p["BoxLowLmt_" + k] += shift[a]
        p["BoxUpLmt_" + k] += shift[a]
    rng = np.random.default_rng(seed + 1000)
    sc["body_kind"] = rng.choice(3, size=len(sc["clump"]["pos"]), p=list(kinds)).astype(np.int32)
    return sc


def make_test_tetra(n_clumps=120, seed=2, r=1e-3, squeeze=0.8, vel=0.5, angvel=200.0,
                    intruder="cylinder", motion="constant_velocity", thresh_ratio=0.0003,
                    dt=2e-7, steps=30, wall="cube", bl=96, sigma=0.15):
    """Tetrahedral clumps with random orientations packed closer than their
    extent (`squeeze` < 1) so many inter-clump pairs overlap."""
    rng = np.random.default_rng(seed)
    rho = MATERIAL["rho"]
    scales = rng.lognormal(0.0, sigma, n_clumps)
    locals_, radii, masses, props = _tetra_members(scales, r, 0.6, rho)
    rmed = r * float(np.median(scales))
    ext = 2 * 1.6 * rmed * squeeze
    nx = int(round(n_clumps ** (1 / 3))) + 1
    lo = np.array([0.5 * ext] * 3)
    pts = lattice_points(rng, n_clumps, ext, lo, nx, nx, 0.03 * ext)
    hi = pts.max(0) + 0.5 * ext
    params = default_params(StepSize=dt, EndStep=steps, OutputInterval=1,
                            Thresh=thresh_ratio * r, BranchLmtLen=bl)
    set_world_box(params, -0.5 * r * np.ones(3), hi + np.array([0.5 * r, 0.5 * r, 8 * r]))
    cube = cyl = None
    if wall == "cube":
        cube = make_cube(0.5 * hi, 0.5 * hi)
    elif wall == "cylinder":
        cyl = make_cylinder(0.5 * max(hi[0], hi[1]), 0.5 * hi[2], 0.5 * hi)
    intr = None
    K = n_clumps
    quats = random_unit_quaternions(rng, K)
    if intruder is not None:
        cid = np.repeat(np.arange(K), [len(m) for m in locals_])
        R = quat_to_body2world(quats)
        sub_pos = pts[cid] + np.einsum("nij,nj->ni", R[cid], np.concatenate(locals_))
        sub_r = np.concatenate(radii)
        xy = (0.5 * hi[0] + 0.3 * r, 0.5 * hi[1] - 0.2 * r)
        Ri, Hi = 3 * r, 2 * r
        z = _place_intruder_on_bed(sub_pos, sub_r, xy, intruder, Ri, Hi, 0.25 * r)
        c = (xy[0], xy[1], z)
        if intruder == "sphere":
            intr = make_intruder("sphere", Ri, c, (0, 0, -0.5), prop=(1, 1, 1, 0.05),
                                 motion=motion)
        else:
            intr = make_intruder("cylinder", Ri, c, (0, 0, -0.5), half_height=Hi,
                                 prop=(1, 1, 1, 0.05), motion=motion)
    return assemble(params, pts, quats,
                    rng.uniform(-vel, vel, (K, 3)), rng.uniform(-angvel, angvel, (K, 3)),
                    props, locals_, radii, masses, cube=cube, cylinder=cyl, intruder=intr)


# ----------------------------------------------------------------------------
# text formats of the reference
# ----------------------------------------------------------------------------

def _g(x) -> str:
    return repr(float(x))


def write_world_par(params: dict, path: str):
    with open(path, "w") as f:
        f.write("# written by nbody-clump_b200 scenegen\n")
        for k in PAR_KEYS:
            v = params[k]
            if isinstance(v, str):
                f.write(f"{k} = {v}\n")
            elif k in ("NumberBody", "ClumpNum", "BranchLmtLen", "EndStep", "StartStep",
                       "OutputInterval", "Update", "isIntruder", "isSelfGravity",
                       "isWallForce", "isQuaternion"):
                f.write(f"{k} = {int(v)}\n")
            else:
                f.write(f"{k} = {_g(v)}\n")


def write_reference_inputs(scene: dict, d: str):
    """Write world.par, ph/ch .bt and Rocks/*.bt into directory d, in the
    layouts the reference reads (src/dem_subsphere_io.cu:52-175,
    src/dem_clumpsphere_io.cu:46-48, src/dem_cube_wall_io.cu:43-48,
    src/dem_penetrator_io.cu:42-115, src/dem_cylind_wall_io.cu:41-49)."""
    os.makedirs(os.path.join(d, "Rocks"), exist_ok=True)
    p = scene["params"]
    write_world_par(p, os.path.join(d, "world.par"))
    s = scene["sub"]
    N = len(s["radius"])
    # per-clump local member index
    cid = s["clump_id"]
    first = np.zeros(N, dtype=np.int64)
    order = np.argsort(cid, kind="stable")
    starts = np.searchsorted(cid[order], cid[order])
    first[order] = np.arange(N) - starts
    with open(os.path.join(d, p["IniConFile"]), "w") as f:
        for i in range(N):
            f.write("%d %d %d %s %s %s %s %s %s %s %s\n" % (
                i, first[i], cid[i], *map(_g, s["pos"][i]), *map(_g, s["local"][i]),
                _g(s["mass"][i]), _g(s["radius"][i])))
    c = scene["clump"]
    with open(os.path.join(d, "ch.00000000.bt"), "w") as f:
        for k in range(len(c["pos"])):
            f.write("%d %s\n" % (k, " ".join(map(_g, np.concatenate(
                [c["pos"][k], c["vel"][k], c["quat"][k], c["angvel"][k], c["prop"][k]])))))
    cube = scene.get("cube")
    if cube is None:  # the reference always reads a cube file; write an inert one
        cube = make_cube((1e3, 1e3, 1e3), (0, 0, 0))
    with open(os.path.join(d, "Rocks", "CubeWall.bt"), "w") as f:
        f.write(" ".join(map(_g, cube["half"])) + "\n")
        f.write(" ".join(map(_g, cube["centre"])) + "\n")
        f.write(" ".join(map(_g, cube["vel"])) + "\n")
        f.write(" ".join(map(_g, cube["quat"])) + "\n")
        f.write(" ".join(map(_g, cube["angvel"])) + "\n")
    cyl = scene.get("cylinder")
    if cyl is not None:
        with open(os.path.join(d, "Rocks", "CylindWall.bt"), "w") as f:
            f.write(f"{_g(cyl['radius'])} {_g(cyl['half_height'])}\n")
            f.write(" ".join(map(_g, cyl["axis"])) + "\n")
            f.write(" ".join(map(_g, cyl["prop"])) + "\n")
            f.write(" ".join(map(_g, cyl["centre"])) + "\n")
            f.write(" ".join(map(_g, cyl["vel"])) + "\n")
            f.write(" ".join(map(_g, cyl["quat"])) + "\n")
            f.write(" ".join(map(_g, cyl["angvel"])) + "\n")
    it = scene.get("intruder")
    if it is None:  # inert intruder far away (the reference always reads one)
        it = make_intruder("sphere", 1e-3, (1e3, 1e3, 1e3), (0, 0, 0))
    with open(os.path.join(d, "Rocks", "Penetrator.bt"), "w") as f:
        if it["shape"] == "sphere":
            f.write(f"sphere {_g(it['radius'])}\n")
        else:
            f.write(f"cylinder {_g(it['radius'])} {_g(it['half_height'])} "
                    + " ".join(map(_g, it["axis"])) + "\n")
        f.write(" ".join(map(_g, it["prop"])) + "\n")
        f.write(" ".join(map(_g, it["pos"])) + "\n")
        f.write(" ".join(map(_g, it["vel"])) + "\n")
        f.write(" ".join(map(_g, it["quat"])) + "\n")
        f.write(" ".join(map(_g, it["angvel"])) + "\n")
        f.write(f"motion {it['motion']}\n")


SPHERE_DRIVER_MODE = {"cylinder": 1 | 4, "cube": 1 | 2, "split": 1 | 4, "hgrid": 1}


def as_sphere_driver(scene: dict, driver: str) -> dict:
    """The scene as the sphere-only driver `driver` runs it (nbc.SPHERE_DRIVERS):
    the driver's NBC_SPHERE_* bits, its wall, and the split driver's body kinds
    (scene["body_kind"]) or the hgrid driver's level table (scene["levels"])."""
    sc = dict(scene)
    sc["sphere_mode"] = SPHERE_DRIVER_MODE[driver]
    sc["params"] = dict(scene["params"], isWallForce=1)
    if driver != "split":
        sc.pop("body_kind", None)
    if driver != "hgrid":
        sc.pop("levels", None)
    return sc


def write_sphere_inputs(scene: dict, d: str, driver: str = "cylinder"):
    """A working directory for the reference's sphere-only drivers (class
    DEMmain): world.par, the 21-column ph file (id, id, Type, pos, vel, quat,
    angular velocity, Ixx Iyy Izz M, radius; src/dem_io.cu:183-185), Rocks/
    (the driver's wall file and Penetrator.bt, which every driver reads) and,
    for the hgrid driver, grid.bt (id, cell size, cells per axis, first cell,
    id per level; src/dem_io.cu:204-248).  The scene holds one-sphere clumps
    at their centres with sphere k = clump k; Type is the grid level (hgrid),
    the body kind (split) or 0."""
    s, c = scene["sub"], scene["clump"]
    K = len(c["pos"])
    if len(s["radius"]) != K or np.abs(s["local"]).max() != 0.0 or np.any(s["clump_id"] != np.arange(K)):
        raise ValueError("the sphere drivers take one-sphere clumps at their centres, sphere k = clump k")
    p = dict(scene["params"])
    typ = np.zeros(K, dtype=np.int64)
    lv = scene.get("levels")
    cells = [3.0 * float(np.max(s["radius"]))]
    if driver == "hgrid" and lv is not None:
        typ = np.asarray(lv["level"], dtype=np.int64)
        cells = [float(x) for x in lv["cell"]]
    if driver == "split":
        typ = np.asarray(scene["body_kind"], dtype=np.int64)
    p["GridLevels"] = len(cells) if driver == "hgrid" else p.get("GridLevels", 1)
    write_reference_inputs(dict(scene, params=p), d)
    with open(os.path.join(d, p["IniConFile"]), "w") as f:
        for k in range(K):
            cols = np.concatenate([c["pos"][k], c["vel"][k], c["quat"][k], c["angvel"][k], c["prop"][k],
                                   [s["radius"][k]]])
            f.write("%d %d %d %s\n" % (k, k, typ[k], " ".join(_g(v) for v in cols)))
    if driver == "hgrid":
        with open(os.path.join(d, "grid.bt"), "w") as f:
            off = 0
            for l, cell in enumerate(cells):
                n = [int(math.ceil(p["WorldSize_" + a] / cell)) for a in "xyz"]
                f.write("%d %s %d %d %d %d %d\n" % (l, _g(cell), n[0], n[1], n[2], off, l))
                off += n[0] * n[1] * n[2]


def read_reference_inputs(d: str) -> dict:
    """Read a reference working directory (world.par, ph/ch .bt, Rocks/) into
    a scene dict; the inverse of write_reference_inputs."""
    params = {}
    with open(os.path.join(d, "world.par")) as f:
        for line in f:
            core = line.split("#", 1)[0].replace("\t", "").replace(" ", "").strip()
            if not core:
                continue
            k, v = core.split("=", 1)
            params[k] = v
    for k in list(params):
        if k not in ("BodyFileDir", "IniConFile"):
            params[k] = float(params[k])
    for k in ("NumberBody", "ClumpNum", "BranchLmtLen", "EndStep", "StartStep",
              "OutputInterval", "Update", "isIntruder", "isSelfGravity", "isWallForce",
              "isQuaternion"):
        params[k] = int(params[k])
    N, K = params["NumberBody"], params["ClumpNum"]
    ph = np.loadtxt(os.path.join(d, params["IniConFile"]), ndmin=2)[:N]
    ch = np.loadtxt(os.path.join(d, "ch.00000000.bt"), ndmin=2)[:K]
    sub = {"clump_id": ph[:, 2].astype(np.int32), "pos": ph[:, 3:6].copy(),
           "local": ph[:, 6:9].copy(), "mass": ph[:, 9].copy(), "radius": ph[:, 10].copy()}
    clump = {"pos": ch[:, 1:4].copy(), "vel": ch[:, 4:7].copy(), "quat": ch[:, 7:11].copy(),
             "angvel": ch[:, 11:14].copy(), "prop": ch[:, 14:18].copy()}
    cw = np.array(open(os.path.join(d, "Rocks", "CubeWall.bt")).read().split(), float)
    cube = make_cube(cw[0:3], cw[3:6], cw[6:9], cw[13:16], cw[9:13])
    tok = open(os.path.join(d, "Rocks", "Penetrator.bt")).read().split()
    shape = tok[0].lower()
    if shape == "sphere":
        radius, hh, axis, rest = float(tok[1]), float(tok[1]), (0, 0, 1.0), tok[2:]
    else:
        off = 1 if shape == "cylinder" else 0
        vals = tok[off:]
        radius, hh, axis, rest = float(vals[0]), float(vals[1]), tuple(map(float, vals[2:5])), vals[5:]
        shape = "cylinder"
    num = list(map(float, rest[:17]))  # property(4) pos(3) vel(3) quat(4) angvel(3)
    motion = "constant_velocity"
    if len(rest) > 18 and rest[17].lower() == "motion":
        motion = rest[18].lower()
        if motion in ("constant", "kinematic"):
            motion = "constant_velocity"
        elif motion == "dynamic":
            motion = "gravity"
    intr = make_intruder(shape, radius, num[4:7], num[7:10], half_height=hh, axis=axis,
                         prop=num[0:4], quat=num[10:14], angvel=num[14:17], motion=motion)
    cyl = None
    cpath = os.path.join(d, "Rocks", "CylindWall.bt")
    if os.path.exists(cpath):
        cv = np.array(open(cpath).read().split(), float)
        cyl = make_cylinder(cv[0], cv[1], cv[9:12], cv[2:5], cv[5:9], cv[12:15], cv[19:22], cv[15:19])
    return {"params": params, "sub": sub, "clump": clump,
            "cube": cube if params["isWallForce"] else cube,
            "cylinder": None, "intruder": intr if params["isIntruder"] else None,
            "cylinder_file": cyl}


# ----------------------------------------------------------------------------
# npz round trip of a scene (golden fixtures and bench inputs)
# ----------------------------------------------------------------------------

def scene_to_npz(scene: dict, path: str):
    flat = {}
    for k, v in scene["params"].items():
        flat["par/" + k] = np.array(v)
    for grp in ("sub", "clump"):
        for k, v in scene[grp].items():
            flat[f"{grp}/{k}"] = np.asarray(v)
    for grp in ("cube", "cylinder", "intruder", "levels"):
        if scene.get(grp) is not None:
            for k, v in scene[grp].items():
                flat[f"{grp}/{k}"] = np.asarray(v)
    for k in ("sphere_mode", "body_kind"):
        if scene.get(k) is not None:
            flat["extra/" + k] = np.asarray(scene[k])
    np.savez_compressed(path, **flat)


def scene_from_npz(path: str) -> dict:
    z = np.load(path, allow_pickle=False)
    scene = {"params": {}, "sub": {}, "clump": {}, "cube": None, "cylinder": None,
             "intruder": None}
    for key in z.files:
        grp, k = key.split("/", 1)
        v = z[key]
        if grp == "par":
            v = v.item() if v.shape == () else v
            if isinstance(v, (np.integer, int)):
                v = int(v)
            elif isinstance(v, (np.floating, float)):
                v = float(v)
            elif isinstance(v, (np.str_, str)):
                v = str(v)
            scene["params"][k] = v
        elif grp == "extra":
            scene[k] = v.item() if v.shape == () else v
        else:
            if scene.get(grp) is None:
                scene[grp] = {}
            if v.shape == ():
                v = v.item()
                if isinstance(v, np.str_):
                    v = str(v)
            scene[grp][k] = v
    return scene


def _cyl_wall_sphere_sites(rng, r, Rc, H, spacing, n_side, n_cap, n_interior):
    """Sphere centres (relative to the cylinder centre, axis z) for a closed
    cylinder of radius Rc and half-height H: n_cap on each cap, n_side on
    the side, a ring at each cap edge, and n_interior clear of every wall.
    Returns (centres, kind) with kind 0 bottom cap, 1 top cap, 2 side,
    3 bottom edge, 4 top edge, 5 interior; the overlap with the wall is
    drawn later per sphere.  Sites are at least `spacing` apart."""
    sites, kind = [], []

    def put(p, k):
        if all(np.linalg.norm(p - q) >= spacing for q in sites):
            sites.append(p)
            kind.append(k)
            return True
        return False

    for k in (3, 4):  # edge rings
        n = int(2 * math.pi * (Rc - r) / spacing)
        for j in range(n):
            a = 2 * math.pi * (j + 0.5 * (k - 3)) / n
            put(np.array([(Rc - r) * math.cos(a), (Rc - r) * math.sin(a), (-1 if k == 3 else 1) * (H - r)]), k)
    for k, cnt in ((0, n_cap), (1, n_cap), (2, n_side), (5, n_interior)):
        placed, tries = 0, 0
        while placed < cnt and tries < 200 * cnt:
            tries += 1
            if k in (0, 1):
                rho, a = (Rc - 3 * r) * math.sqrt(rng.random()), 2 * math.pi * rng.random()
                p = np.array([rho * math.cos(a), rho * math.sin(a), (-1 if k == 0 else 1) * (H - r)])
            elif k == 2:
                a, z = 2 * math.pi * rng.random(), rng.uniform(-(H - 3 * r), H - 3 * r)
                p = np.array([(Rc - r) * math.cos(a), (Rc - r) * math.sin(a), z])
            else:
                rho, a = (Rc - 3.5 * r) * math.sqrt(rng.random()), 2 * math.pi * rng.random()
                p = np.array([rho * math.cos(a), rho * math.sin(a), rng.uniform(-(H - 3.5 * r), H - 3.5 * r)])
            placed += put(p, k)
    return np.array(sites), np.array(kind)


def make_test_cyl(kind="spheres", seed=31, r=1e-3, Rc=12e-3, H=9e-3, overlap=(0.005, 0.04), vel=0.2,
                  angvel=300.0, dt=2e-6, steps=24, thresh_ratio=3e-4, bl=64, sigma=0.1, squeeze=0.8):
    """Clumps in a closed cylinder wall (axis z) in contact with its bottom
    cap, top cap, side and both cap edges from the first step.

    kind "spheres": one-sphere clumps (LocalPos = 0, radius r x LogNormal(0,
    sigma) clipped to [0.8, 1.25] r) at least 2.6 r_max apart, so the only
    contacts are with the wall: the scene the reference's sphere-only driver
    runs (its cylinder wall, src/dem_force_cylind_wall.cu:152-237) and the
    clump path must match.  Each sphere on a wall site is pushed into the
    wall by overlap x r (uniform in the given range; at an edge into both),
    random linear and angular velocities stretch, break and make wall
    contacts over the run, and a small Thresh rebuilds the list every few
    steps.

    kind "tetra": tetrahedral clumps on a lattice clipped to the cylinder,
    packed closer than their extent (inter-clump contacts); every clump of
    the outer ring, the top layer and the bottom layer is moved until its
    farthest subsphere presses into the wall by overlap x r, so the side,
    both caps and the rings where they meet carry contacts."""
    rng = np.random.default_rng(seed)
    rho = MATERIAL["rho"]
    if kind == "spheres":
        rmax = 1.25 * r
        sites, skind = _cyl_wall_sphere_sites(rng, rmax, Rc, H, 2.6 * rmax, 16, 12, 12)
        K = len(sites)
        rad = r * np.clip(np.exp(sigma * rng.standard_normal(K)), 0.8, 1.25)
        ov = rng.uniform(overlap[0], overlap[1], (K, 2)) * rad[:, None]
        pts = sites.copy()
        for i in range(K):
            ri, k = rad[i], skind[i]
            rho_xy = math.hypot(pts[i, 0], pts[i, 1])
            if k in (0, 3):
                pts[i, 2] = -(H - ri + ov[i, 0])
            elif k in (1, 4):
                pts[i, 2] = H - ri + ov[i, 0]
            if k in (2, 3, 4):
                f = (Rc - ri + ov[i, 1]) / rho_xy
                pts[i, 0] *= f
                pts[i, 1] *= f
        m = rho * 4 / 3 * math.pi * rad ** 3
        I = 0.4 * m * rad ** 2
        props = np.stack([I, I, I, m], axis=1)
        locals_ = [np.zeros((1, 3))] * K
        radii = [np.array([x]) for x in rad]
        masses = [np.array([x]) for x in m]
        rmin = float(rad.min())
        quats = random_unit_quaternions(rng, K)
    elif kind == "tetra":
        n_side = 6
        scales = rng.lognormal(0.0, sigma, 4 * n_side ** 3)
        rmed = r * float(np.median(scales))
        ext = 2 * 1.6 * rmed * squeeze
        g = (np.arange(n_side) - (n_side - 1) / 2.0) * ext
        gx, gy, gz = np.meshgrid(g, g, g, indexing="ij")
        keep = gx ** 2 + gy ** 2 <= (g.max() + 1e-12) ** 2
        pts = np.stack([gx[keep], gy[keep], gz[keep]], axis=1)
        pts = pts + rng.uniform(-0.03 * ext, 0.03 * ext, pts.shape)
        K = len(pts)
        scales = scales[:K]
        locals_, radii, masses, props = _tetra_members(scales, r, 0.6, rho)
        quats = random_unit_quaternions(rng, K)
        Rm = quat_to_body2world(quats)
        cid = np.repeat(np.arange(K), 4)
        arm = np.einsum("nij,nj->ni", Rm[cid], np.concatenate(locals_))
        sr = np.concatenate(radii)
        rho_k = np.hypot(pts[:, 0], pts[:, 1])
        Rc = float(rho_k.max() + 1.4 * rmed)
        H = float(np.abs(pts[:, 2]).max() + 1.4 * rmed)
        dl = rng.uniform(overlap[0], overlap[1], (K, 2)) * r
        zmax = np.abs(pts[:, 2]).max()
        for k in range(K):
            sub = slice(4 * k, 4 * k + 4)
            if rho_k[k] > rho_k.max() - 0.5 * ext:
                u = pts[k, :2] / rho_k[k]
                reach = np.max((pts[k, :2] + arm[sub, :2]) @ u + sr[sub])
                pts[k, :2] += (Rc - reach + dl[k, 0]) * u
            if abs(pts[k, 2]) > zmax - 0.5 * ext:
                sgn = 1.0 if pts[k, 2] > 0 else -1.0
                reach = np.max(sgn * (pts[k, 2] + arm[sub, 2]) + sr[sub])
                pts[k, 2] += sgn * (H - reach + dl[k, 1])
        rmin = r * float(scales.min())
        rmax = r * float(scales.max())
    else:
        raise ValueError(kind)
    c = np.array([Rc + 2 * rmax, Rc + 2 * rmax, H + 2 * rmax])
    params = default_params(StepSize=dt, EndStep=steps, OutputInterval=1, Thresh=thresh_ratio * rmin,
                            BranchLmtLen=bl)
    set_world_box(params, np.zeros(3), 2 * c)
    return assemble(params, pts + c, quats, rng.uniform(-vel, vel, (K, 3)), rng.uniform(-angvel, angvel, (K, 3)),
                    props, locals_, radii, masses, cylinder=make_cylinder(Rc, H, c))


def make_test_converging(n_side=8, seed=5, r=1e-3, loose=1.6, shrink=0.45, steps=1500, sigma=0.15):
    """Tetrahedral clumps on a loose lattice (spacing `loose` x their extent, so
    the first list holds little more than the pairs inside clumps), moving
    towards the centre with a uniform compression rate that would shrink the
    lattice by `shrink` over `steps` steps: the list grows several-fold
    after the first step.  No walls, no gravity."""
    rng = np.random.default_rng(seed)
    rho = MATERIAL["rho"]
    K = n_side ** 3
    scales = rng.lognormal(0.0, sigma, K)
    locals_, radii, masses, props = _tetra_members(scales, r, 0.6, rho)
    rmed = r * float(np.median(scales))
    sp = 2 * 1.6 * rmed * loose
    lo = np.array([0.5 * sp] * 3)
    pts = lattice_points(rng, K, sp, lo, n_side, n_side, 0.03 * sp)
    hi = pts.max(0) + 0.5 * sp
    dt = 0.2 * rayleigh_dt(r * float(scales.min()), rho, MATERIAL["Ymod"], MATERIAL["Prat"])
    rate = shrink / (steps * dt)
    centre = 0.5 * (pts.min(0) + pts.max(0))
    vel = -rate * (pts - centre)
    params = default_params(StepSize=dt, EndStep=steps, OutputInterval=steps, Thresh=0.2 * r,
                            BranchLmtLen=96, Gravity=0.0,
                            **{k: v for k, v in MATERIAL.items() if k != "rho"})
    set_world_box(params, -4 * sp * np.ones(3), hi + 4 * sp)
    return assemble(params, pts, random_unit_quaternions(rng, K), vel,
                    rng.uniform(-50.0, 50.0, (K, 3)), props, locals_, radii, masses)


def make_test_poly(n_clumps=150, seed=3, rmin=0.5e-3, rmax=2.5e-3, max_members=3, vel=0.5, angvel=200.0,
                   intruder="sphere", motion="constant_velocity", thresh_ratio=0.0003, dt=1e-7, steps=24,
                   wall="cube", bl=256):
    """Polydisperse clumps (1..max_members subspheres, radii log-uniform in
    [rmin, rmax]) on a lattice sized by the median clump, so large clumps
    overlap their neighbours: a contact-rich scene for hierarchical grids."""
    rng = np.random.default_rng(seed)
    rho = MATERIAL["rho"]
    locals_, radii, masses, props = [], [], [], []
    for k in range(n_clumps):
        m = int(rng.integers(1, max_members + 1))
        rr = np.exp(rng.uniform(np.log(rmin), np.log(rmax), m))
        if m == 1:
            cen = np.zeros((1, 3))
        else:
            d = rng.normal(size=(m, 3))
            d /= np.linalg.norm(d, axis=1)[:, None]
            cen = d * (0.6 * rr.min())
        cen = cen - cen.mean(0)
        M = float(np.sum(rho * 4.0 / 3.0 * np.pi * rr ** 3)) * 0.8
        I = 0.4 * M * float(np.max(rr)) ** 2
        locals_.append(cen)
        radii.append(rr)
        masses.append(np.full(m, M / m))
        props.append([I, I, I, M])
    props = np.array(props)
    ext = 2.0 * np.median([np.linalg.norm(c, axis=1).max() + r.max() for c, r in zip(locals_, radii)])
    nx = int(round(n_clumps ** (1 / 3))) + 1
    pts = lattice_points(rng, n_clumps, ext, np.full(3, 0.5 * ext), nx, nx, 0.03 * ext)
    hi = pts.max(0) + 0.5 * ext
    params = default_params(StepSize=dt, EndStep=steps, OutputInterval=1, Thresh=thresh_ratio * rmin,
                            BranchLmtLen=bl)
    set_world_box(params, -rmax * np.ones(3), hi + np.array([rmax, rmax, 6 * rmax]))
    cube = make_cube(0.5 * hi, 0.5 * hi) if wall == "cube" else None
    cyl = make_cylinder(0.5 * max(hi[0], hi[1]), 0.5 * hi[2], 0.5 * hi) if wall == "cylinder" else None
    K = n_clumps
    quats = random_unit_quaternions(rng, K)
    intr = None
    if intruder is not None:
        cid = np.repeat(np.arange(K), [len(m) for m in locals_])
        R = quat_to_body2world(quats)
        sub_pos = pts[cid] + np.einsum("nij,nj->ni", R[cid], np.concatenate(locals_))
        xy = (0.5 * hi[0], 0.5 * hi[1])
        z = _place_intruder_on_bed(sub_pos, np.concatenate(radii), xy, intruder, 3 * rmax, 2 * rmax, 0.2 * rmin)
        intr = make_intruder(intruder, 3 * rmax, (xy[0], xy[1], z), (0, 0, -0.5), half_height=2 * rmax,
                             prop=(1, 1, 1, 0.05), motion=motion)
    return assemble(params, pts, quats, rng.uniform(-vel, vel, (K, 3)), rng.uniform(-angvel, angvel, (K, 3)),
                    props, locals_, radii, masses, cube=cube, cylinder=cyl, intruder=intr)

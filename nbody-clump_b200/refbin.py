"""Readers and writers for the reference's raw binary snapshot files.

All files are native little-endian field blocks with no header and no padding
(``src/dem_binary_io.h:17-25``); names are ``dir/prefix.%08d.bin`` with the
completed step number (``src/dem_binary_io.h:47-55``).

    OutPart/ph.N.bin   int32 n; int32[n] sorted id; int32[n] original id;
                       int32[n] clump id; f64[n,3] pos; f64[n,3] local;
                       f64[n] mass; f64[n] radius   (src/dem_subsphere_io.cu:262-274)
    OutClump/ch.N.bin  int32 c; int32[c] id (intruder -1 first); then the
                       blocks pos f64[c,3], vel f64[c,3], quat f64[c,4],
                       angvel f64[c,3], property f64[c,4]   (src/dem_binary_io.h:148-180)
    OutForce/fc.N.bin  int32 n; int32[n] sample; f64[n,3] force; f64[n,3] torque
                       (src/dem_binary_io.h:123-144)
    OutForce/yi.N.bin  int32 c; int32[c] clump id; f64[c,3] Fn, Ft, Tn, Tt
                       (src/dem_subsphere_io.cu:279-303)
    OutCnt/{Nei,Fcn,Cpt}.N.bin  int32 n; int32 bl; then n x bl int32 / f64x3
                       rows (src/dem_binary_io.h:100-121)

The sphere-only drivers (class DEMmain) write their own particle file:

    OutPart/ph.N.bin   int32 n; int32[n] sorted id; int32[n] original id;
                       int32[n] Type; f64[n,3] pos; f64[n,3] vel; f64[n,4] quat;
                       f64[n,3] angvel; f64[n,4] property; f64[n] radius
                       (src/dem_io.cu:313-329)
    OutPart/intruder.N.bin  the OutClump/ch layout with the intruder alone
                       (src/dem_io.cu:331-342)
"""
from __future__ import annotations

import os

import numpy as np


def file_name(directory: str, prefix: str, step: int) -> str:
    return os.path.join(directory, "%s.%08d.bin" % (prefix, step))


def _reader(path):
    with open(path, "rb") as f:
        return memoryview(f.read())


class _Cursor:
    def __init__(self, path):
        self.buf = _reader(path)
        self.off = 0

    def take(self, dtype, count, shape=None):
        dt = np.dtype(dtype)
        n = int(count) * dt.itemsize
        a = np.frombuffer(self.buf[self.off:self.off + n], dtype=dt, count=int(count))
        self.off += n
        if shape is not None:
            a = a.reshape(shape)
        return a.copy()

    def done(self):
        return self.off == len(self.buf)


def read_ph(path):
    c = _Cursor(path)
    n = int(c.take("<i4", 1)[0])
    out = {"sorted_id": c.take("<i4", n), "part_fix": c.take("<i4", n),
           "clump_id": c.take("<i4", n), "pos": c.take("<f8", 3 * n, (n, 3)),
           "local": c.take("<f8", 3 * n, (n, 3)), "mass": c.take("<f8", n),
           "radius": c.take("<f8", n)}
    assert c.done(), path
    return out


def read_sphere_ph(path):
    c = _Cursor(path)
    n = int(c.take("<i4", 1)[0])
    out = {"sorted_id": c.take("<i4", n), "part_fix": c.take("<i4", n), "type": c.take("<i4", n),
           "pos": c.take("<f8", 3 * n, (n, 3)), "vel": c.take("<f8", 3 * n, (n, 3)),
           "quat": c.take("<f8", 4 * n, (n, 4)), "angvel": c.take("<f8", 3 * n, (n, 3)),
           "prop": c.take("<f8", 4 * n, (n, 4)), "radius": c.take("<f8", n)}
    assert c.done(), path
    return out


def read_ch(path):
    c = _Cursor(path)
    n = int(c.take("<i4", 1)[0])
    out = {"id": c.take("<i4", n), "pos": c.take("<f8", 3 * n, (n, 3)),
           "vel": c.take("<f8", 3 * n, (n, 3)), "quat": c.take("<f8", 4 * n, (n, 4)),
           "angvel": c.take("<f8", 3 * n, (n, 3)), "prop": c.take("<f8", 4 * n, (n, 4))}
    assert c.done(), path
    return out


def read_fc(path):
    c = _Cursor(path)
    n = int(c.take("<i4", 1)[0])
    out = {"sample": c.take("<i4", n), "force": c.take("<f8", 3 * n, (n, 3)),
           "torque": c.take("<f8", 3 * n, (n, 3))}
    assert c.done(), path
    return out


def read_yi(path):
    c = _Cursor(path)
    n = int(c.take("<i4", 1)[0])
    out = {"clump_id": c.take("<i4", n)}
    for k in ("fn", "ft", "tn", "tt"):
        out[k] = c.take("<f8", 3 * n, (n, 3))
    assert c.done(), path
    return out


def read_cnt(path, dtype):
    c = _Cursor(path)
    n = int(c.take("<i4", 1)[0])
    bl = int(c.take("<i4", 1)[0])
    if dtype == "3f8":
        a = c.take("<f8", 3 * n * bl, (n, bl, 3))
    else:
        a = c.take(dtype, n * bl, (n, bl))
    assert c.done(), path
    return a


# ----------------------------------------------------------------------------
# writers (same byte layout)
# ----------------------------------------------------------------------------

def _w(f, a, dtype):
    np.ascontiguousarray(a, dtype=dtype).tofile(f)


def write_ph(path, sorted_id, part_fix, clump_id, pos, local, mass, radius):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    n = len(part_fix)
    with open(path, "wb") as f:
        _w(f, [n], "<i4")
        _w(f, sorted_id, "<i4")
        _w(f, part_fix, "<i4")
        _w(f, clump_id, "<i4")
        _w(f, pos, "<f8")
        _w(f, local, "<f8")
        _w(f, mass, "<f8")
        _w(f, radius, "<f8")


def write_ch(path, pos, vel, quat, angvel, prop, intruder=None):
    """intruder: None or dict with pos, vel, quat, angvel (stored first, id -1,
    zero property)."""
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    k = len(pos)
    c = k + (1 if intruder is not None else 0)
    ids = np.arange(k, dtype=np.int32)
    if intruder is not None:
        ids = np.concatenate([[-1], ids]).astype(np.int32)
    with open(path, "wb") as f:
        _w(f, [c], "<i4")
        _w(f, ids, "<i4")
        for key, arr, width in (("pos", pos, 3), ("vel", vel, 3), ("quat", quat, 4),
                                ("angvel", angvel, 3)):
            if intruder is not None:
                _w(f, np.asarray(intruder[key]).reshape(1, width), "<f8")
            _w(f, arr, "<f8")
        if intruder is not None:
            _w(f, np.zeros((1, 4)), "<f8")
        _w(f, prop, "<f8")

"""The C oracle against an independent pure-Python restatement of the reference's
VoxelConstrainedSphere path, on small seeded tracks (CPU only); and the oracle's FP32 geometry
variant against a numpy float32 restatement of it.

The restatement follows the reference directly: geometry (SphericalGeometry.cu:7-32), z-origin
shift (VoxelConstrainedSphereMethod.cu:138-154), XY shift and strict box test (:176-177, :198),
lattice index llrint(a/d) and the sphere test summed x -> y -> z (:249-258, :271), key and value
(:301-322), reduce-by-key and the [lo, hi) bin rule (Histogram.cu:150-158). Per-sphere sums are
taken as the correctly rounded exact sum (math.fsum) and as the left-to-right sum in deposit
order. Every sphere record of the oracle (key, hits, both sums, bin) must match exactly.
"""
import math

import numpy as np
import pytest

import pyoracle as po

U64 = 1 << 64
ZSHIFT = {"plus": 1.0, "minus": -1.0, "none": 0.0}


def py_geometry(hl, d):
    n = math.floor(2.0 * hl / d)
    length = n * d
    half = length / 2.0
    r = d / 2.0
    gso = -half + r
    if r > half:
        half, n = r, 1
    return {"N": n, "HL": half, "gSO": gso, "d": d, "r": r}


def py_job(x, y, z, edep, hl, d, zshift, sxsy, edges, rnd=round, inside=lambda a, b: a <= b):
    g = py_geometry(hl, d)
    hlp, gso, n, r2 = g["HL"], g["gSO"], g["N"], g["r"] * g["r"]
    lineal = (2.0 / 3.0) * d
    zs = [float(v) + ZSHIFT[zshift] * hlp for v in z]
    records = []
    for os_, (sx, sy) in enumerate(sxsy):
        spheres = {}
        for i in range(len(x)):
            xs, ys = float(x[i]) + sx, float(y[i]) + sy
            if not (abs(xs) < hlp and abs(ys) < hlp and abs(zs[i]) < hlp):
                continue
            a = (xs - gso, ys - gso, zs[i] - gso)
            k = [rnd(v / d) for v in a]                # llrint: round half to even
            dx, dy, dz = (float(kk) * d - v for kk, v in zip(k, a))
            if inside(dx * dx + dy * dy + dz * dz, r2):
                key = (k[0] + k[1] * n + k[2] * n * n) % U64
                spheres.setdefault(key, []).append(float(edep[i]) / lineal)
        for key in sorted(spheres):
            vals = spheres[key]
            seq = vals[0]
            for v in vals[1:]:
                seq = seq + v
            yx = math.fsum(vals)
            b = int(np.searchsorted(edges, yx, side="right")) - 1
            records.append((os_, key, len(vals), yx, seq, b if 0 <= b < len(edges) - 1 else -1))
    return g, records


def _cases():
    rs = np.random.default_rng(11)
    out = []
    # scattered deposits in and around the voxel, shifts on
    for hl, d, zs in ((50.0, 10.0, "none"), (50.0, 3.0, "plus"), (40.0, 7.0, "minus")):
        n = 160
        x = rs.uniform(-1.3 * hl, 1.3 * hl, n)
        y = rs.uniform(-1.3 * hl, 1.3 * hl, n)
        z = rs.uniform(-2.3 * hl, 2.3 * hl, n)        # the z-origin shift moves some inside
        e = rs.lognormal(3.0, 1.0, n)
        out.append((f"scatter-d{d}-{zs}", x, y, z, e, hl, d, zs, True))
    # clustered deposits: several hits per sphere
    hl, d = 50.0, 10.0
    centres = rs.uniform(-40, 40, (12, 3))
    pts = np.repeat(centres, 12, axis=0) + rs.normal(0, 1.5, (144, 3))
    out.append(("clusters", pts[:, 0], pts[:, 1], pts[:, 2], rs.lognormal(2, 0.5, 144), hl, d,
                "none", True))
    # lattice half-integers, no shift: every deposit is an llrint tie on one axis (the other two
    # at sphere centres), so it lies on a sphere surface (dist == r^2) and hits
    hl, d = 50.0, 4.0
    g = py_geometry(hl, d)
    ks = np.arange(-3, 4)
    tie = g["gSO"] + (ks + 12 + 0.5) * d
    centre = g["gSO"] + (ks + 12) * d
    x = np.concatenate([tie, centre, centre + 2.0, centre - 2.0])
    y = np.concatenate([centre, centre, centre, centre])
    z = np.concatenate([centre, tie, centre, centre])
    out.append(("ties", x, y, z, np.full(len(x), 20.0 / 3.0), hl, d, "none", False))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_oracle_matches_python_restatement(case):
    name, x, y, z, e, hl, d, zs, shift = case
    g, _ = py_job([], [], [], [], hl, d, zs, [], np.zeros(2))
    og = po.geometry(hl, d)
    assert (og["N"], og["HL"], og["gSO"], og["r"]) == (g["N"], g["HL"], g["gSO"], g["r"])
    n_os = 4
    sx = po.shifts(hl, d, shift, 1234, 7, n_os)
    edges = po.edges("log", 60, 0.01, 1e4)
    counts, yfy, stats, sph = po.run_job(x, y, z, e, half_length=hl, sphere_diameter=d, sxsy=sx,
                                         edges_arr=edges, zshift=zs, spheres_cap=1 << 16)
    _, rec = py_job(x, y, z, e, hl, d, zs, [tuple(v) for v in sx], edges)
    assert len(rec) == len(sph) and stats["spheres"] == len(rec)
    assert len(rec) > 0, name
    got = sorted((int(s["os"]), int(s["key"]), int(s["nhits"]), float(s["y"]),
                  float(s["y_seq"]), int(s["bin"])) for s in sph)
    assert got == sorted(rec)
    assert stats["hits"] == sum(r[2] for r in rec)
    pc = np.zeros(len(edges) - 1, dtype=np.int64)
    for r in rec:
        if r[5] >= 0:
            pc[r[5]] += 1
    assert np.array_equal(counts, pc)
    py_yfy = np.zeros(len(edges) - 1)
    for r in rec:                                 # per oversample in key order, as the oracle
        if r[5] >= 0:
            py_yfy[r[5]] += r[3]
    assert np.array_equal(yfy, py_yfy)
    if name == "clusters":
        assert max(r[2] for r in rec) > 1       # spheres with several hits were exercised
    if name == "ties":
        assert stats["hits"] == len(x) * n_os
        # the case tells both rules apart: a strict sphere test loses the surface hits, and
        # rounding halves up moves them to other spheres
        pts = [tuple(v) for v in sx]
        _, strict = py_job(x, y, z, e, hl, d, zs, pts, edges, inside=lambda a, b: a < b)
        assert sum(r[2] for r in strict) < stats["hits"]
        _, half_up = py_job(x, y, z, e, hl, d, zs, pts, edges,
                            rnd=lambda v: math.floor(v + 0.5))
        assert sorted(half_up) != sorted(rec)


def py_job_f32(x, y, z, edep, hl, d, zshift, sxsy, edges):
    """The FP32 geometry variant: x, y, the shifts and the voxel half-length rounded to float and
    the box test in float; a = x' - gSO, k = rint(a * (1/d)), dx = k*d - a and
    dist = (dx^2 + dy^2) + float(dz^2) in float, with z, keys and values as in the FP64 path.
    numpy float32 scalars round every operation and never contract to FMA."""
    f = np.float32
    g = py_geometry(hl, d)
    hlp, gso, n, r2 = g["HL"], g["gSO"], g["N"], g["r"] * g["r"]
    lineal = (2.0 / 3.0) * d
    f_hl, f_gso, f_d, f_r2 = f(hlp), f(gso), f(d), f(r2)
    f_inv_d = f(1.0) / f_d
    zs = [float(v) + ZSHIFT[zshift] * hlp for v in z]
    records = []
    for os_, (sx, sy) in enumerate(sxsy):
        spheres = {}
        for i in range(len(x)):
            fx, fy = f(x[i]) + f(sx), f(y[i]) + f(sy)
            if not (abs(fx) < f_hl and abs(fy) < f_hl and abs(zs[i]) < hlp):
                continue
            ax, ay = fx - f_gso, fy - f_gso
            kx, ky = np.rint(ax * f_inv_d), np.rint(ay * f_inv_d)
            dx, dy = kx * f_d - ax, ky * f_d - ay
            az = zs[i] - gso
            kz = round(az / d)
            dz = float(kz) * d - az
            if (dx * dx + dy * dy) + f(dz * dz) <= f_r2:
                key = (int(kx) + int(ky) * n + kz * n * n) % U64
                spheres.setdefault(key, []).append(float(edep[i]) / lineal)
        for key in sorted(spheres):
            vals = spheres[key]
            seq = vals[0]
            for v in vals[1:]:
                seq = seq + v
            yx = math.fsum(vals)
            b = int(np.searchsorted(edges, yx, side="right")) - 1
            records.append((os_, key, len(vals), yx, seq, b if 0 <= b < len(edges) - 1 else -1))
    return records


@pytest.mark.parametrize("case", [c for c in _cases() if c[0] != "ties"], ids=lambda c: c[0])
def test_fp32_oracle_matches_float32_restatement(case):
    name, x, y, z, e, hl, d, zs, shift = case
    n_os = 4
    sx = po.shifts(hl, d, shift, 99, 3, n_os)
    edges = po.edges("log", 60, 0.01, 1e4)
    counts, yfy, stats, sph = po.run_job(x, y, z, e, half_length=hl, sphere_diameter=d, sxsy=sx,
                                         edges_arr=edges, zshift=zs, spheres_cap=1 << 16,
                                         precision=32)
    rec = py_job_f32(x, y, z, e, hl, d, zs, [tuple(v) for v in sx], edges)
    assert len(rec) > 0, name
    got = sorted((int(s["os"]), int(s["key"]), int(s["nhits"]), float(s["y"]),
                  float(s["y_seq"]), int(s["bin"])) for s in sph)
    assert got == sorted(rec)
    assert stats["hits"] == sum(r[2] for r in rec)

"""Restatement of the reference's density file (TEST INFRASTRUCTURE ONLY: imported by tests/
as the checker of the library's writer and restart reader, never by the product).

  write     src/module_postprocessing.f90:45-95  (Fortran unformatted sequential records,
            4-byte length markers as gfortran writes them)
  restart   read_restart_file, src/module_density.f90:61-261: header, site checks,
            projections -> proj2angl -> trilinear interpolation in the reference's loop order
The per-point angular transforms are the C oracle's (oracle.Oracle.angl2proj / proj2angl).
"""
from __future__ import annotations

import math
import struct

import numpy as np

SITE = struct.Struct("<100sii3ddddddi")   # site_type: name, type, n_sites, r(3), q, sig, eps, lambda1, lambda2, Z
assert SITE.size == 176


def read_records(path: str) -> list[bytes]:
    out = []
    with open(path, "rb") as f:
        data = f.read()
    i = 0
    while i < len(data):
        (n,) = struct.unpack_from("<i", data, i)
        rec = data[i + 4:i + 4 + n]
        (m,) = struct.unpack_from("<i", data, i + 4 + n)
        assert m == n and len(rec) == n, "record markers do not match"
        out.append(rec)
        i += 8 + n
    return out


def parse(path: str) -> dict:
    r = read_records(path)
    ns = struct.unpack("<i", r[0])[0]
    d = dict(ns=ns, mmax=struct.unpack("<i", r[1])[0], no=struct.unpack("<i", r[2])[0], np=struct.unpack("<i", r[3])[0],
             n3=struct.unpack("<3i", r[4]), d3=struct.unpack("<3d", r[5]), nsite=struct.unpack("<i", r[6])[0])
    sites = [SITE.unpack(r[7 + k]) for k in range(d["nsite"])]
    d["sites"] = [dict(r=s[3:6], q=s[6], sig=s[7], eps=s[8], Z=s[11], name=s[0]) for s in sites]
    body = r[7 + d["nsite"]:]
    npt = d["n3"][0] * d["n3"][1] * d["n3"][2]
    if ns < 0:
        assert len(body) == npt * d["no"]
        d["xi"] = np.array([struct.unpack("<d", b)[0] for b in body]).reshape(d["n3"][2], d["n3"][1], d["n3"][0], d["no"])
    else:
        assert len(body) == npt
        d["proj"] = np.array([np.frombuffer(b, dtype=np.complex128) for b in body]).reshape(
            d["n3"][2], d["n3"][1], d["n3"][0], d["np"])
    return d


def restart(orc, d: dict, grid_n3, grid_d3, grid_L, xi_start):
    """xi on this grid from a parsed projection file, as read_restart_file computes it:
    proj2angl per file point, then the literal interpolation loops (1-based indices)."""
    nxp, nyp, nzp = d["n3"]
    dxp, dyp, dzp = d["d3"]
    nx, ny, nz = grid_n3
    dx, dy, dz = grid_d3
    offx, offy, offz = [(grid_L[a] - d["d3"][a] * d["n3"][a]) / 2 for a in range(3)]
    np_ = orc.np
    no = orc.no
    pad = np.zeros((nzp, nyp, nxp, np_), dtype=np.complex128)
    pad[..., :d["np"]] = d["proj"]
    xp = np.zeros((nzp, nyp, nxp, no))
    for k in range(nzp):
        for j in range(nyp):
            for i in range(nxp):
                xp[k, j, i] = orc.proj2angl(pad[k, j, i])
    xi = np.array(xi_start, dtype=np.float64, copy=True)
    for io in range(no):
        for izp in range(1, nzp):
            z0 = (izp - 1) * dzp + offz
            z1 = izp * dzp + offz
            for iyp in range(1, nyp):
                y0 = (iyp - 1) * dyp + offy
                y1 = iyp * dyp + offy
                for ixp in range(1, nxp):
                    x0 = (ixp - 1) * dxp + offx
                    x1 = ixp * dxp + offx
                    for iz in range(max(1, math.ceil(z0 / dz + 1)), min(nz, math.floor(z1 / dz + 1)) + 1):
                        for iy in range(max(1, math.ceil(y0 / dy + 1)), min(ny, math.floor(y1 / dy + 1)) + 1):
                            for ix in range(max(1, math.ceil(x0 / dx + 1)), min(nx, math.floor(x1 / dx + 1)) + 1):
                                z, y, x = (iz - 1) * dz, (iy - 1) * dy, (ix - 1) * dx
                                xd, yd, zd = (x - x0) / (x1 - x0), (y - y0) / (y1 - y0), (z - z0) / (z1 - z0)
                                a = lambda I, J, K: xp[K - 1, J - 1, I - 1, io]
                                xi00 = a(ixp, iyp, izp) * (1 - xd) + a(ixp + 1, iyp, izp) * xd
                                xi01 = a(ixp, iyp, izp + 1) * (1 - xd) + a(ixp + 1, iyp, izp + 1) * xd
                                xi10 = a(ixp, iyp + 1, izp) * (1 - xd) + a(ixp + 1, iyp + 1, izp) * xd
                                xi11 = a(ixp, iyp + 1, izp + 1) * (1 - xd) + a(ixp + 1, iyp + 1, izp + 1) * xd
                                xi0 = xi00 * (1 - yd) + xi10 * yd
                                xi1 = xi01 * (1 - yd) + xi11 * yd
                                xi[iz - 1, iy - 1, ix - 1, io] = xi0 * (1 - zd) + xi1 * zd
    return xi

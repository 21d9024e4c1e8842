"""Pins of the density-file restatement (oracle/restart_ref.py), the checker of the library's
writer and restart reader: record framing, the exact angular round trip of band-limited
fields, and the re-grid reproducing a field linear in position on every covered point."""
import struct

import numpy as np
import pytest

import cases
from oracle import oracle as O
from oracle import restart_ref as R

SV = cases.SOLVENT


def _write(path, ns, mmax, no, np_, n3, d3, sites, body):
    def rec(f, b):
        f.write(struct.pack("<i", len(b)) + b + struct.pack("<i", len(b)))
    with open(path, "wb") as f:
        for v in (ns, mmax, no, np_):
            rec(f, struct.pack("<i", v))
        rec(f, struct.pack("<3i", *n3))
        rec(f, struct.pack("<3d", *d3))
        rec(f, struct.pack("<i", len(sites)))
        for s in sites:
            rec(f, R.SITE.pack(b" " * 100, 0, 0, *s["r"], s["q"], s["sig"], s["eps"], 0.0, 0.0, s["Z"]))
        for b in body:
            rec(f, b)


@pytest.fixture(scope="module")
def orc(tmp_path_factory):
    ck = cases.ck_path(tmp_path_factory.mktemp("ck"), 1)
    return O.Oracle(8, 4.0, 1, ck, SV.kT, SV.n0)


def test_band_limited_round_trip_is_exact(orc):
    u = orc.rotm[:, :, 2]
    x = 1.0 + 0.3 * u[:, 2] - 0.2 * u[:, 0] + 0.1 * u[:, 1]
    assert np.abs(orc.proj2angl(orc.angl2proj(x)) - x).max() < 1e-14


def test_records_and_linear_regrid(orc, tmp_path):
    # a 6^3 file grid (0.5 A) centred in the 8^3, 4 A grid: offset 0.5 A on every axis
    n3p, dp = (6, 6, 6), (0.5, 0.5, 0.5)
    u = orc.rotm[:, :, 2]
    coef = np.array([0.05, -0.03, 0.02])
    body, xi_file = [], np.zeros((6, 6, 6, orc.no))
    for k in range(6):
        for j in range(6):
            for i in range(6):
                r = np.array([i, j, k]) * 0.5 + 0.5                      # position in the new box
                xi_file[k, j, i] = 1.0 + 0.3 * u[:, 2] + coef @ r       # linear in r, band-limited in omega
                body.append(np.ascontiguousarray(orc.angl2proj(xi_file[k, j, i])).tobytes())
    sites = [dict(r=(1.0, 1.5, 2.0), q=0.5, sig=3.0, eps=0.4, Z=6)]
    path = str(tmp_path / "density.bin")
    _write(path, 1, 1, orc.no, orc.np, n3p, dp, sites, body)
    f = R.parse(path)
    assert (f["ns"], f["mmax"], f["no"], f["np"], f["n3"], f["d3"], f["nsite"]) == (1, 1, orc.no, orc.np, n3p, dp, 1)
    assert f["sites"][0]["r"] == (1.0, 1.5, 2.0) and f["sites"][0]["Z"] == 6
    start = np.full((8, 8, 8, orc.no), -7.0)
    xi = R.restart(orc, f, (8, 8, 8), (0.5, 0.5, 0.5), (4.0, 4.0, 4.0), start)
    covered = np.zeros((8, 8, 8), bool)
    covered[1:7, 1:7, 1:7] = True                                        # new points 0.5 .. 3.0 A
    for k in range(8):
        for j in range(8):
            for i in range(8):
                if covered[k, j, i]:
                    r = np.array([i, j, k]) * 0.5
                    assert np.abs(xi[k, j, i] - (1.0 + 0.3 * u[:, 2] + coef @ r)).max() < 1e-13
                else:
                    assert (xi[k, j, i] == -7.0).all()


def test_mismatched_record_markers_are_refused(tmp_path):
    p = str(tmp_path / "bad.bin")
    with open(p, "wb") as f:
        f.write(struct.pack("<i", 4) + struct.pack("<i", 1) + struct.pack("<i", 8))
    with pytest.raises(AssertionError):
        R.read_records(p)

"""The reference's density file: the library's writer against the restatement's parser and
the C oracle's angl2proj, and the restart reader (proj2angl + re-grid) against the literal
loops of read_restart_file (oracle/restart_ref.py)."""
import struct

import numpy as np
import pytest

import cases
from mdft_b200 import Engine, MdftError, synth
from oracle import oracle as O
from oracle import restart_ref as R

pytestmark = pytest.mark.gpu
SV = cases.SOLVENT


@pytest.fixture(scope="module")
def solved(tmp_path_factory):
    c = cases.CASES["mol16_m2"]
    d = tmp_path_factory.mktemp("restart")
    ck = cases.ck_path(d, c["mmax"])
    e = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0)
    sol = cases.solute_of(c)
    sol.Z = np.arange(1, sol.nsite + 1)
    xi = np.zeros(e.shape)
    r = e.solve(sol, SV, rvdw=c["rvdw"], m=5, pgtol=1e-5, ftol_abs=-1.0, itermax=2000, xi_out=xi)
    o = O.Oracle(c["n"], c["L"], c["mmax"], ck, SV.kT, SV.n0)
    yield c, ck, e, sol, xi, r, o, d
    e.close()


def test_projection_file_matches_the_restatement(solved):
    c, _, e, sol, xi, _, o, d = solved
    path = str(d / "density.bin")
    e.write_density_bin(path, sol)           # the last solve's density
    f = R.parse(path)
    assert (f["ns"], f["mmax"], f["no"], f["np"]) == (1, c["mmax"], e.no, e.np)
    assert f["n3"] == (c["n"],) * 3 and np.allclose(f["d3"], c["L"] / c["n"], rtol=0, atol=0)
    assert f["nsite"] == sol.nsite
    for k, s in enumerate(f["sites"]):
        assert s["r"] == tuple(sol.xyz[k]) and (s["q"], s["sig"], s["eps"], s["Z"]) == (sol.q[k], sol.sig[k], sol.eps[k], k + 1)
    ref = np.array([o.angl2proj(np.ascontiguousarray(xi[iz, iy, ix])) for iz in range(c["n"]) for iy in range(c["n"])
                    for ix in range(c["n"])]).reshape(f["proj"].shape)
    assert np.abs(f["proj"] - ref).max() <= 1e-13 * np.abs(ref).max()


def test_full_density_file_is_exact(solved):
    c, _, e, sol, xi, _, _, d = solved
    path = str(d / "density_full.bin")
    e.write_density_bin(path, sol, xi=xi, full=True)
    f = R.parse(path)
    assert f["ns"] == -1 and np.array_equal(f["xi"], xi)
    back = e.read_density_bin(path, sol)
    assert np.array_equal(back, xi)
    # the exact converged density: the minimiser stops at its first evaluation
    _, rr = e.minimize(back, m=5, pgtol=1e-5, ftol_abs=-1.0, itermax=2000)
    assert rr["status"] == 0 and rr["evaluations"] <= 2


def test_restart_on_the_same_grid(solved):
    c, _, e, sol, xi, r, o, d = solved
    path = str(d / "density.bin")
    e.write_density_bin(path, sol, xi=xi)
    start = e.guess_density()
    got = e.read_density_bin(path, sol, xi_start=start)
    ref = R.restart(o, R.parse(path), (c["n"],) * 3, (c["L"] / c["n"],) * 3, (c["L"],) * 3, start)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    # from the restart point the minimiser needs fewer evaluations than from the bulk (the
    # projection file keeps only the band-limited part of xi: 79 against 95 here)
    _, rr = e.minimize(got, m=5, pgtol=1e-5, ftol_abs=-1.0, itermax=2000)
    assert rr["status"] == 0 and rr["evaluations"] < r["evaluations"]


def test_restart_onto_a_larger_box_and_higher_mmax(tmp_path):
    ca = dict(n=12, L=6.0, mmax=1)
    cb = dict(n=16, L=8.0, mmax=2)
    ea = Engine(ca["n"], ca["L"], ca["mmax"], cases.ck_path(tmp_path, 1), temperature=SV.temperature, n0=SV.n0)
    ckb = cases.ck_path(tmp_path, 2)
    eb = Engine(cb["n"], cb["L"], cb["mmax"], ckb, temperature=SV.temperature, n0=SV.n0)
    sa = synth.random_walk_solute(4, seed=8, radius=1.5)
    sa.xyz = synth.center_solute(sa.xyz, (ca["L"],) * 3)
    sb = synth.Solute(q=sa.q, sig=sa.sig, eps=sa.eps, xyz=sa.xyz + 1.0)   # the centring offset (8 - 12 x 0.5)/2
    rng = np.random.default_rng(9)
    xa = rng.uniform(0.5, 1.5, ea.shape)
    path = str(tmp_path / "density.bin")
    ea.write_density_bin(path, sa, xi=xa)
    start = rng.uniform(0.9, 1.1, eb.shape)
    got = eb.read_density_bin(path, sb, xi_start=start)
    ob = O.Oracle(cb["n"], cb["L"], cb["mmax"], ckb, SV.kT, SV.n0)
    ref = R.restart(ob, R.parse(path), (cb["n"],) * 3, (cb["L"] / cb["n"],) * 3, (cb["L"],) * 3, start)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.array_equal(got[0], start[0]) and not np.array_equal(got[8], start[8])  # z = 0 lies outside the file's box
    with pytest.raises(MdftError, match="differs"):
        eb.read_density_bin(path, sa, xi_start=start)                        # positions without the offset
    # a file of higher mmax than the reading grid is refused (its projections do not fit)
    e0 = Engine(8, 4.0, 0, cases.ck_path(tmp_path, 0), temperature=SV.temperature, n0=SV.n0)
    with pytest.raises(MdftError, match="mmax"):
        e0.read_density_bin(path, synth.Solute(q=sa.q, sig=sa.sig, eps=sa.eps, xyz=sa.xyz - 1.0))
    e0.close()
    with open(path, "rb") as f:
        head = f.read(200)
    with open(str(tmp_path / "short.bin"), "wb") as f:
        f.write(head)
    with pytest.raises(MdftError):
        eb.read_density_bin(str(tmp_path / "short.bin"), sb, xi_start=start)
    # a corrupt grid spacing (zero, negative, NaN, huge) is refused before any interpolation;
    # the spacing record's data sits at bytes 72..96 (after five framed integer records)
    with open(path, "rb") as f:
        whole = bytearray(f.read())
    assert struct.unpack_from("<i", whole, 68)[0] == 24
    for bad in (0.0, -0.5, float("nan"), float("inf"), 1e300):
        patched = bytearray(whole)
        struct.pack_into("<d", patched, 80, bad)
        with open(str(tmp_path / "bad_spacing.bin"), "wb") as f:
            f.write(patched)
        with pytest.raises(MdftError, match="spacing"):
            eb.read_density_bin(str(tmp_path / "bad_spacing.bin"), sb, xi_start=start)
    ea.close()
    eb.close()

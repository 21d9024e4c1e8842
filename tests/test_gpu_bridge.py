"""The bridges (bridge = "cgb" and "hard_sphere") on the GPU against the FP64 oracle, through
the C-ABI: the seam (energy_bridge), full evaluations, and L-BFGS trajectories with the term.

Tolerances as the FP64 path: F <= 1e-10 relative, df <= 1e-8 of max|df|.
"""
import numpy as np
import pytest

from oracle import oracle as O
from mdft_b200 import Engine, Mixture, MdftError, PREC_FP64, PREC_MIXED
import cases

pytestmark = pytest.mark.gpu
SV = cases.SOLVENT
PARAMS = {1: dict(B6=5.0, sigma=1.0, c00=-13.665), 2: dict(B6=3.0, sigma=1.3, c00=-11.9078)}


def pair(tmp_path, name):
    c = cases.ALL_CASES[name]
    ck = cases.case_ck(tmp_path, c)
    o = O.Oracle(c["n"], c["L"], c["mmax"], ck, SV.kT, SV.n0)
    e = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0)
    sol = cases.solute_of(c)
    lj = o.compute_vext(sol, SV, rvdw=c["rvdw"])
    e.set_vext(o.get_vext())
    corr = cases.charge_correction(sol, c["L"])
    o.set_const_corr(corr)
    e.set_constant_correction(corr)
    return c, o, e, lj


@pytest.mark.parametrize("version", [1, 2])
@pytest.mark.parametrize("name", ["mol16_m2", "ion32_m1"])
def test_bridge_energy_gradient_parity(tmp_path, name, version):
    c, o, e, _ = pair(tmp_path, name)
    o.set_bridge_cgb(version, **PARAMS[version])
    e.set_bridge_cgb(version, **PARAMS[version])
    xi = cases.xi_of(c, o.shape, amp=0.3)
    f0, df0, t0 = o.energy_grad(xi)
    f1, df1, t1 = e.energy_and_gradient(xi)
    assert abs(f1 - f0) <= 1e-10 * abs(f0), (f1, f0)
    assert np.all(np.abs(t1 - t0) <= 1e-10 * abs(f0))
    assert np.abs(df1 - df0).max() <= 1e-8 * np.abs(df0).max()
    # the seam alone: F_b and the gradient it adds
    g0 = np.zeros(o.shape)
    g1 = np.zeros(o.shape)
    fb0 = o.bridge_energy(xi, g0)
    fb1 = e.bridge_energy(xi, g1)
    assert abs(fb1 - fb0) <= 1e-10 * max(abs(fb0), abs(f0))
    assert np.abs(g1 - g0).max() <= 1e-8 * np.abs(g0).max()
    # removing the term restores the plain functional
    e.set_bridge_cgb(0)
    o.set_bridge_cgb(0)
    f2, _, _ = e.energy_and_gradient(xi)
    f3, _, _ = o.energy_grad(xi)
    assert abs(f2 - f3) <= 1e-10 * abs(f3)
    e.close()


def test_bridge_minimize_trajectory_parity(tmp_path):
    # the FP64 minimiser includes the bridge (F, gradient and the stopping quantities): the
    # same L-BFGS trajectory as the oracle's for 25 iterations, and the same dG
    c, o, e, lj = pair(tmp_path, "mol16_m2")
    o.set_bridge_cgb(1, **PARAMS[1])
    e.set_bridge_cgb(1, **PARAMS[1])
    x0 = o.guess_density()
    xo, fo, nfo, ito, sto = o.minimize(x0, m=5, pgtol=1e-12, tol=-1.0, itermax=25)
    xg, r = e.minimize(x0, m=5, pgtol=1e-12, ftol_abs=-1.0, itermax=25)
    assert (r["iterations"], r["evaluations"], r["status"]) == (ito, nfo, sto)
    assert abs(r["f"] - fo) <= 1e-9 * abs(fo)
    assert np.abs(xg - xo).max() <= 1e-6
    pg = e.pressure_correction(xg, r["f"], lj)
    po = o.pressure_correction(xo, fo, lj)
    assert abs(pg["dG"] - po["dG"]) <= 1e-6, (pg, po)
    e.close()


def test_bridge_refusals(tmp_path):
    c, o, e, _ = pair(tmp_path, "mol16_m2")
    ck = cases.case_ck(tmp_path, c)
    mixed = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=PREC_MIXED)
    with pytest.raises(MdftError, match="FP64 handle"):
        mixed.set_bridge_cgb(1, **PARAMS[1])
    with pytest.raises(MdftError, match="FP64 handle"):
        mixed.set_bridge_fmt(1, 1.4)
    with pytest.raises(MdftError, match="packing fraction"):
        e.set_bridge_fmt(1, 3.0)
    with pytest.raises(MdftError, match="sigma"):
        e.set_bridge_cgb(1, B6=1.0, sigma=0.0, c00=-13.665)
    e.set_bridge_cgb(1, **PARAMS[1])
    # FP32 evaluations (a mixed solve) are refused while the bridge is set
    with pytest.raises(MdftError, match="FP64 only"):
        e.minimize(e.guess_density(), precision=PREC_MIXED, itermax=5)
    # the reference's bridges take one species
    other = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0 * 0.5)
    e.close()
    e = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0 * 0.5)
    e.set_bridge_cgb(1, **PARAMS[1])
    with pytest.raises(MdftError, match="bridge"):
        Mixture([e, other], [0.5, 0.5])
    for h in (e, other, mixed):
        h.close()


# ---- bridge = "hard_sphere" ---------------------------------------------------------------

@pytest.mark.parametrize("functional", [1, 2])
@pytest.mark.parametrize("name", ["mol16_m2", "ion32_m1"])
def test_fmt_bridge_energy_gradient_parity(tmp_path, name, functional):
    c, o, e, _ = pair(tmp_path, name)
    o.set_bridge_fmt(functional, 1.4)
    e.set_bridge_fmt(functional, 1.4)
    po, pe = o.fmt_params(), e.bridge_fmt_params()
    assert po[3] == pe[3]
    np.testing.assert_allclose(pe[:3], po[:3], rtol=1e-14)
    xi = cases.xi_of(c, o.shape, amp=0.3)
    f0, df0, t0 = o.energy_grad(xi)
    f1, df1, t1 = e.energy_and_gradient(xi)
    assert abs(f1 - f0) <= 1e-10 * abs(f0), (f1, f0)
    assert np.all(np.abs(t1 - t0) <= 1e-10 * abs(f0))
    assert np.abs(df1 - df0).max() <= 1e-8 * np.abs(df0).max()
    g0 = np.zeros(o.shape)
    g1 = np.zeros(o.shape)
    fb0 = o.bridge_energy(xi, g0)
    fb1 = e.bridge_energy(xi, g1)
    assert abs(fb1 - fb0) <= 1e-10 * max(abs(fb0), abs(f0))
    assert np.abs(g1 - g0).max() <= 1e-8 * np.abs(g0).max()
    # empty box: -Fexc0, no gradient; n3 >= 1: an error, and the handle evaluates after it
    g2 = np.zeros(o.shape)
    assert e.bridge_energy(np.zeros(o.shape), g2) == -pe[2]
    assert not g2.any()
    with pytest.raises(MdftError, match="hard-sphere"):
        e.energy_and_gradient(3.0 * np.ones(o.shape))
    f3, _, _ = e.energy_and_gradient(xi)
    assert f3 == f1
    e.close()


def test_fmt_bridge_minimize_trajectory_parity(tmp_path):
    # R = 0.5 A (bulk packing fraction 0.017): in this 8 A box the first iterates grow xi at
    # the solute's contact, and from R = 0.7 A a trial point reaches a weighted density
    # n3 >= 1, where the reference's functional stops (the oracle and the GPU both report it)
    c, o, e, lj = pair(tmp_path, "mol16_m2")
    o.set_bridge_fmt(1, 0.5)
    e.set_bridge_fmt(1, 0.5)
    x0 = o.guess_density()
    xo, fo, nfo, ito, sto = o.minimize(x0, m=5, pgtol=1e-12, tol=-1.0, itermax=25)
    xg, r = e.minimize(x0, m=5, pgtol=1e-12, ftol_abs=-1.0, itermax=25)
    assert (r["iterations"], r["evaluations"], r["status"]) == (ito, nfo, sto)
    assert abs(r["f"] - fo) <= 1e-9 * abs(fo)
    assert np.abs(xg - xo).max() <= 1e-6
    pg = e.pressure_correction(xg, r["f"], lj)
    po = o.pressure_correction(xo, fo, lj)
    assert abs(pg["dG"] - po["dG"]) <= 1e-6, (pg, po)
    e.close()

"""Multi-species solvent on the GPU (mdft_mixture_*) against the FP64 oracle's
energy_cproj_mrso_mixture restatement, through the C-ABI.

Tolerances as the single-species FP64 path: F <= 1e-10 relative, each term <= 1e-10 of
|F|, gradient max|df_gpu - df_oracle| <= 1e-8 * max|df_oracle| over all species.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from mdft_b200 import Engine, Mixture, MdftError, PREC_MIXED, engine, synth
import cases

pytestmark = pytest.mark.gpu
SV = cases.SOLVENT
# a second water model (TIP3P geometry, charges and LJ; its pure-fluid density)
TIP3P = synth.Solvent(q=(-0.834, 0.417, 0.417), sig=(3.15061, 0.0, 0.0), eps=(0.636386, 0.0, 0.0),
                      xyz=((0.0, 0.0, 0.0), (0.756950, 0.0, 0.585882), (-0.756950, 0.0, 0.585882)), n0=0.03349459)

MIXES = {
    # name: grid n, box L, mmax, solute, seed, rvdw, species [(solvent, c(k) seed, mole fraction)]
    "walk5_16_m2": dict(n=16, L=8.0, mmax=2, solute="walk5", seed=2, rvdw=3.9,
                        species=[(SV, 20260000, 0.3), (TIP3P, 20260011, 0.7)]),
    "ion32_m1": dict(n=32, L=20.0, mmax=1, solute="ion", seed=21, rvdw=10.0, dk=0.01, kmax=12.0,
                     species=[(SV, 20260000, 0.5), (TIP3P, 20260012, 0.5)]),
    "walk6_24_m3_three": dict(n=24, L=12.0, mmax=3, solute="walk6", seed=4, rvdw=5.9,
                              species=[(SV, 20260000, 0.25), (TIP3P, 20260013, 0.25), (SV, 20260014, 0.5)]),
}


def build(tmp_path, name):
    c = MIXES[name]
    sol = cases.solute_of(c)
    oracles, engines = [], []
    for solvent, seed, x in c["species"]:
        ck = cases.ck_path(tmp_path, c["mmax"], kmax=c.get("kmax", 14.0), dk=c.get("dk"), seed=seed)
        o = O.Oracle(c["n"], c["L"], c["mmax"], ck, SV.kT, solvent.n0 * x)
        e = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=solvent.n0 * x)
        o.compute_vext(sol, solvent, rvdw=c["rvdw"])
        e.set_vext(o.get_vext())
        oracles.append(o)
        engines.append(e)
    corr = cases.charge_correction(sol, c["L"])
    oracles[0].set_const_corr(corr)
    engines[0].set_constant_correction(corr)
    fr = [x for _, _, x in c["species"]]
    rng = np.random.default_rng(c["seed"] + 500)
    xi = np.stack([1.0 + 0.15 * rng.standard_normal(oracles[0].shape) for _ in fr])
    return c, oracles, engines, fr, xi


@pytest.mark.parametrize("name", sorted(MIXES))
def test_mixture_energy_gradient_parity(tmp_path, name):
    c, oracles, engines, fr, xi = build(tmp_path, name)
    f0, df0, t0 = O.mixture_energy_grad(oracles, fr, xi)
    with Mixture(engines, fr) as mix:
        f1, df1, t1 = mix.energy_and_gradient(xi)
        assert abs(f1 - f0) <= 1e-10 * abs(f0), (f1, f0)
        assert np.all(np.abs(t1 - t0) <= 1e-10 * abs(f0)), (t1, t0)
        err = np.abs(df1 - df0).max() / np.abs(df0).max()
        assert err <= 1e-8, err
        # energy only (no gradient) gives the same F; a second call the same result
        f2, _, t2 = mix.energy_and_gradient(xi, want_grad=False)
        assert f2 == f1 and np.array_equal(t2, t1)
        f3, df3, _ = mix.energy_and_gradient(xi)
        assert f3 == f1 and np.array_equal(df3, df1)
    for e in engines:
        e.close()


def test_species_handles_evaluate_alone_after_the_mixture(tmp_path):
    # the mixture borrows the handles' buffers; once closed, each handle's own
    # single-species evaluation still matches the oracle's
    c, oracles, engines, fr, xi = build(tmp_path, "walk5_16_m2")
    with Mixture(engines, fr) as mix:
        mix.energy_and_gradient(xi)
    f0, df0, _ = oracles[1].energy_grad(xi[1])
    f1, df1, _ = engines[1].energy_and_gradient(xi[1])
    assert abs(f1 - f0) <= 1e-10 * abs(f0)
    assert np.abs(df1 - df0).max() <= 1e-8 * np.abs(df0).max()
    for e in engines:
        e.close()


def test_mixture_refusals(tmp_path):
    c, oracles, engines, fr, xi = build(tmp_path, "walk5_16_m2")
    with pytest.raises(MdftError, match="at least two"):
        Mixture(engines[:1], [1.0])
    with pytest.raises(MdftError, match="sum to"):
        Mixture(engines, [0.3, 0.6])
    with pytest.raises(MdftError, match="outside"):
        Mixture(engines, [1.3, -0.3])
    with pytest.raises(MdftError, match="same handle"):
        Mixture([engines[0], engines[0]], [0.5, 0.5])
    ck = cases.ck_path(tmp_path, c["mmax"], seed=20260000)
    other = Engine(8, 4.0, c["mmax"], ck, temperature=SV.temperature, n0=SV.n0 * 0.7)
    with pytest.raises(MdftError, match="differs"):
        Mixture([engines[0], other], fr)
    mixed = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0 * 0.7, precision=PREC_MIXED)
    with pytest.raises(MdftError, match="FP64"):
        Mixture([engines[0], mixed], fr)
    for e in engines + [other, mixed]:
        e.close()


def test_mixture_minimize_trajectory_parity(tmp_path):
    # the L-BFGS over both species' xi: the same trajectory as the oracle's for 25 iterations
    c, oracles, engines, fr, _ = build(tmp_path, "walk5_16_m2")
    x0 = np.stack([o.guess_density() for o in oracles])
    xo, fo, nfo, ito, sto = O.mixture_minimize(oracles, fr, x0, m=5, pgtol=1e-12, tol=-1.0, itermax=25)
    with Mixture(engines, fr) as mix:
        xg, r = mix.minimize(x0, m=5, pgtol=1e-12, ftol_abs=-1.0, itermax=25)
        assert (r["iterations"], r["evaluations"], r["status"]) == (ito, nfo, sto)
        assert abs(r["f"] - fo) <= 1e-9 * abs(fo)
        assert np.abs(xg - xo).max() <= 1e-6
        # the result is a point of the mixture's functional
        f1, _, _ = mix.energy_and_gradient(xg)
        assert abs(f1 - r["f"]) <= 1e-12 * abs(f1)
        # a mixed-precision minimisation is refused (the binding always asks for FP64)
        o = engine._MinOpts(5, 1e-6, 1e-3, 5, PREC_MIXED, 0.0, 1, 0.0)
        res = engine._MinRes()
        x = np.ascontiguousarray(x0)
        with pytest.raises(MdftError, match="FP64"):
            engine._check(engine.lib().mdft_mixture_minimize(mix.h, engine._p(x), ctypes.byref(o), ctypes.byref(res)))
    # species 0's handle minimises on its own afterwards
    x1, r1 = engines[0].minimize(oracles[0].guess_density(), m=5, pgtol=1e-12, ftol_abs=-1.0, itermax=3)
    assert r1["iterations"] == 3
    for e in engines:
        e.close()

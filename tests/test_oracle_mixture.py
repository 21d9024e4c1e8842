"""The oracle's multi-species functional (energy_cproj_mrso_mixture) against properties the
reference's algorithm implies, on the CPU.

* mmax 0: the rotations are the identity, so the mixture routine of one species equals the
  single-species routine exactly (src/module_energy_cproj_mrso_mixture.f90:541-557 against
  src/module_energy_cproj_mrso.f90:508-522).
* mmax >= 1: the two routines differ -- the mixture rotates -q with R(m,mup,khi) where the
  single-species routine uses R(m,mup,-khi) -- and the oracle keeps that difference.
* Splitting one species into two identical halves (n0 and mole fraction halved, the same c,
  vext and xi) leaves F unchanged and halves each species' gradient: every term is linear in
  rho0 x, gamma_{s2} sums over s, and the prefactor's n0(s2) cancels x(s2)
  (src/module_energy_cproj_mrso_mixture.f90:791).
* Relabelling the species permutes the gradient blocks and keeps F (to rounding: gamma sums
  over s in another order).
"""
import numpy as np
import pytest

from oracle import oracle as O
import cases

SV = cases.SOLVENT


def _species(tmp_path, n, L, mmax, seeds, fracs, vexts):
    out = []
    for seed, x, v in zip(seeds, fracs, vexts):
        ck = cases.ck_path(tmp_path, mmax, seed=seed)
        o = O.Oracle(n, L, mmax, ck, SV.kT, SV.n0 * x)
        o.set_vext(v)
        out.append(o)
    return out


def _case(n=12, L=6.0, mmax=2):
    return dict(n=n, L=L, mmax=mmax, solute="none", seed=3, rvdw=2.9, xseed=13)


def test_one_species_at_mmax0_is_the_single_species_routine(tmp_path):
    c = _case(mmax=0)
    ck = cases.ck_path(tmp_path, 0)
    o = O.Oracle(c["n"], c["L"], 0, ck, SV.kT, SV.n0)
    o.set_vext(cases.random_vext(c, o.shape))
    xi = cases.xi_of(c, o.shape)
    f1, df1, t1 = o.energy_grad(xi)
    fm, dfm, tm = O.mixture_energy_grad([o], [1.0], xi[None])
    assert fm == f1
    assert np.array_equal(tm, t1)
    assert np.array_equal(dfm[0], df1)


@pytest.mark.parametrize("mmax", [1, 3])
def test_mixture_keeps_its_own_minus_q_rotation(tmp_path, mmax):
    c = _case(mmax=mmax)
    ck = cases.ck_path(tmp_path, mmax)
    o = O.Oracle(c["n"], c["L"], mmax, ck, SV.kT, SV.n0)
    o.set_vext(cases.random_vext(c, o.shape))
    xi = cases.xi_of(c, o.shape)
    f1, df1, t1 = o.energy_grad(xi)
    fm, dfm, tm = O.mixture_energy_grad([o], [1.0], xi[None])
    # the ideal and external terms are the same functions; the excess terms differ
    assert tm[0] == t1[0] and tm[1] == t1[1]
    assert abs(tm[2] - t1[2]) > 1e-6 * abs(t1[2])
    assert np.abs(dfm[0] - df1).max() > 1e-6 * np.abs(df1).max()


@pytest.mark.parametrize("mmax", [1, 2, 3])
def test_two_identical_halves_equal_one_species(tmp_path, mmax):
    c = _case(mmax=mmax)
    ck = cases.ck_path(tmp_path, mmax)
    one = O.Oracle(c["n"], c["L"], mmax, ck, SV.kT, SV.n0)
    v = cases.random_vext(c, one.shape)
    one.set_vext(v)
    xi = cases.xi_of(c, one.shape)
    f1, df1, t1 = O.mixture_energy_grad([one], [1.0], xi[None])
    halves = _species(tmp_path, c["n"], c["L"], mmax, [20260000, 20260000], [0.5, 0.5], [v, v])
    f2, df2, t2 = O.mixture_energy_grad(halves, [0.5, 0.5], np.stack([xi, xi]))
    assert abs(f2 - f1) <= 1e-13 * abs(f1)
    assert np.all(np.abs(t2 - t1) <= 1e-13 * abs(f1))
    scale = np.abs(df1).max()
    assert np.abs(df2[0] - 0.5 * df1[0]).max() <= 1e-13 * scale
    assert np.array_equal(df2[0], df2[1])


def test_relabelling_species_permutes_the_gradient(tmp_path):
    c = _case(mmax=2)
    rng = np.random.default_rng(7)
    fr = [0.2, 0.3, 0.5]
    seeds = [20260001, 20260002, 20260003]
    probe = O.Oracle(c["n"], c["L"], 2, cases.ck_path(tmp_path, 2, seed=seeds[0]), SV.kT, SV.n0)
    vs = [0.6 * rng.standard_normal(probe.shape) for _ in fr]
    xi = np.stack([1.0 + 0.15 * rng.standard_normal(probe.shape) for _ in fr])
    sp = _species(tmp_path, c["n"], c["L"], 2, seeds, fr, vs)
    f, df, t = O.mixture_energy_grad(sp, fr, xi)
    perm = [2, 0, 1]
    sq = _species(tmp_path, c["n"], c["L"], 2, [seeds[i] for i in perm], [fr[i] for i in perm], [vs[i] for i in perm])
    fp, dfp, tp = O.mixture_energy_grad(sq, [fr[i] for i in perm], xi[perm])
    assert abs(fp - f) <= 1e-12 * abs(f)
    assert np.abs(dfp - df[perm]).max() <= 1e-12 * np.abs(df).max()


def test_mixture_argument_checks(tmp_path):
    c = _case(mmax=1)
    ck = cases.ck_path(tmp_path, 1)
    a = O.Oracle(c["n"], c["L"], 1, ck, SV.kT, SV.n0 * 0.5)
    b = O.Oracle(c["n"], c["L"], 1, ck, SV.kT, SV.n0 * 0.5)
    other = O.Oracle(8, 4.0, 1, ck, SV.kT, SV.n0 * 0.5)
    xi = np.ones((2,) + a.shape)
    with pytest.raises(RuntimeError, match="sum to 1"):
        O.mixture_energy_grad([a, b], [0.5, 0.4], xi)
    with pytest.raises(RuntimeError, match="outside"):
        O.mixture_energy_grad([a, b], [1.5, -0.5], xi)
    with pytest.raises(RuntimeError, match="differ"):
        O.mixture_energy_grad([a, other], [0.5, 0.5], xi)

"""The oracle reproduces its committed golden fixtures (tests/golden/*.npz)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
import cases

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def build(name, ckdir):
    c = cases.ALL_CASES[name]
    sv = cases.SOLVENT
    o = O.Oracle(c["n"], c["L"], c["mmax"], cases.case_ck(ckdir, c), sv.kT, sv.n0)
    sol = cases.solute_of(c)
    lj = o.compute_vext(sol, sv, rvdw=c["rvdw"]) if sol is not None else 0.0
    if sol is None:
        o.set_vext(cases.random_vext(c, o.shape))
    o.set_const_corr(cases.charge_correction(sol, c["L"]))
    return o, lj


@pytest.mark.parametrize("name", sorted(cases.ALL_CASES))
def test_oracle_matches_golden(tmp_path, name):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    o, lj = build(name, tmp_path)
    c = cases.ALL_CASES[name]
    xi = cases.xi_of(c, o.shape)
    f, df, terms = o.energy_grad(xi)
    assert abs(f - g["f"]) <= 1e-12 * abs(g["f"])
    np.testing.assert_allclose(terms, g["terms"], rtol=1e-12, atol=1e-12 * abs(g["f"]))
    np.testing.assert_allclose(df.reshape(-1)[g["idx"]], g["df_samples"], rtol=0, atol=1e-12 * np.abs(df).max())
    assert abs(lj - g["lj_tail"]) <= 1e-12 * max(1.0, abs(g["lj_tail"]))
    v = o.get_vext()
    assert abs(v.sum() - g["vext_sum"]) <= 1e-11 * abs(g["vext_sum"]) + 1e-9

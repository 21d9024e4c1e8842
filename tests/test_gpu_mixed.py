"""Mixed-precision path (FP32 projections, FFTs, OZ and per-element arithmetic; FP64 sums,
L-BFGS vectors and the final check) against the FP64 oracle and the FP64 engine.

Tolerances: energy 2e-6 of |F|, the ideal and external terms 1e-7 of |F| (FP32 per-element
arithmetic, FP64 sums) and gradient 1e-4 of max|df| for one evaluation; a mixed solve's dG
within 0.1 kJ/mol of the FP64 solve (the bar of the throughput metric)."""
import numpy as np
import pytest

from oracle import oracle as O
from mdft_b200 import Engine, PREC_MIXED
import cases

pytestmark = pytest.mark.gpu
SV = cases.SOLVENT


@pytest.mark.parametrize("name", ["ion16_m1", "mol16_m2", "rand12_m3", "mol24_m3", "rand8_m5"] + sorted(cases.CONFIG_CASES))
def test_mixed_energy_gradient(tmp_path, name):
    c = cases.ALL_CASES[name]
    ck = cases.case_ck(tmp_path, c)
    o = O.Oracle(c["n"], c["L"], c["mmax"], ck, SV.kT, SV.n0)
    sol = cases.solute_of(c)
    if sol is not None:
        o.compute_vext(sol, SV, rvdw=c["rvdw"])
    else:
        o.set_vext(cases.random_vext(c, o.shape))
    e = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=PREC_MIXED)
    e.set_vext(o.get_vext())
    xi = cases.xi_of(c, o.shape)
    f0, df0, t0 = o.energy_grad(xi)
    f1, df1, t1 = e.energy_and_gradient(xi)
    assert abs(f1 - f0) <= 2e-6 * abs(f0), (f1, f0)
    assert abs(t1[0] - t0[0]) <= 1e-7 * abs(f0) and abs(t1[1] - t0[1]) <= 1e-7 * abs(f0), (t1, t0)
    assert np.abs(df1 - df0).max() <= 1e-4 * np.abs(df0).max()
    e.close()


@pytest.mark.parametrize("name", ["ion16_m1", "mol16_m2"])
def test_mixed_solve_free_energy(tmp_path, name):
    c = cases.CASES[name]
    ck = cases.ck_path(tmp_path, c["mmax"])
    sol = cases.solute_of(c)
    e64 = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0)
    r64 = e64.solve(sol, SV, rvdw=c["rvdw"], m=5, pgtol=1e-6, ftol_abs=-1.0, itermax=3000)
    e32 = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=PREC_MIXED)
    r32 = e32.solve(sol, SV, rvdw=c["rvdw"], m=5, pgtol=1e-6, ftol_abs=-1.0, itermax=3000, precision=PREC_MIXED)
    assert r32["evaluations_mixed"] > 0
    assert abs(r32["dG"] - r64["dG"]) <= 0.1, (r32, r64)
    e64.close()
    e32.close()

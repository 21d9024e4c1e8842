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


@pytest.mark.parametrize("name", ["ion16_m1", "mol16_m2", "mol24_m3", "mol8_m0", "ion32_m1", "mol64_m3"])
def test_tensor_core_angular_transforms(tmp_path, name, monkeypatch):
    # The FP32 evaluation with the angular contractions on the tensor cores (split BF16:
    # hi*hi + hi*lo + lo*hi, FP32 accumulation) against the same evaluation with the FP32
    # FFMA kernels (MDFT_ANGULAR=ffma) and against the FP64 oracle.  Bars: the excess term
    # within 2e-5 of |F_exc| of the oracle's, the total within 2e-6 of |F|, the gradient within
    # 1e-4 of max|df| (the mixed path's bars); the two FP32 forms within 2e-5 of |F_exc|.
    c = cases.ALL_CASES[name]
    ck = cases.case_ck(tmp_path, c)
    o = O.Oracle(c["n"], c["L"], c["mmax"], ck, SV.kT, SV.n0)
    sol = cases.solute_of(c)
    o.compute_vext(sol, SV, rvdw=c["rvdw"])
    monkeypatch.setenv("MDFT_ANGULAR", "ffma")
    e0 = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=PREC_MIXED)
    monkeypatch.delenv("MDFT_ANGULAR")
    e1 = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=PREC_MIXED)
    for e in (e0, e1):
        e.set_vext(o.get_vext())
    xi = cases.xi_of(c, o.shape)
    fo, dfo, to = o.energy_grad(xi)
    f0, df0, t0 = e0.energy_and_gradient(xi)
    f1, df1, t1 = e1.energy_and_gradient(xi)
    w = e1.weights
    rho = xi ** 2 * e1.rho0
    dfid = np.where(rho > np.finfo(float).eps, w * 2 * e1.rho0 * xi * (SV.kT * np.log(rho / e1.rho0) + o.get_vext()), 0.0)
    exc_o, exc1 = dfo - dfid, df1 - dfid
    rel_exc = abs(t1[2] - to[2]) / abs(to[2])
    print("\n%s: F_exc rel err umma %.3e ffma %.3e; F rel err umma %.3e; excess df err / max umma %.3e ffma %.3e"
          % (name, rel_exc, abs(t0[2] - to[2]) / abs(to[2]), abs(f1 - fo) / abs(fo),
             np.abs(exc1 - exc_o).max() / np.abs(exc_o).max(), np.abs(df0 - dfid - exc_o).max() / np.abs(exc_o).max()))
    assert rel_exc <= 2e-5, (t1, to)
    assert abs(t1[2] - t0[2]) <= 2e-5 * abs(to[2]), (t1, t0)
    assert abs(f1 - fo) <= 2e-6 * abs(fo)
    assert np.abs(df1 - dfo).max() <= 1e-4 * np.abs(dfo).max()
    e0.close()
    e1.close()


@pytest.mark.parametrize("mode", ["ffma", "umma", "ring"])
def test_tensor_core_forms_in_a_mixed_solve(tmp_path, mode, monkeypatch):
    # The FP32 phase of a mixed solve (FP32 point, vext, gradient and direction) with each form
    # of the angular contractions: FFMA kernels, the tensor-core register forms, and the
    # tensor-core bulk-copy ring forms (the default at 24^3, no = 84).  Each solve's dG is
    # within 0.1 kJ/mol of the FP64 solve of the same solute (the metric's bar).
    c = cases.ALL_CASES["mol24_m3"]
    ck = cases.case_ck(tmp_path, c)
    sol = cases.solute_of(c)
    e64 = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0)
    r64 = e64.solve(sol, SV, rvdw=c["rvdw"], m=5, pgtol=1e-6, ftol_abs=-1.0, itermax=3000, guni_tol=0.01)
    e64.close()
    if mode == "ring":
        monkeypatch.delenv("MDFT_ANGULAR", raising=False)
    else:
        monkeypatch.setenv("MDFT_ANGULAR", mode)
    e32 = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=PREC_MIXED)
    r32 = e32.solve(sol, SV, rvdw=c["rvdw"], m=5, pgtol=1e-4, ftol_abs=-1.0, itermax=3000, precision=PREC_MIXED,
                    guni_tol=0.1)
    print("\n%s: dG %.6f (FP64 %.6f), FP32 evaluations %d, FP64 %d, status %d"
          % (mode, r32["dG"], r64["dG"], r32["evaluations_mixed"], r32["evaluations"], r32["status"]))
    assert r32["evaluations_mixed"] > 0
    assert abs(r32["dG"] - r64["dG"]) <= 0.1, (r32, r64)
    e32.close()


@pytest.mark.parametrize("name", ["ion16_m1", "mol16_m2", "mol24_m3", "mol8_m0", "mol64_m3", "mol32x128_m1"])
def test_oz_factored_rotations(tmp_path, name, monkeypatch):
    # The FP32 OZ with R(q) = e^{-i mu' alpha} D(q) (k_ozd, the default) against the kernel that
    # runs the reference's complex recursion (k_ozp, MDFT_OZ=ozp) and against the FP64 oracle,
    # at the mixed path's bars (energy 2e-6 of |F|, gradient 1e-4 of max|df|); the excess terms
    # of the two FP32 kernels agree to 1e-5 of |F_exc|.
    c = cases.ALL_CASES[name]
    ck = cases.case_ck(tmp_path, c)
    o = O.Oracle(c["n"], c["L"], c["mmax"], ck, SV.kT, SV.n0)
    o.compute_vext(cases.solute_of(c), SV, rvdw=c["rvdw"])
    monkeypatch.setenv("MDFT_OZ", "ozp")
    e0 = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=PREC_MIXED)
    monkeypatch.delenv("MDFT_OZ")
    e1 = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=PREC_MIXED)
    for e in (e0, e1):
        e.set_vext(o.get_vext())
    xi = cases.xi_of(c, o.shape)
    fo, dfo, to = o.energy_grad(xi)
    f0, df0, t0 = e0.energy_and_gradient(xi)
    f1, df1, t1 = e1.energy_and_gradient(xi)
    print("\n%s: F_exc oracle %.12g ozp %.12g ozd %.12g; df err ozd %.3e" % (name, to[2], t0[2], t1[2],
                                                                            np.abs(df1 - dfo).max() / np.abs(dfo).max()))
    assert abs(t1[2] - t0[2]) <= 1e-5 * abs(t0[2]), (t1, t0)
    assert abs(f1 - fo) <= 2e-6 * abs(fo)
    assert np.abs(df1 - dfo).max() <= 1e-4 * np.abs(dfo).max()
    e0.close()
    e1.close()


@pytest.mark.parametrize("precision", [0, PREC_MIXED])
def test_pipeline_graphs_match_direct_launches(tmp_path, precision, monkeypatch):
    # The evaluation pipeline replayed as CUDA graphs (the default) against direct launches
    # (MDFT_GRAPHS=0): the same solve, bit for bit (dG, iteration and evaluation counts), and
    # the same number of kernels counted.
    c = cases.ALL_CASES["mol24_m3"]
    ck = cases.case_ck(tmp_path, c)
    sol = cases.solute_of(c)
    opts = dict(m=5, pgtol=1e-4, ftol_abs=-1.0, itermax=3000, precision=precision, guni_tol=0.1)
    res = []
    for graphs in ("0", "1"):
        monkeypatch.setenv("MDFT_GRAPHS", graphs)
        e = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=precision)
        l0 = e.launch_count
        r = e.solve(sol, SV, rvdw=c["rvdw"], **opts)
        res.append((r["dG"], r["iterations"], r["evaluations"], r["evaluations_mixed"], e.launch_count - l0))
        e.close()
    monkeypatch.delenv("MDFT_GRAPHS")
    assert res[0] == res[1], res


@pytest.mark.parametrize("tune", ["1", "0"])
def test_autotuner_picks_measured_forms(tmp_path, tune, monkeypatch):
    # The autotuner times the default and the alternative FP32 forms when a mixed handle is
    # created (once per shape and device in a process) and keeps, stage by stage, the default
    # unless the alternative is more than 5 % faster;
    # with MDFT_AUTOTUNE=0 the defaults stay and nothing is measured.  Either way the solve
    # lands within 0.1 kJ/mol of the FP64 solve.
    c = cases.ALL_CASES["mol24_m3"]
    ck = cases.case_ck(tmp_path, c)
    sol = cases.solute_of(c)
    e64 = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0)
    r64 = e64.solve(sol, SV, rvdw=c["rvdw"], m=5, pgtol=1e-6, ftol_abs=-1.0, itermax=3000, guni_tol=0.01)
    e64.close()
    monkeypatch.delenv("MDFT_ANGULAR", raising=False)
    monkeypatch.delenv("MDFT_OZ", raising=False)
    monkeypatch.setenv("MDFT_AUTOTUNE", tune)
    e = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=PREC_MIXED)
    monkeypatch.delenv("MDFT_AUTOTUNE")
    kf = e.kernel_forms()
    r = e.solve(sol, SV, rvdw=c["rvdw"], m=5, pgtol=1e-4, ftol_abs=-1.0, itermax=3000, precision=PREC_MIXED, guni_tol=0.1)
    assert e.kernel_forms() == kf  # chosen at create, kept by the solve
    print("\nautotune %s: %s" % (tune, kf))
    if tune == "1":
        assert kf["tuned"]
        for stage, (m0, m1) in kf["stage_ms"].items():
            assert m0 > 0 and m1 > 0, (stage, m0, m1)
        ms = kf["stage_ms"]
        # the alternative (configuration 1) wins only when more than 5 % faster
        assert kf["project_ring"] == (ms["project"][1] < 0.95 * ms["project"][0])
        assert kf["gather_ring"] == (not ms["gather"][1] < 0.95 * ms["gather"][0])
        assert kf["oz_factored"] == (not ms["oz"][1] < 0.95 * ms["oz"][0])
    else:
        assert not kf["tuned"] and kf["gather_ring"] and not kf["project_ring"] and kf["oz_factored"]
        assert kf["stage_ms"] == {"project": [-1.0, -1.0], "oz": [-1.0, -1.0], "gather": [-1.0, -1.0]}
    assert abs(r["dG"] - r64["dG"]) <= 0.1, (r["dG"], r64["dG"])
    e.close()

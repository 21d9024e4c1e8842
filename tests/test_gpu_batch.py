"""Concurrent solves through mdft_solve_batch against one-at-a-time mdft_solve.

Every kernel reduces in a fixed order and each handle owns its buffers and stream, so a
solute solved inside a batch must give the same numbers as the same solute solved alone on
a handle of the same grid (compared to 1e-9 relative, i.e. up to the last digits only)."""
import numpy as np
import pytest

import cases
from mdft_b200 import Engine, PREC_MIXED, solve_batch, synth

pytestmark = pytest.mark.gpu
SV = cases.SOLVENT
OPTS = dict(m=5, pgtol=1e-5, ftol_abs=-1.0, itermax=2000)


def _solutes(L, seeds):
    out = []
    for sd in seeds:
        s = synth.random_walk_solute(5, seed=sd)
        s.xyz = synth.center_solute(s.xyz, (L,) * 3)
        out.append(s)
    return out


def _same(a, b):
    for k in ("dG", "f", "pmv", "deltaN"):
        assert abs(a[k] - b[k]) <= 1e-9 * max(1.0, abs(b[k])), (k, a[k], b[k])
    assert a["evaluations"] == b["evaluations"] and a["iterations"] == b["iterations"]


@pytest.mark.parametrize("precision", [0, PREC_MIXED])
def test_batch_matches_single_solves(tmp_path, precision):
    c = cases.CASES["mol16_m2"]
    ck = cases.ck_path(tmp_path, c["mmax"])
    sols = _solutes(c["L"], [31, 32, 33])
    engs = [Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=precision) for _ in range(2)]
    xo = [np.zeros(engs[0].shape) for _ in sols]
    got = solve_batch(engs, sols, SV, rvdw=c["rvdw"], precision=precision, xi_out=xo, **OPTS)
    ref = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=precision)
    for s, g, x in zip(sols, got, xo):
        xr = np.zeros(ref.shape)
        r = ref.solve(s, SV, rvdw=c["rvdw"], precision=precision, xi_out=xr, **OPTS)
        _same(g, r)
        assert np.abs(x - xr).max() <= 1e-9 * np.abs(xr).max()
    for e in engs + [ref]:
        e.close()


def test_batch_mixed_grids(tmp_path):
    # two handles on different grids and mmax; each solute pinned to one of them
    ca, cb = cases.CASES["mol16_m2"], cases.CASES["ion16_m1"]
    ea = Engine(ca["n"], ca["L"], ca["mmax"], cases.ck_path(tmp_path, ca["mmax"]), temperature=SV.temperature, n0=SV.n0)
    eb = Engine(cb["n"], cb["L"], cb["mmax"], cases.ck_path(tmp_path, cb["mmax"]), temperature=SV.temperature, n0=SV.n0)
    sa, sb = _solutes(ca["L"], [41, 42]), [cases.solute_of(cb)]
    got = solve_batch([ea, eb], sa + sb, SV, rvdw=min(ca["rvdw"], cb["rvdw"]), handles=[0, 0, 1], **OPTS)
    for s, g in zip(sa, got[:2]):
        _same(g, ea.solve(s, SV, rvdw=min(ca["rvdw"], cb["rvdw"]), **OPTS))
    _same(got[2], eb.solve(sb[0], SV, rvdw=min(ca["rvdw"], cb["rvdw"]), **OPTS))
    ea.close()
    eb.close()

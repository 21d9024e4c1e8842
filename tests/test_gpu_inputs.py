"""A solve set up from the reference's own input files (dft.in, solute.in) through the
library's readers gives the same result as the same system given directly."""
import numpy as np
import pytest

import cases
from mdft_b200 import Engine, inputs, synth

pytestmark = pytest.mark.gpu
SV = cases.SOLVENT


def test_solve_from_input_files(tmp_path):
    c = cases.CASES["mol16_m2"]
    ck = cases.ck_path(tmp_path, c["mmax"])
    (tmp_path / "dft.in").write_text(
        "# mol16_m2 as a dft.in\nboxnod = 16 16 16\nboxlen = 8. 8. 8.\nmmax = 2\ntemperature = %r\n"
        "rvdw = %r\ntranslate_solute_to_center = T\n" % (SV.temperature, c["rvdw"]))
    raw = synth.random_walk_solute(5, seed=c["seed"], radius=2.0)
    raw.write(str(tmp_path / "solute.in"))
    d = inputs.DftInput(str(tmp_path / "dft.in"))
    e = d.engine(ck, n0=SV.n0)
    sol = inputs.read_solute(str(tmp_path / "solute.in"), d.dp("solute_charges_scale_factor", 1.0))
    sol.xyz = inputs.center_solute(sol.xyz, e.box, d.log("translate_solute_to_center", True))
    opts = dict(m=5, pgtol=1e-5, ftol_abs=-1.0, itermax=2000)
    r1 = e.solve(sol, SV, rvdw=d.dp("rvdw", 10.0), **opts)
    ref = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0)
    # the same sites (as read from solute.in) given directly to an engine built without dft.in
    direct = synth.Solute(q=sol.q.copy(), sig=sol.sig.copy(), eps=sol.eps.copy(), xyz=sol.xyz.copy())
    assert np.allclose(sol.q, raw.q, atol=1e-10)
    r2 = ref.solve(direct, SV, rvdw=c["rvdw"], **opts)
    assert r1["evaluations"] == r2["evaluations"]
    assert abs(r1["dG"] - r2["dG"]) <= 1e-8 * max(1.0, abs(r2["dG"]))
    e.close()
    ref.close()
    d.close()

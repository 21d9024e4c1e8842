"""dft.in / solute.in readers of the library (host code, no GPU) against the restatement of
the reference's reading rules in oracle/inputs_ref.py, on fixtures that hit each rule."""
import os

import numpy as np
import pytest

from mdft_b200 import MdftError, inputs, synth
from oracle import inputs_ref as R

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DFT = os.path.join(GOLD, "dft_quirks.in")
SOL = os.path.join(GOLD, "solute_quirks.in")


@pytest.fixture(scope="module")
def dft():
    d = inputs.DftInput(DFT)
    yield d
    d.close()


def test_line_clean_up_matches_the_restatement(dft):
    text = open(DFT).read()
    assert max(len(l) for l in text.split("\n")) > 100  # one record is cut at 100 characters
    assert dft.lines == R.clean_lines(text)
    assert all("#" not in l for l in dft.lines)


@pytest.mark.parametrize("tag,n", [("boxnod", 3), ("mmax", 1), ("molrotsymorder", 1)])
def test_integers(dft, tag, n):
    ref = [R.int_of(t) for t in R.items_of(R.field_of(R.clean_lines(open(DFT).read()), tag))[:n]]
    got = dft.int(tag, n=n)
    assert (list(got) if n > 1 else [got]) == ref


def test_values_by_the_reference_rules(dft):
    assert dft.int("boxnod", n=3) == (64, 64, 48)
    assert dft.dp("boxlen", n=3) == (32.0, 32.0, 24.0)   # d and E exponents
    assert dft.int("mmax") == 3                          # first occurrence wins
    assert dft.dp("temperature", 300.0) == 300.0         # "temperature=298.15" does not carry the tag
    assert dft.int("molrotsymorder") == 2
    assert dft.dp("rvdw") == 8.5 and dft.dp("rvdw", n=2) == (8.5, 9.5)
    assert dft.dp("pressure", n=2) == (1.5, 1.5)         # repeat count
    assert dft.log("translate_solute_to_center") is False and dft.log("write_angular_density") is True
    assert dft.log("restart_missing", True) is True
    assert dft.char("solvent") == "spce"
    assert dft.dp("precision_factor") == 1.0             # the 9 after column 100 is cut off
    lines = R.clean_lines(open(DFT).read())
    for tag, n in (("boxlen", 3), ("rvdw", 2), ("pressure", 2), ("precision_factor", 1)):
        ref = tuple(R.real_of(t) for t in R.items_of(R.field_of(lines, tag))[:n])
        assert (dft.dp(tag, n=n) if n > 1 else (dft.dp(tag),)) == ref


def test_values_the_reference_rejects(dft):
    with pytest.raises(MdftError, match="logical"):
        dft.log("restart")                               # ".true." starts with '.'
    with pytest.raises(MdftError, match="integer"):
        dft.int("maximum_iteration_nbr")
    with pytest.raises(MdftError, match="nothing"):
        dft.char("bridge_tag_only")
    with pytest.raises(MdftError, match="not found"):
        dft.int("nb_solvent")


def test_desc_of_the_grid_tags(dft):
    a = dft.desc("ck.txt", n0=0.0333)
    assert a["n"] == (64, 64, 48) and a["box"] == (32.0, 32.0, 24.0) and a["mmax"] == 3 and a["mrso"] == 2
    assert a["temperature"] == 300.0


def test_desc_defaults(tmp_path):
    p = tmp_path / "dft.in"
    p.write_text("boxlen = 20. 20. 20.\n")
    d = inputs.DftInput(str(p))
    a = d.desc("ck.txt")
    assert a["n"] == (67, 67, 67) and a["mmax"] == 0 and a["mrso"] == 2 and a["temperature"] == 300.0
    d.close()


def test_solute_reader_matches_the_restatement():
    q, sg, ep, xyz, Z = R.read_solute(open(SOL).read(), scale=2.0)
    s = inputs.read_solute(SOL, charge_scale=2.0)
    assert s.nsite == 3
    assert np.array_equal(s.q, q) and np.array_equal(s.sig, sg) and np.array_equal(s.eps, ep)
    assert np.array_equal(s.xyz, np.array(xyz)) and list(s.Z) == Z
    assert s.xyz[1].tolist() == [-1.5, 0.5, -2.0] and list(s.Z) == [8, 1, 1]  # a site continued on the next line


def test_solute_written_by_synth_reads_back(tmp_path):
    sol = synth.random_walk_solute(7, seed=3)
    p = str(tmp_path / "solute.in")
    sol.write(p)
    s = inputs.read_solute(p)
    assert np.allclose(s.q, sol.q, atol=1e-10) and np.allclose(s.xyz, sol.xyz, atol=1e-10)


def test_center_solute_matches_the_restatement():
    rng = np.random.default_rng(4)
    xyz = rng.uniform(-40, 40, (9, 3))
    box = (32.0, 30.0, 24.0)
    for tr in (True, False):
        got = inputs.center_solute(xyz, box, tr)
        assert np.array_equal(got, np.array(R.center(xyz.tolist(), box, tr)))
        assert (got >= 0).all() and (got < np.array(box)).all()
    assert np.allclose(inputs.center_solute(xyz, box), synth.center_solute(xyz, box))


def test_missing_files():
    with pytest.raises(MdftError, match="cannot open"):
        inputs.DftInput("/nonexistent/dft.in")
    with pytest.raises(MdftError, match="cannot be opened"):
        inputs.read_solute("/nonexistent/solute.in")

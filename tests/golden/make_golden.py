"""Generate tests/golden/*.npz with the FP64 CPU oracle.

Run from the repository root:  python tests/golden/make_golden.py [case ...]
Each fixture stores, for one seeded case of tests/cases.py, the oracle's
F, {F_id, F_ext, F_exc, correction}, df at 128 seeded indices, sum(df) and
sum(df^2), and the vext checksum.  Inputs are regenerated from the seeds.
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "mdft-dev_general_b200"), os.path.join(ROOT, "tests")]

from oracle import oracle as O  # noqa: E402
import cases  # noqa: E402


def run_case(name, ckdir):
    c = cases.ALL_CASES[name]
    sv = cases.SOLVENT
    ck = cases.case_ck(ckdir, c)
    o = O.Oracle(c["n"], c["L"], c["mmax"], ck, sv.kT, sv.n0)
    sol = cases.solute_of(c)
    lj = 0.0
    if sol is not None:
        lj = o.compute_vext(sol, sv, rvdw=c["rvdw"])
    else:
        o.set_vext(cases.random_vext(c, o.shape))
    o.set_const_corr(cases.charge_correction(sol, c["L"]))
    vext = o.get_vext()
    xi = cases.xi_of(c, o.shape)
    f, df, terms = o.energy_grad(xi)
    rng = np.random.default_rng(7)
    idx = rng.integers(0, df.size, 128)
    return dict(f=f, terms=terms, idx=idx, df_samples=df.reshape(-1)[idx], df_sum=df.sum(), df_sq=(df * df).sum(),
                vext_sum=vext.sum(), vext_sq=(np.minimum(vext, 1e3) ** 2).sum(), lj_tail=lj)


def main(names):
    out = os.path.join(ROOT, "tests", "golden")
    with tempfile.TemporaryDirectory() as ckdir:
        for name in names or cases.ALL_CASES:
            r = run_case(name, ckdir)
            np.savez(os.path.join(out, name + ".npz"), **r)
            print(name, r["f"], r["terms"])


if __name__ == "__main__":
    main(sys.argv[1:])

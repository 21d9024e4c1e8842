"""Uneven batch: many solutes on different grids and angular orders solved concurrently.

64 seeded solutes of 1-40 sites (random walk as the 24-site workload), each on a grid drawn
from {32, 48, 64, 96}^3 with a box of 0.5 A x nodes and an mmax drawn from {1, 3}.  One
engine handle per (grid, mmax); each solute is pinned to its handle and mdft_solve_batch runs
the handles' solves concurrently.  Stop rule: max|df| <= 1e-4 and |sum w df dv| <= 0.1 kJ/mol.
Reported: aggregate solutes/s (wall clock around the batch call) and each solute's
|dG - dG_FP64|, the FP64 solve to max|df| <= 1e-6 (and |sum w df dv| <= 0.01) from the
bulk guess being the reference.  rvdw is 7.9 A for every solute: the 16 A box of the 32^3
grid allows at most 8 A (src/module_lennardjones.f90:55-59).

    python -m mdft_b200.uneven_batch [--solutes 64] [--report out.json]
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import engine as E
from . import synth

GRIDS = (32, 48, 64, 96)
MMAXES = (1, 3)
RVDW = 7.9
CK_SEED = 20260001


def draw(nsolutes: int, seed0: int = 60000000):
    """(seed, nsite, n, mmax) per solute, all from numpy's PCG64 seeded per solute."""
    out = []
    for i in range(nsolutes):
        rng = np.random.default_rng(seed0 + i)
        out.append((seed0 + i, int(rng.integers(1, 41)), int(rng.choice(GRIDS)), int(rng.choice(MMAXES))))
    return out


def solutes_of(plan):
    sols = []
    for seed, nsite, n, _ in plan:
        s = synth.random_walk_solute(nsite, seed)
        s.xyz = synth.center_solute(s.xyz, (0.5 * n,) * 3)
        sols.append(s)
    return sols


def run(plan, ck_dir, precision, pgtol, solvent, workers_per_combo=1, guni_tol=0.0):
    combos = sorted({(n, m) for _, _, n, m in plan})
    ck = {}
    for m in MMAXES:
        ck[m] = os.path.join(ck_dir, "ck_m%d.txt" % m)
        if not os.path.exists(ck[m]):
            synth.make_ck_file(ck[m], m, seed=CK_SEED, kmax=12.0)
    engines, index = [], {}
    for n, m in combos:
        index[(n, m)] = []
        for _ in range(workers_per_combo):
            index[(n, m)].append(len(engines))
            engines.append(E.Engine(n, 0.5 * n, m, ck[m], temperature=solvent.temperature, n0=solvent.n0,
                                    precision=precision))
    sols = solutes_of(plan)
    count = {}
    handles = []
    for _, _, n, m in plan:
        k = count.get((n, m), 0)
        handles.append(index[(n, m)][k % workers_per_combo])
        count[(n, m)] = k + 1
    t0 = time.perf_counter()
    res = E.solve_batch(engines, sols, solvent, rvdw=RVDW, m=5, pgtol=pgtol, ftol_abs=-1.0, itermax=5000,
                        precision=precision, handles=handles, guni_tol=guni_tol)
    wall = time.perf_counter() - t0
    for e in engines:
        e.close()
    return res, wall


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--solutes", type=int, default=64)
    ap.add_argument("--pgtol", type=float, default=1e-4)
    ap.add_argument("--guni-tol", type=float, default=0.1,
                    help="also stop only when |sum w df dv| <= this (kJ/mol; <= 0: off)")
    ap.add_argument("--workers-per-grid", type=int, default=1)
    ap.add_argument("--forms", default="mixed,fp64", help="forms to time, comma-separated: mixed, fp64")
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    solvent = synth.Solvent()
    plan = draw(a.solutes)
    d = tempfile.mkdtemp()
    forms = [f for f in a.forms.split(",") if f]
    out = {}
    for f in forms:
        prec = E.PREC_MIXED if f == "mixed" else E.PREC_FP64
        out[f] = run(plan, d, prec, a.pgtol, solvent, a.workers_per_grid, a.guni_tol)
    ref, t_ref = run(plan, d, E.PREC_FP64, 1e-6, solvent, a.workers_per_grid, 0.01)
    rows = []
    for i, (seed, nsite, n, m) in enumerate(plan):
        row = dict(seed=seed, nsite=nsite, n=n, mmax=m, dG_fp64=ref[i]["dG"])
        for f in forms:
            x = out[f][0][i]
            row.update({f + "_err": x["dG"] - ref[i]["dG"], f + "_evals": x["evaluations"] + x["evaluations_mixed"],
                        f + "_status": x["status"]})
        rows.append(row)
    summ = dict(solutes=len(plan), handles=len({(n, m) for _, _, n, m in plan}) * a.workers_per_grid, pgtol=a.pgtol,
                guni_tol=a.guni_tol,
                rvdw=RVDW, wall_s=dict({f: out[f][1] for f in forms}, fp64_ref_1e6=t_ref))
    for f in forms:
        errs = [abs(r[f + "_err"]) for r in rows]
        summ.update({f + "_solutes_per_s": len(plan) / out[f][1], f + "_max_abs_err": float(max(errs)),
                     f + "_over_0p1": int(sum(e > 0.1 for e in errs))})
    print(json.dumps(summ))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(dict(summary=summ, solutes=rows), f)


if __name__ == "__main__":
    main()

"""ΔG along an FP64 L-BFGS path of the C oracle for one solute of the uneven batch (TEST AND
ANALYSIS INFRASTRUCTURE ONLY: never imported by the product).  Per iteration: F, ΔG (with the
pressure correction of src/module_pressure_correction.f90:7-156), ΔN, max|df|, the L2 norm of df
and g_uni = sum_{r,io} w(io) df dv, the gradient along a uniform change of xi.

    python oracle/stop_rule_trace.py 60000013 > trace.jsonl
"""
import json
import os
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, 'tests'), os.path.join(ROOT, 'mdft-dev_general_b200')]
os.environ.setdefault("OMP_NUM_THREADS", "8")
import numpy as np
from scipy.optimize import minimize
from oracle import oracle as O
from mdft_b200 import synth
from mdft_b200 import uneven_batch as U

seed = int(sys.argv[1]) if len(sys.argv) > 1 else 60000013
plan = [p for p in U.draw(64) if p[0] == seed][0]
_, nsite, n, mmax = plan
sv = synth.Solvent()
ck = os.path.join(tempfile.gettempdir(), "stop_ck_m%d.txt" % mmax)
if not os.path.exists(ck):
    synth.make_ck_file(ck, mmax, seed=U.CK_SEED, kmax=12.0)
L = 0.5 * n
o = O.Oracle(n, L, mmax, ck, sv.kT, sv.n0)
sol = U.solutes_of([plan])[0]
lj = o.compute_vext(sol, sv, rvdw=U.RVDW)
xi0 = o.guess_density()
w = o.weights
dv, rho0 = o.dv, o.rho0
pc = o.pressure_correction(xi0, 0.0, lj)
pbulk = pc["pbulk"]
nwithout = sv.n0 * L ** 3
shape = xi0.shape
log = []
cache = {}
t0 = time.time()

def fg(x):
    f, df, _ = o.energy_grad(x.reshape(shape))
    cache["f"], cache["df"] = f, df
    return f, (df * dv).ravel()

def dG_of(x, f):
    nwith = float((x.reshape(shape) ** 2 * w).sum() * rho0 * dv)
    dN = nwithout - nwith
    return f + (-dN / sv.n0 * pbulk) + lj, dN

def cb(xk):
    f, df = cache["f"], cache["df"]
    g, dN = dG_of(xk, f)
    rec = dict(it=len(log), t=time.time() - t0, F=f, dG=g, dN=dN, gmax=float(np.abs(df).max()),
               g2=float(np.sqrt((df ** 2).sum() * dv)), guni=float((df * w).sum() * dv))
    log.append(rec)
    print(json.dumps(rec), flush=True)

r = minimize(fg, xi0.ravel(), jac=True, method="L-BFGS-B", callback=cb,
             options=dict(maxcor=5, gtol=1e-7, ftol=0.0, maxiter=400, maxfun=600))
print(json.dumps(dict(done=str(r.message), nit=int(r.nit), nfev=int(r.nfev))))


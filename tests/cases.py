"""Seeded test systems shared by the CPU and GPU tests and the golden fixtures.

A case is fully determined by its parameters: the c(k) file is regenerated
from its seed (numpy's PCG64 is reproducible), the solute from its seed, and
xi from its seed.  Nothing here reads the reference tree.
"""
from __future__ import annotations

import os

import numpy as np

from mdft_b200 import synth

SOLVENT = synth.Solvent()

CASES = {
    # name: grid n, box L, mmax, solute kind, solute seed, rvdw, xi seed
    "ion16_m1": dict(n=16, L=8.0, mmax=1, solute="ion", seed=1, rvdw=3.9, xseed=11),
    "mol16_m2": dict(n=16, L=8.0, mmax=2, solute="walk5", seed=2, rvdw=3.9, xseed=12),
    "rand12_m3": dict(n=12, L=6.0, mmax=3, solute="none", seed=3, rvdw=2.9, xseed=13),
    "mol24_m3": dict(n=24, L=12.0, mmax=3, solute="walk6", seed=4, rvdw=5.9, xseed=14),
    "mol8_m0": dict(n=8, L=4.0, mmax=0, solute="walk3", seed=5, rvdw=1.9, xseed=15),
    "rand8_m5": dict(n=8, L=4.0, mmax=5, solute="none", seed=6, rvdw=1.9, xseed=16, dk=0.1),
}


def ck_path(directory, mmax, kmax=14.0, dk=None, seed=20260000):
    if dk is None:
        dk = 0.1 if mmax >= 5 else 0.02
    path = os.path.join(str(directory), "ck_m%d_k%g_d%g_s%d.txt" % (mmax, kmax, dk, seed))
    if not os.path.exists(path):
        synth.make_ck_file(path, mmax, kmax=kmax, dk=dk, seed=seed)
    return path


def solute_of(case):
    kind = case["solute"]
    if kind == "ion":
        s = synth.ion_solute()
    elif kind.startswith("walk"):
        s = synth.random_walk_solute(int(kind[4:]), seed=case["seed"], radius=2.0)
    else:
        return None
    s.xyz = synth.center_solute(s.xyz, (case["L"],) * 3)
    return s


def xi_of(case, shape, amp=0.15):
    rng = np.random.default_rng(case["xseed"])
    return 1.0 + amp * rng.standard_normal(shape)


def random_vext(case, shape):
    rng = np.random.default_rng(case["seed"] + 100)
    return 0.8 * rng.standard_normal(shape)


def charge_correction(solute, L):
    if solute is None:
        return 0.0
    q = float(np.sum(solute.q))
    if abs(q) <= 1e-7:
        return 0.0
    pbc = -1971.01 * q * q / L * (1 - 1.0 / SOLVENT.eps_r)
    psch = -SOLVENT.quadrupole_trace * SOLVENT.n0 * 2909.857 * q
    return pbc + psch

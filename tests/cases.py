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

# The benchmark workloads and every FFT length the engine dispatches on: the single LJ ion
# (sigma 2.5, eps 0.5, q +1) at the centre of a 20 A box on 32^3 at mmax 1; a 24-site
# random-walk solute (6 A radius) in a 32 A box on 64^3 at mmax 3; the uneven batch's
# 48^3 and 96^3 grids (0.5 A spacing); a 128-long z axis.  c(k) tabulated with dk 0.01.
CONFIG_CASES = {
    "ion32_m1": dict(n=32, L=20.0, mmax=1, solute="ion", seed=21, rvdw=10.0, xseed=31, dk=0.01, kmax=12.0),
    "mol64_m3": dict(n=64, L=32.0, mmax=3, solute="walk24", seed=22, rvdw=10.0, xseed=32, dk=0.01, kmax=12.0,
                     radius=6.0),
    "mol48_m3": dict(n=48, L=24.0, mmax=3, solute="walk10", seed=23, rvdw=10.0, xseed=33, dk=0.01, kmax=12.0,
                     radius=6.0),
    "mol96_m1": dict(n=96, L=48.0, mmax=1, solute="walk12", seed=24, rvdw=10.0, xseed=34, dk=0.01, kmax=12.0,
                     radius=6.0),
    "mol32x128_m1": dict(n=(32, 32, 128), L=(16.0, 16.0, 64.0), mmax=1, solute="walk6", seed=25, rvdw=7.9,
                         xseed=35, dk=0.01, kmax=14.0, radius=4.0),
}

ALL_CASES = {**CASES, **CONFIG_CASES}


def ck_path(directory, mmax, kmax=14.0, dk=None, seed=20260000):
    if dk is None:
        dk = 0.1 if mmax >= 5 else 0.02
    path = os.path.join(str(directory), "ck_m%d_k%g_d%g_s%d.txt" % (mmax, kmax, dk, seed))
    if not os.path.exists(path):
        synth.make_ck_file(path, mmax, kmax=kmax, dk=dk, seed=seed)
    return path


def case_ck(directory, case):
    """The c(k) file of a case (its mmax, and its dk and kmax where it names them)."""
    return ck_path(directory, case["mmax"], kmax=case.get("kmax", 14.0), dk=case.get("dk"))


def box_of(case):
    L = case["L"]
    return tuple(L) if not np.isscalar(L) else (L,) * 3


def solute_of(case):
    kind = case["solute"]
    if kind == "ion":
        s = synth.ion_solute()
    elif kind.startswith("walk"):
        s = synth.random_walk_solute(int(kind[4:]), seed=case["seed"], radius=case.get("radius", 2.0))
    else:
        return None
    s.xyz = synth.center_solute(s.xyz, box_of(case))
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

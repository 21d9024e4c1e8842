"""Seeded synthetic inputs for the MDFT engine: water, direct correlation
functions c^{mn}_{mu nu chi}(k) written in Luc's file format, and solutes.

The reference reads c(k) from ``data/dcf/<solvent>/<solvent>-ck_nonzero_nmax<M>_ml``
(format: src/module_read_c_luc.f90:65-109 -- 10 comment lines, an ``alpha``
line, five index rows m, n, mu, nu, khi, a blank line, then rows
``q (re,im) (re,im) ...``).  The SPC/E files for nmax>=3 are not shipped with
the reference, so every c(k) used here is generated: c000 is the
Percus-Yevick hard-sphere direct correlation function times the solvent
number density (the reference normalises c by n0, src/module_energy_cproj_mrso.f90:728),
the other projections are seeded Gaussian-damped amplitudes that respect the
symmetries stated in the header of luc-files/ck_nmax1:5-7.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Sequence

import numpy as np

BOLTZ = 1.3806488e-23  # src/module_constants.f90:26
NAVO = 6.02214129e23  # src/module_constants.f90:24

# number of c(k) projections per mmax in Luc's files (src/module_solvent.f90:223)
NPLUC = {0: 1, 1: 6, 2: 75, 3: 252, 4: 877, 5: 2002}


def kT_of(temperature: float) -> float:
    """kT in kJ/mol (src/module_thermo.f90:62)."""
    return BOLTZ * NAVO * temperature * 1.0e-3


@dataclasses.dataclass
class Solvent:
    """Rigid 3-site water with O at the origin (the synthetic water of every workload)."""
    q: tuple = (-0.8476, 0.4238, 0.4238)
    sig: tuple = (3.166, 0.0, 0.0)
    eps: tuple = (0.65, 0.0, 0.0)
    xyz: tuple = ((0.0, 0.0, 0.0), (0.816497, 0.0, 0.577350), (-0.816497, 0.0, 0.577350))
    n0: float = 0.0333
    temperature: float = 298.0
    mrso: int = 2
    eps_r: float = 71.0

    @property
    def kT(self) -> float:
        return kT_of(self.temperature)

    @property
    def rho0(self) -> float:
        return self.n0 / (8.0 * math.pi ** 2 / self.mrso)

    @property
    def quadrupole_trace(self) -> float:
        """Trace of sum_s q_s r_s r_s (src/module_solvent.f90:323-326)."""
        return float(sum(q * (x * x + y * y + z * z) for q, (x, y, z) in zip(self.q, self.xyz)))


@dataclasses.dataclass
class Solute:
    q: np.ndarray
    sig: np.ndarray
    eps: np.ndarray
    xyz: np.ndarray  # (nsite, 3) Angstrom
    Z: np.ndarray | None = None

    @property
    def nsite(self) -> int:
        return int(len(self.q))

    @property
    def net_charge(self) -> float:
        return float(np.sum(self.q))

    def write(self, path: str) -> None:
        """solute.in format read at src/module_solute.f90:44-50."""
        Z = self.Z if self.Z is not None else np.zeros(self.nsite, dtype=int)
        with open(path, "w") as fh:
            fh.write("# synthetic solute\n%d\n# index q sigma epsilon x y z Z\n" % self.nsite)
            for i in range(self.nsite):
                fh.write("%d %.10f %.10f %.10f %.10f %.10f %.10f %d\n" % (
                    i + 1, self.q[i], self.sig[i], self.eps[i], *self.xyz[i], int(Z[i])))


def center_solute(xyz: np.ndarray, box: Sequence[float], translate: bool = True) -> np.ndarray:
    """mv_solute_to_center (src/module_solute.f90:146-187)."""
    out = np.array(xyz, dtype=np.float64, copy=True)
    L = np.asarray(box, dtype=np.float64)
    if translate:
        out = out + L / 2.0 - out.mean(axis=0)
    return np.mod(out, L)


# ----------------------------------------------------------------------------
# c(k)
def luc_tuples(mmax: int, mrso: int) -> list[tuple[int, int, int, int, int]]:
    """All (m, n, mu, nu, khi) of a Luc file: |mu|<=m, |nu|<=n in steps of mrso, |khi|<=min(m,n)."""
    out = []
    for m in range(mmax + 1):
        for n in range(mmax + 1):
            for mu in range(-(m // mrso) * mrso, m + 1, mrso):
                for nu in range(-(n // mrso) * mrso, n + 1, mrso):
                    for khi in range(-min(m, n), min(m, n) + 1):
                        out.append((m, n, mu, nu, khi))
    return out


def py_cq(k: np.ndarray, eta: float, sigma: float) -> np.ndarray:
    """Percus-Yevick hard-sphere direct correlation function c(k) in Angstrom^3.

    c(r) = -l1 - 6 eta l2 (r/s) - eta l1/2 (r/s)^3 for r < s (Wertheim/Thiele),
    transformed as 4 pi int c(r) r^2 sin(kr)/(kr) dr with 256-point Gauss-Legendre.
    """
    l1 = (1 + 2 * eta) ** 2 / (1 - eta) ** 4
    l2 = -(1 + eta / 2) ** 2 / (1 - eta) ** 4
    x, w = np.polynomial.legendre.leggauss(256)
    r = 0.5 * sigma * (x + 1.0)
    w = 0.5 * sigma * w
    cr = -l1 - 6 * eta * l2 * (r / sigma) - 0.5 * eta * l1 * (r / sigma) ** 3
    kr = np.outer(np.asarray(k, dtype=np.float64), r)
    j0 = np.where(kr > 1e-12, np.sin(kr) / np.where(kr > 1e-12, kr, 1.0), 1.0)
    return 4 * np.pi * (j0 * (cr * r * r * w)[None, :]).sum(axis=1)


def _symmetrise(tuples, vals, sign_tab):
    index = {t: i for i, t in enumerate(tuples)}
    v = vals.copy()
    for _ in range(4):
        # T1: c(m,n,-mu,-nu;khi) = (-1)^(m+n+mu+nu) conj(c(m,n,mu,nu;khi))
        w = v.copy()
        for i, (m, n, mu, nu, khi) in enumerate(tuples):
            j = index[(m, n, -mu, -nu, khi)]
            w[i] = 0.5 * (v[i] + sign_tab[(m + n + mu + nu) % 2] * np.conj(v[j]))
        v = w
        # T2: c(n,m,nu,mu;khi) = (-1)^(m+n) c(m,n,mu,nu;khi)
        w = v.copy()
        for i, (m, n, mu, nu, khi) in enumerate(tuples):
            j = index[(n, m, nu, mu, khi)]
            w[i] = 0.5 * (v[i] + sign_tab[(m + n) % 2] * v[j])
        v = w
        # T3 (C2v): c(m,n,-mu,-nu;khi) = c(m,n,mu,nu;-khi)
        w = v.copy()
        for i, (m, n, mu, nu, khi) in enumerate(tuples):
            j = index[(m, n, -mu, -nu, -khi)]
            w[i] = 0.5 * (v[i] + v[j])
        v = w
    return v


def synthetic_ck(mmax: int, mrso: int = 2, n0: float = 0.0333, seed: int = 20260000,
                 kmax: float = 50.0, dk: float = 0.01, eta: float = 0.45, sigma: float = 2.8,
                 amp: float = 0.2, margin: float = 0.5):
    """Return (q, tuples, values[nq, ntuple]) of a synthetic c^{mn}_{mu nu khi}(k).

    c000 = n0 * c_PY(k).  Every other projection is a_t g_t(k) with
    |a_t| <= amp*|c000(0)| drawn from ``seed`` and a Gaussian envelope
    g_t(k) = exp(-(k l_t)^2/2), l_t in [1, 2) Angstrom; projections with mu or
    nu != 0 use g_t(k) = (k l_t)^2 exp(1-(k l_t)^2/2)/2 instead, which vanishes at
    k=0 (as in the reference's SPC/E tables: the k=0 point is handled in a fixed
    frame, and a frame-dependent c there would make the functional's gradient
    inconsistent with its energy).  The coefficients are projected
    onto the symmetric subspace, then all non-000 amplitudes are scaled by one
    factor so that, for every k and khi, the Hermitian part of the matrix
    [c^{mn}_{mu nu khi}(k)]_{(m,mu),(n,nu)} has all eigenvalues <= 1 - margin
    (1 - rho c positive definite in the file's normalisation).
    """
    tuples = luc_tuples(mmax, mrso)
    nt = len(tuples)
    q = np.arange(0, int(round(kmax / dk)) + 1) * dk
    c000 = n0 * py_cq(q, eta, sigma)
    rng = np.random.default_rng(seed)
    sign_tab = {0: 1.0, 1: -1.0}
    # orbit-invariant envelope width
    def orbit_key(t):
        m, n, mu, nu, khi = t
        a, b = sorted([(m, abs(mu)), (n, abs(nu))])
        return (a, b, abs(khi))
    keys = sorted({orbit_key(t) for t in tuples})
    widths = {k: 1.0 + rng.random() for k in keys}
    a = (rng.standard_normal(nt) + 1j * rng.standard_normal(nt))
    a = a / np.maximum(1.0, np.abs(a)) * amp * abs(c000[0]) * rng.random(nt)
    i000 = tuples.index((0, 0, 0, 0, 0))
    a[i000] = 0.0
    a = _symmetrise(tuples, a, sign_tab)
    # eigenvalue control on a coarse k grid (the envelopes are smooth)
    tindex = {t: i for i, t in enumerate(tuples)}
    blocks = []
    for khi in range(-mmax, mmax + 1):
        basis = [(m, mu) for m in range(abs(khi), mmax + 1) for mu in range(-(m // mrso) * mrso, m + 1, mrso)]
        blocks.append(np.array([[tindex[(m, n, mu, nu, khi)] for (n, nu) in basis] for (m, mu) in basis]))
    kcheck = np.arange(0.0, 50.0 + 1e-9, 0.125)  # fixed: the table values do not depend on kmax
    wvec = np.array([widths[orbit_key(t)] for t in tuples])
    vanish = np.array([t[2] != 0 or t[3] != 0 for t in tuples])

    def envelope(k):
        x2 = (k[:, None] * wvec[None, :]) ** 2
        return np.where(vanish[None, :], 0.5 * x2 * np.exp(1.0 - 0.5 * x2), np.exp(-0.5 * x2))
    envk = envelope(kcheck)
    c000k = n0 * py_cq(kcheck, eta, sigma)
    scale = 1.0
    for _ in range(60):
        worst = -np.inf
        for ik in range(len(kcheck)):
            vals = scale * a * envk[ik]
            vals[i000] = c000k[ik]
            for idx in blocks:
                Mx = vals[idx]
                worst = max(worst, float(np.linalg.eigvalsh(0.5 * (Mx + Mx.conj().T)).max()))
        if worst <= 1.0 - margin:
            break
        scale *= 0.7
    vals = (scale * a[None, :] * envelope(q)).astype(np.complex128)
    vals[:, i000] = c000
    return q, tuples, vals


def write_luc_file(path: str, q: np.ndarray, tuples, vals: np.ndarray, title: str = "synthetic c(k)") -> None:
    """Write c(k) in the layout parsed by src/module_read_c_luc.f90:65-109."""
    nt = len(tuples)
    with open(path, "w") as fh:
        fh.write("# %s\n" % title)
        for _ in range(9):
            fh.write("#\n")
        fh.write(" alpha " + " ".join("%d" % (i + 1) for i in range(nt)) + "\n")
        for lab, col in zip(("m", "n", "mu", "nu", "khi"), range(5)):
            fh.write(" %s " % lab + " ".join("%d" % t[col] for t in tuples) + "\n")
        fh.write("\n")
        for iq in range(len(q)):
            row = ["%.17e" % q[iq]]
            for v in vals[iq]:
                row.append("(%.17e,%.17e)" % (v.real, v.imag))
            fh.write(" ".join(row) + "\n")


def make_ck_file(path: str, mmax: int, mrso: int = 2, n0: float = 0.0333, seed: int = 20260000,
                 kmax: float = 50.0, dk: float = 0.01) -> str:
    q, tuples, vals = synthetic_ck(mmax, mrso=mrso, n0=n0, seed=seed, kmax=kmax, dk=dk)
    write_luc_file(path, q, tuples, vals, title="synthetic c(k) mmax=%d mrso=%d seed=%d" % (mmax, mrso, seed))
    return path


# ----------------------------------------------------------------------------
# solutes
def ion_solute(sig=2.5, eps=0.5, q=1.0) -> Solute:
    """Single LJ ion (one site)."""
    return Solute(q=np.array([q]), sig=np.array([sig]), eps=np.array([eps]), xyz=np.zeros((1, 3)))


def random_walk_solute(nsite: int, seed: int, radius: float = 6.0, bond=(1.4, 1.6), sig=(2.5, 3.8),
                       eps=(0.2, 1.0), qsd: float = 0.3, min_sep: float = 1.2) -> Solute:
    """Sites by random walk with bonds U[bond] inside a sphere; q ~ N(0, qsd) shifted to sum 0."""
    rng = np.random.default_rng(seed)
    xyz = [np.zeros(3)]
    tries = 0
    while len(xyz) < nsite:
        tries += 1
        if tries > 100000:
            raise RuntimeError("random walk could not place all sites")
        base = xyz[rng.integers(len(xyz))] if tries % 20 == 0 else xyz[-1]
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        p = base + v * rng.uniform(*bond)
        if np.linalg.norm(p) > radius:
            continue
        if min(np.linalg.norm(p - s) for s in xyz) < min_sep:
            continue
        xyz.append(p)
    q = rng.normal(0.0, qsd, nsite)
    q -= q.mean()
    return Solute(q=q, sig=rng.uniform(*sig, nsite), eps=rng.uniform(*eps, nsite), xyz=np.array(xyz))


def packed_cluster_solute(nsite: int, seed: int, radius: float = 15.0, min_sep: float = 3.0, sig=(3.0, 3.9),
                          eps=(0.3, 0.9), charged_frac: float = 0.2, qabs: float = 0.5) -> Solute:
    """Sites by rejection sampling at >= min_sep spacing inside a sphere; +-qabs charges on a fraction, net 0."""
    rng = np.random.default_rng(seed)
    pts = []
    tries = 0
    while len(pts) < nsite:
        tries += 1
        if tries > 5_000_000:
            raise RuntimeError("rejection sampling could not place all sites")
        p = rng.uniform(-radius, radius, 3)
        if np.linalg.norm(p) > radius:
            continue
        if pts and np.min(np.linalg.norm(np.array(pts) - p, axis=1)) < min_sep:
            continue
        pts.append(p)
    q = np.zeros(nsite)
    nch = int(round(charged_frac * nsite)) // 2 * 2
    idx = rng.permutation(nsite)[:nch]
    q[idx[: nch // 2]] = qabs
    q[idx[nch // 2:]] = -qabs
    return Solute(q=q, sig=rng.uniform(*sig, nsite), eps=rng.uniform(*eps, nsite), xyz=np.array(pts))

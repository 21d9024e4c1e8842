"""Known-answer tests that pin the FP64 oracle to the reference's own checks."""
import os

import numpy as np
import pytest

from oracle import oracle as O
import cases

REF = "/root/reference"


def test_wigner_closed_forms():
    # the 13 closed forms of tools/test_function_harm_sph_de_luc.f90:23-35 at 20 random angles
    rng = np.random.default_rng(2024)
    for th in rng.random(20) * np.pi:
        c, s = np.cos(th), np.sin(th)
        forms = {
            (1, 0, 0): c, (1, 1, 1): (1 + c) / 2, (1, 1, 0): -s / np.sqrt(2), (1, 1, -1): (1 - c) / 2,
            (2, 2, 2): ((1 + c) / 2) ** 2, (2, 2, 1): -(1 + c) / 2 * s, (2, 2, 0): np.sqrt(6) / 4 * s ** 2,
            (2, 2, -1): -(1 - c) / 2 * s, (2, 2, -2): ((1 - c) / 2) ** 2, (2, 1, 1): (1 + c) / 2 * (2 * c - 1),
            (2, 1, 0): -np.sqrt(1.5) * s * c, (2, 1, -1): (1 - c) / 2 * (2 * c + 1), (2, 0, 0): 1.5 * c ** 2 - 0.5,
        }
        for (m, mu, mup), v in forms.items():
            assert abs(O.wigner_small_d(m, mu, mup, th) - v) < 1e-14


def test_gauss_legendre_matches_numpy():
    for n in range(1, 8):
        x, w = O.gauss_legendre(n)
        xr, wr = np.polynomial.legendre.leggauss(n)
        np.testing.assert_allclose(np.sort(x), np.sort(xr), atol=1e-15)
        np.testing.assert_allclose(np.sort(w), np.sort(wr / 2), atol=1e-15)
        assert abs(w.sum() - 1) < 1e-15


@pytest.mark.parametrize("mmax,np_,no,ncoef", [(1, 4, 6, 6), (2, 14, 45, 56), (3, 28, 84, 178)])
def test_sizes_and_quadrature(tmp_path, mmax, np_, no, ncoef):
    ck = cases.ck_path(tmp_path, mmax, kmax=14.0)
    o = O.Oracle(8, 4.0, mmax, ck, 2.477, 0.0333)
    assert (o.np, o.no, o.ncoef) == (np_, no, ncoef)
    # src/module_grid.f90:147-154: the weights sum to 8 pi^2 / mrso
    assert abs(o.weights.sum() - 8 * np.pi ** 2 / 2) < 1e-12


def test_sizes_mmax5(tmp_path):
    ck = cases.ck_path(tmp_path, 5, kmax=14.0, dk=0.1)
    o = O.Oracle(8, 4.0, 5, ck, 2.477, 0.0333)
    assert (o.np, o.no, o.ncoef) == (88, 330, 1268)


def test_rotation_matrix_identities():
    # q along +z: the q-frame is the lab frame -> identity
    R = O.rotation_matrix(4, [0.0, 0.0, 1.3])
    for m in range(5):
        blk = R[m, 4 - m:4 + m + 1, 4 - m:4 + m + 1]
        np.testing.assert_allclose(blk, np.eye(2 * m + 1), atol=1e-15)
    # unitarity of every block for random q
    rng = np.random.default_rng(5)
    for _ in range(10):
        q = rng.standard_normal(3)
        R = O.rotation_matrix(5, q)
        for m in range(6):
            blk = R[m, 5 - m:5 + m + 1, 5 - m:5 + m + 1]
            np.testing.assert_allclose(blk @ blk.conj().T, np.eye(2 * m + 1), atol=1e-13)


def test_projection_round_trip(tmp_path):
    # proj2angl(angl2proj(o)) == o for an orientation field of band mmax
    for mmax in (1, 2, 3):
        ck = cases.ck_path(tmp_path, mmax, kmax=14.0)
        o = O.Oracle(8, 4.0, mmax, ck, 2.477, 0.0333)
        rng = np.random.default_rng(mmax)
        p = rng.standard_normal(o.np) + 1j * rng.standard_normal(o.np)
        f = o.proj2angl(p)          # a real, band-limited field
        p2 = o.angl2proj(f)
        f2 = o.proj2angl(p2)
        np.testing.assert_allclose(f2, f, atol=1e-12 * np.abs(f).max())


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not mounted")
def test_reads_reference_spce_table():
    # the reference's own SPC/E c(k) table parses, with its dq and c000(0)
    ck = os.path.join(REF, "data/dcf/spce/spce-ck_nonzero_nmax1_ml")
    o = O.Oracle(16, 12.0, 1, ck, 2.477, 0.0333)
    assert abs(o.dq - 0.0613592315) < 1e-9
    c = o.ctable()
    # (m,khi,mu2,n,nu2) = (0,0,0,0,0) is the first coefficient: conj and sign (+1) applied
    assert abs(c[0, 0] - (-13.6652260 + 0j)) < 1e-6

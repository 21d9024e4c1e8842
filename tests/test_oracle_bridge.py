"""The oracle's coarse-grained bridge (bridge = "cgb") on the CPU.

* 'sla' (src/module_coarse_grained_gageat_bridge.f90:274-347): the gradient the reference
  writes is the derivative of its F_b -- central differences agree to 1e-6 relative.
* 'wda' (:349-419): the reference convolves Phi' before multiplying by (n - 1), so its
  gradient is not the derivative of its F_b; the oracle keeps that (differences disagree).
* At the bulk density (xi = 1 everywhere) n_cg = 1 up to the discretised Gaussian's sum:
  F_b and the gradient nearly vanish.
* energy_and_gradient with the bridge set = without it + the seam's F_b and gradient.
"""
import numpy as np
import pytest

from oracle import oracle as O
import cases

SV = cases.SOLVENT


def system(tmp_path, mmax=2, n=16, L=8.0):
    c = dict(n=n, L=L, mmax=mmax, solute="none", seed=3, rvdw=2.9, xseed=13)
    o = O.Oracle(n, L, mmax, cases.ck_path(tmp_path, mmax), SV.kT, SV.n0)
    o.set_vext(cases.random_vext(c, o.shape))
    xi = cases.xi_of(c, o.shape, amp=0.3)
    return o, xi


def fd_check(o, xi, seed=0, h=1e-6):
    g = np.zeros(o.shape)
    o.bridge_energy(xi, g)
    d = np.random.default_rng(seed).standard_normal(o.shape)
    fd = (o.bridge_energy(xi + h * d) - o.bridge_energy(xi - h * d)) / (2 * h)
    return fd, float(np.sum(g * d) * o.dv)


def test_sla_gradient_is_the_derivative(tmp_path):
    o, xi = system(tmp_path)
    o.set_bridge_cgb(1, B6=5.0, sigma=1.0, c00=-13.665)
    fd, an = fd_check(o, xi)
    assert abs(fd - an) <= 1e-6 * abs(fd), (fd, an)


def test_wda_gradient_follows_the_reference_not_the_derivative(tmp_path):
    o, xi = system(tmp_path)
    o.set_bridge_cgb(2, B6=5.0, sigma=1.0, c00=-13.665)
    fd, an = fd_check(o, xi)
    assert abs(fd - an) > 0.1 * abs(fd), (fd, an)


@pytest.mark.parametrize("version", [1, 2])
def test_bulk_density_has_no_bridge(tmp_path, version):
    o, _ = system(tmp_path)
    o.set_bridge_cgb(version, B6=5.0, sigma=1.0, c00=-13.665)
    xi = np.ones(o.shape)
    g = np.zeros(o.shape)
    fb = o.bridge_energy(xi, g)
    # against |F_b| of about 0.24 with 30 % density noise
    assert abs(fb) < 1e-6
    assert np.abs(g).max() < 1e-6


@pytest.mark.parametrize("version", [1, 2])
def test_energy_and_gradient_adds_the_bridge(tmp_path, version):
    o, xi = system(tmp_path)
    f0, df0, t0 = o.energy_grad(xi)
    o.set_bridge_cgb(version, B6=3.0, sigma=1.2, c00=-11.9078)
    f1, df1, t1 = o.energy_grad(xi)
    g = df0.copy()
    fb = o.bridge_energy(xi, g)
    assert f1 == f0 + fb or abs(f1 - (f0 + fb)) <= 1e-14 * abs(f1)
    assert np.array_equal(t1, t0)
    np.testing.assert_allclose(df1, g, rtol=0, atol=1e-14 * np.abs(g).max())
    o.set_bridge_cgb(0)
    f2, _, _ = o.energy_grad(xi)
    assert f2 == f0


# ---- bridge = "hard_sphere" (src/module_fmt.f90) ------------------------------------------

@pytest.mark.parametrize("functional", [1, 2])
def test_fmt_bulk_parameters_match_the_closed_forms(tmp_path, functional):
    # the Kierlik-Rosinberg functional reproduces the Percus-Yevick (compressibility) and
    # Carnahan-Starling equations of state: beta mu_exc and the excess free energy per
    # particle in closed form in the packing fraction eta
    o, _ = system(tmp_path)
    R = 1.4
    o.set_bridge_fmt(functional, R)
    r, mu, fexc0, nbk = o.fmt_params()
    eta = 4.0 / 3.0 * np.pi * SV.n0 * R ** 3
    if functional == 1:
        bmu = -np.log(1 - eta) + eta * (14 - 13 * eta + 5 * eta ** 2) / (2 * (1 - eta) ** 3)
        bf = -np.log(1 - eta) + 3 * eta * (2 - eta) / (2 * (1 - eta) ** 2)
    else:
        bmu = eta * (8 - 9 * eta + 3 * eta ** 2) / (1 - eta) ** 3
        bf = eta * (4 - 3 * eta) / (1 - eta) ** 2
    assert abs(mu / SV.kT - bmu) <= 1e-12 * bmu
    V = 8.0 ** 3
    # Fexc0 = (f_exc - mu n0) V, so f_exc / n0 = Fexc0 / (V n0) + mu
    assert abs((fexc0 / (V * SV.n0) + mu) / SV.kT - bf) <= 1e-12 * bf
    assert nbk > 1


@pytest.mark.parametrize("functional", [1, 2])
def test_fmt_gradient_is_the_derivative(tmp_path, functional):
    # the energy's weights are the reference's single-precision cmplx(w_k, 0), the gradient's
    # are not (module_fmt.f90:92 against :170-174): agreement to 1e-5, not to rounding
    o, xi = system(tmp_path)
    o.set_bridge_fmt(functional, 1.4)
    fd, an = fd_check(o, xi, h=1e-4)
    assert abs(fd - an) <= 1e-5 * abs(fd), (fd, an)


@pytest.mark.parametrize("functional", [1, 2])
def test_fmt_bulk_and_empty_box(tmp_path, functional):
    o, _ = system(tmp_path)
    o.set_bridge_fmt(functional, 1.4)
    fexc0 = o.fmt_params()[2]
    # bulk: the functional is shifted to vanish there (up to the single-precision weights)
    assert abs(o.bridge_energy(np.ones(o.shape))) < 1e-4
    # empty box (every |xi| <= epsilon): -Fexc0 and no gradient (:46-49)
    g = np.zeros(o.shape)
    assert o.bridge_energy(np.zeros(o.shape), g) == -fexc0
    assert not g.any()
    # a weighted density n3 >= 1 stops the reference; the oracle reports it
    with pytest.raises(RuntimeError, match="w3"):
        o.bridge_energy(3.0 * np.ones(o.shape))

"""Physics checks of the oracle: normalisation of the excess term, gradient
consistency and symmetry of the excess operator."""
import numpy as np
import pytest

from oracle import oracle as O
import cases

SV = cases.SOLVENT


@pytest.fixture(autouse=True)
def _reset_quirks():
    yield
    O.set_quirks(3)


@pytest.mark.parametrize("mmax", [0, 1, 3])
def test_uniform_density_kat(tmp_path, mmax):
    # uniform xi: F_exc = -(kT/2) V dn^2 c000(0)/n0 and F_id = kT V n0 (x ln x - x + 1), x = xi^2
    ck = cases.ck_path(tmp_path, mmax)
    o = O.Oracle(12, 6.0, mmax, ck, SV.kT, SV.n0)
    xi0 = 1.07
    V = 6.0 ** 3
    x = xi0 ** 2
    c000 = o.ctable()[0, 0].real
    dn = SV.n0 * (x - 1)
    want = -(SV.kT / 2) * V * dn ** 2 * c000 / SV.n0
    # the k=0 gamma is real, so the reference's flush rounds it to FP32 (1e-7 relative)
    for quirks, tol in ((0, 1e-11), (3, 1e-7)):
        O.set_quirks(quirks)
        f, df, t = o.energy_grad(np.full(o.shape, xi0))
        assert abs(t[2] - want) < tol * abs(want)
        assert abs(t[0] - SV.kT * V * SV.n0 * (x * np.log(x) - x + 1)) < 1e-10 * abs(t[0])
        assert t[1] == 0.0


@pytest.mark.parametrize("mmax", [1, 2, 3])
def test_gradient_matches_finite_differences(tmp_path, mmax):
    # dF/dxi = dv * df.  Without the reference's FP32 roundings the match is exact to FD error;
    # with them (default) F is a staircase at the 1e-8 relative level.
    ck = cases.ck_path(tmp_path, mmax)
    o = O.Oracle(8, 4.0, mmax, ck, SV.kT, SV.n0)
    rng = np.random.default_rng(mmax)
    o.set_vext(0.5 * rng.standard_normal(o.shape))
    xi = 1.0 + 0.1 * rng.standard_normal(o.shape)
    for quirks, tol in ((0, 1e-8), (3, 1e-4)):
        O.set_quirks(quirks)
        f, df, _ = o.energy_grad(xi)
        scale = np.abs(df).max() * o.dv
        for _ in range(6):
            idx = tuple(rng.integers(0, s) for s in o.shape)
            h = 1e-4
            xp = xi.copy(); xp[idx] += h
            xm = xi.copy(); xm[idx] -= h
            fd = (o.energy_grad(xp, False)[0] - o.energy_grad(xm, False)[0]) / (2 * h)
            assert abs(fd - o.dv * df[idx]) < tol * scale


def test_charge_corrections_values():
    # module_energy_and_gradient.f90:313,342 for a +1 ion in a 20 A box
    c = O.charge_corrections(1.0, 20.0, 71.0, SV.quadrupole_trace, SV.n0)
    pbc = -1971.01 / 20.0 * (1 - 1 / 71.0)
    psch = -SV.quadrupole_trace * SV.n0 * 2909.857
    assert abs(c - (pbc + psch)) < 1e-12
    assert O.charge_corrections(0.0, 20.0, 71.0, 0.8, SV.n0) == 0.0


@pytest.mark.parametrize("mmax", [1, 2, 3])
def test_projections_of_a_real_field_are_hermitian(tmp_path, mmax):
    # p(m, -mu', 0) = (-1)^mu' conj p(m, mu', 0) for any real o(omega): the reference's sign
    # and conjugation conventions (angl2proj, src/module_orientation_projection_transform.f90:159-199)
    # with d^m_{-mu',0} = (-1)^mu' d^m_{mu',0}
    o = O.Oracle(8, 4.0, mmax, cases.ck_path(tmp_path, mmax), 2.477, 0.0333)
    plist = [(m, mup, mu) for m in range(mmax + 1) for mup in range(-m, m + 1) for mu in range(0, m + 1, 2)]
    idx = {t: i for i, t in enumerate(plist)}
    assert len(plist) == o.np
    for seed in range(3):
        p = o.angl2proj(np.random.default_rng(seed).uniform(0.0, 2.0, o.no))
        for m, mup, mu in plist:
            if mu == 0:
                assert abs(p[idx[(m, -mup, 0)]] - (-1) ** mup * np.conj(p[idx[(m, mup, 0)]])) < 1e-14

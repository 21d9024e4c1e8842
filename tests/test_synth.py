"""Synthetic c(k): layout, symmetries, stability margin, and file round trip."""
import numpy as np
import pytest

from mdft_b200 import synth


@pytest.mark.parametrize("mmax", [0, 1, 2, 3, 4, 5])
def test_tuple_counts_match_npluc(mmax):
    assert len(synth.luc_tuples(mmax, 2)) == synth.NPLUC[mmax]


@pytest.mark.parametrize("mmax", [1, 2, 3])
def test_symmetries_and_margin(mmax):
    q, tuples, V = synth.synthetic_ck(mmax, kmax=10.0, dk=0.05)
    T = {t: i for i, t in enumerate(tuples)}
    s = lambda k: -1.0 if k % 2 else 1.0
    for i, (m, n, mu, nu, khi) in enumerate(tuples):
        # luc-files/ck_nmax1:5-7
        np.testing.assert_allclose(V[:, i], s(m + n + mu + nu) * np.conj(V[:, T[(m, n, -mu, -nu, khi)]]), atol=1e-14)
        np.testing.assert_allclose(V[:, i], s(m + n) * V[:, T[(n, m, nu, mu, khi)]], atol=1e-14)
        np.testing.assert_allclose(V[:, i], V[:, T[(m, n, -mu, -nu, -khi)]], atol=1e-14)
        if mu != 0 or nu != 0:
            assert V[0, i] == 0  # vanishes at k = 0
    # 1 - c positive definite per (k, khi) block, with the margin of 0.1
    for ik in range(0, len(q), 7):
        for khi in range(-mmax, mmax + 1):
            basis = [(m, mu) for m in range(abs(khi), mmax + 1) for mu in range(-(m // 2) * 2, m + 1, 2)]
            M = np.array([[V[ik, T[(m, n, mu, nu, khi)]] for (n, nu) in basis] for (m, mu) in basis])
            assert np.linalg.eigvalsh(0.5 * (M + M.conj().T)).max() <= 0.9 + 1e-12


def test_file_round_trip(tmp_path):
    q, tuples, V = synth.synthetic_ck(1, kmax=2.0, dk=0.1)
    p = tmp_path / "ck.txt"
    synth.write_luc_file(str(p), q, tuples, V)
    lines = p.read_text().splitlines()
    assert lines[10].split()[0] == "alpha" and lines[16] == ""
    row = lines[17 + 3].replace("(", " ").replace(")", " ").replace(",", " ").split()
    assert float(row[0]) == pytest.approx(q[3])
    np.testing.assert_allclose([float(row[1]), float(row[2])], [V[3, 0].real, V[3, 0].imag])


def test_solute_generators():
    s = synth.random_walk_solute(24, seed=1)
    assert s.nsite == 24 and abs(s.q.sum()) < 1e-12
    assert np.linalg.norm(s.xyz, axis=1).max() <= 6.0
    c = synth.packed_cluster_solute(50, seed=2)
    d = np.linalg.norm(c.xyz[:, None] - c.xyz[None], axis=2) + 1e9 * np.eye(50)
    assert d.min() >= 3.0 and abs(c.q.sum()) < 1e-12
    x = synth.center_solute(s.xyz, (32.0,) * 3)
    assert np.all((x >= 0) & (x < 32.0))


def test_uneven_batch_plan():
    from mdft_b200 import uneven_batch as U
    plan = U.draw(64)
    assert plan == U.draw(64)
    assert {n for _, _, n, _ in plan} == set(U.GRIDS) and {m for _, _, _, m in plan} == set(U.MMAXES)
    assert all(1 <= k <= 40 for _, k, _, _ in plan)
    for s, (_, k, n, _) in zip(U.solutes_of(plan), plan):
        assert s.nsite == k and (s.xyz >= 0).all() and (s.xyz < 0.5 * n).all()
        assert 0.5 * n / 2 >= U.RVDW  # the reference's cut-off check holds on every grid

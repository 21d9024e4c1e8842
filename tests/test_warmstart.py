"""Learned warm start, CPU side: the oracle's definitions and the host logic.

The network's GPU kernels are checked against oracle/warmnet_ref.py in
test_gpu_warmnet.py; here the oracle itself is pinned (its BF16 rounding against torch's,
the exactness of the m <= 1 projections on the solver's quadrature, the channels'
symmetries), and the library's argument checks run without a GPU."""
import ctypes

import numpy as np
import pytest
import torch

import cases
from mdft_b200 import engine, synth, warmstart
from oracle import oracle as O
from oracle import warmnet_ref as W


def test_parameter_count_and_layout():
    assert W.num_params() == 906772
    flat = torch.arange(W.num_params(), dtype=torch.float64)
    parts = W.unpack(flat, torch)
    assert parts[0][0].shape == (16, 3, 3, 3, 3) and parts[8][0].shape == (128, 64, 2, 2, 2)
    assert parts[-1][0].shape == (4, 16, 1, 1, 1) and parts[-1][1].shape == (4,)


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.standard_normal(10000).astype(np.float32) * 10.0 ** rng.integers(-6, 6, 10000),
                        np.array([1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -0.0, 65504.0], np.float32)])
    ref = torch.tensor(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(W.bf16_round(x), ref)
    assert np.array_equal(warmstart.bf16_round(x), ref)


def test_parameter_file_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    p = rng.standard_normal(1000).astype(np.float32)
    path = str(tmp_path / "w.npz")
    warmstart.save_params(path, p, dict(note="x"))
    q, meta = warmstart.load_params(path)
    assert meta == dict(note="x", nout=4)  # files without an output count are the m <= 1 form
    assert np.array_equal(q, W.bf16_round(p))


@pytest.fixture(scope="module")
def grid16(tmp_path_factory):
    c = cases.CASES["mol16_m2"]
    ck = cases.ck_path(tmp_path_factory.mktemp("ck"), c["mmax"])
    sv = cases.SOLVENT
    o = O.Oracle(c["n"], c["L"], c["mmax"], ck, sv.kT, sv.n0)
    return c, o


def test_projections_are_exact_on_the_quadrature(grid16):
    # a log-density in span{1, u_x, u_y, u_z} projects back to its coefficients, and the
    # expansion of those coefficients rebuilds the density
    c, o = grid16
    tab = W.orientation_table(o.rotm, o.weights)
    assert np.allclose(np.linalg.norm(tab[:, :3], axis=1), 1.0)
    rng = np.random.default_rng(3)
    n = c["n"]
    a = rng.uniform(-0.45, 0.45, (4, n, n, n))  # f = a0 + a.u stays above the start floor
    f = a[0][..., None] + sum(a[k + 1][..., None] * tab[:, k] for k in range(3))
    xi = np.exp(0.5 * f)
    vext = np.zeros_like(xi)
    t, mask = W.target(xi, vext, tab, vmax=1e3)
    assert np.abs(t - a).max() < 1e-12
    assert mask.min() == 1.0
    assert np.abs(W.expand(t, vext, tab, 1e3) - xi).max() < 1e-12 * xi.max()


def test_target_floor_mask_and_expand_core(grid16):
    c, o = grid16
    tab = W.orientation_table(o.rotm, o.weights)
    n, no = c["n"], len(o.weights)
    xi = np.ones((n, n, n, no))
    vext = np.zeros_like(xi)
    xi[0, 0, 0] = 0.0
    vext[0, 0, 0] = 1e6
    t, mask = W.target(xi, vext, tab, vmax=100.0)
    assert t[0, 0, 0, 0] == W.FLOOR and mask[0, 0, 0] == 0.0 and mask[1, 0, 0] == 1.0
    x = W.expand(np.zeros((4, n, n, n)), vext, tab, 100.0)
    assert x[0, 0, 0].max() == 0.0 and x[1, 1, 1].min() == 1.0


def test_channels_of_one_ion_are_radial():
    n, L = 16, 8.0
    sol = synth.ion_solute()
    sol.xyz = np.array([[4.0, 4.0, 4.0]])
    f = W.features((n, n, n), (L, L, L), sol, synth.Solvent(), synth.kT_of(298.0), rvdw=3.9)
    assert f.shape == (3, n, n, n)
    # site at grid point (8, 8, 8): site density 1 there, symmetric under axis swaps
    assert abs(f[2, 8, 8, 8] - 1.0) < 1e-12
    for ch in range(3):
        assert np.allclose(f[ch], f[ch].transpose(1, 0, 2)) and np.allclose(f[ch], f[ch].transpose(2, 1, 0))
    # positive ion: potential positive and decreasing outwards; LJ repulsive at contact
    assert f[1, 8, 8, 8] > f[1, 8, 8, 11] > 0
    assert f[0, 8, 8, 9] > 1.0 and f[0, 8, 8, 15] < 0.0 and f[0, 8, 8, 0] == 0.0  # 3.5 A attractive, 4 A > rvdw


def test_network_argument_errors_without_gpu():
    L = engine.lib()
    h = ctypes.c_void_p()
    assert L.mdft_warm_net_create(12, 16, 16, 0, ctypes.byref(h)) == -1
    assert b"multiple of 8" in L.mdft_last_error()
    assert L.mdft_warm_net_destroy(None) == 0
    n = ctypes.c_longlong()
    assert L.mdft_warm_net_num_params(None, ctypes.byref(n)) == -1
    assert L.mdft_set_warm_net(None, None) == -1
    assert L.mdft_warm_target(None, None, None, None) == -1


def test_shipped_parameters_load():
    import os
    assert os.path.exists(warmstart.WEIGHTS)
    p, meta = warmstart.load_params()
    assert p.size == W.num_params() and np.isfinite(p).all()
    assert np.array_equal(p, W.bf16_round(p))                      # stored as BF16
    assert meta["train"] == 2000 and meta["final_val_loss"] < 0.1


def test_projection_form_round_trip(grid16):
    # a band-limited log-density (proj2angl of projections of a real field) projects to
    # planes whose expansion rebuilds the density: the projection form loses nothing there
    c, o = grid16
    A, B = W.angular_maps(o)
    rng = np.random.default_rng(4)
    n, no = 6, len(o.weights)
    raw = rng.uniform(-0.6, 0.6, (n, n, n, no))
    f = np.einsum("zyxk,kn->zyxn", np.moveaxis(np.stack([(raw @ A).real, (raw @ A).imag], -1).reshape(n, n, n, -1), -1, 0)
                  .transpose(1, 2, 3, 0), B)
    assert f.min() > W.START_FLOOR and f.max() < W.CEIL
    xi = np.exp(0.5 * f)
    vext = np.zeros_like(xi)
    t, mask = W.target_proj(xi, vext, A, vmax=1e3)
    assert t.shape == (2 * o.np, n, n, n) and mask.min() == 1.0
    assert np.abs(W.expand_proj(t, vext, B, 1e3) - xi).max() < 1e-12 * xi.max()


def test_network_head_width():
    # the head's width is the output count; the other layers do not change
    assert W.num_params(56) - W.num_params(4) == (56 - 4) * (16 + 1)
    import torch
    flat = torch.zeros(W.num_params(28), dtype=torch.float64)
    y = W.forward(flat, torch.zeros((3, 8, 8, 8), dtype=torch.float64), torch, nout=28)
    assert tuple(y.shape) == (28, 8, 8, 8)

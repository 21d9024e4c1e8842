"""Learned warm start on the GPU against the CPU oracle (oracle/warmnet_ref.py).

* the network's forward and every parameter gradient (library kernels: BF16 weights, FP32
  activations and accumulation) against torch float64 autograd of the same network with
  the same BF16-rounded weights, on a 16^3 grid;
* training steps lower the loss;
* the solver-side kernels (input channels, log-density projections and mask, starting
  density) against their numpy restatements;
* warm-started solves converge to the cold solve's result, and with the committed trained
  parameters they are compared with cold solves on held-out solutes at 64^3."""
import os

import numpy as np
import pytest
import torch

import cases
from mdft_b200 import Engine, PREC_MIXED, synth, warmstart
from oracle import oracle as O
from oracle import warmnet_ref as W

pytestmark = pytest.mark.gpu
SV = cases.SOLVENT
N16 = 16


def _dev(a, dtype=torch.float32):
    t = torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")
    torch.cuda.synchronize()
    return t


@pytest.fixture(scope="module")
def net16():
    net = warmstart.WarmNet(N16, seed=5)
    yield net
    net.close()


def _sample(seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((3, N16, N16, N16)).astype(np.float32)
    t = rng.standard_normal((4, N16, N16, N16)).astype(np.float32)
    m = (rng.random((N16, N16, N16)) > 0.25).astype(np.float32)
    return x, t, m


def test_forward_matches_oracle(net16):
    x, _, _ = _sample(11)
    dx = _dev(x)
    out = torch.empty((4, N16, N16, N16), device="cuda")
    net16.forward(dx.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    p = W.bf16_weights(net16.get_params()).astype(np.float64)
    ref = W.forward(torch.tensor(p), torch.tensor(x, dtype=torch.float64), torch).numpy()
    got = out.cpu().numpy()
    assert np.isfinite(got).all()
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-5, err


def test_gradients_match_oracle(net16):
    x, t, m = _sample(12)
    dx, dt, dm = _dev(x), _dev(t), _dev(m)
    g, loss = net16.gradients(dx.data_ptr(), dt.data_ptr(), dm.data_ptr())
    p = W.bf16_weights(net16.get_params()).astype(np.float64)
    pt = torch.tensor(p, requires_grad=True)
    y = W.forward(pt, torch.tensor(x, dtype=torch.float64), torch)
    L = W.loss(y, torch.tensor(t, dtype=torch.float64), torch.tensor(m, dtype=torch.float64))
    L.backward()
    assert abs(loss - L.item()) <= 1e-5 * abs(L.item())
    ref = pt.grad.numpy()
    off = 0
    for li, (k, _, _, ci, co, _, _) in enumerate(W.LAYERS):
        n = int(np.prod(W.weight_shape(k, ci, co)))
        for a, b, what in ((off, off + n, "W"), (off + n, off + n + co, "b")):
            e = np.abs(g[a:b] - ref[a:b]).max() / np.abs(ref[a:b]).max()
            assert e < 2e-4, (li, what, e)
        off += n + co


def test_training_lowers_the_loss():
    net = warmstart.WarmNet(N16, seed=6)
    rng = np.random.default_rng(13)
    data = []
    for _ in range(2):
        x = rng.standard_normal((3, N16, N16, N16)).astype(np.float32)
        t = np.stack([np.tanh(x[0] - 0.5 * x[1]), 0.3 * x[2], np.roll(x[0], 1, axis=2), x[1] * 0.5]).astype(np.float32)
        data.append((_dev(x), _dev(t), _dev(np.ones((N16,) * 3, np.float32))))
    before = warmstart.evaluate_loss(net, data)
    for _ in range(80):
        net.train_step([d[0].data_ptr() for d in data], [d[1].data_ptr() for d in data], [d[2].data_ptr() for d in data],
                       2e-3)
    assert np.isfinite(net.take_loss())
    after = warmstart.evaluate_loss(net, data)
    assert after < 0.3 * before, (before, after)
    net.close()


@pytest.fixture(scope="module")
def sys16(tmp_path_factory):
    c = cases.CASES["mol16_m2"]
    ck = cases.ck_path(tmp_path_factory.mktemp("ck"), c["mmax"])
    e = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0)
    sol = cases.solute_of(c)
    e.compute_vext(sol, SV, rvdw=c["rvdw"])
    o = O.Oracle(c["n"], c["L"], c["mmax"], ck, SV.kT, SV.n0)
    tab = W.orientation_table(o.rotm, o.weights)
    yield c, ck, e, sol, tab
    e.close()


def _vmax(kT):
    return (-np.log(np.finfo(np.float64).eps) - float(np.float32(0.05))) * kT


def test_channels_match_oracle(sys16):
    c, _, e, sol, _ = sys16
    n = c["n"]
    feat = torch.empty((3, n ** 3), device="cuda")
    e.warm_features(sol, SV, feat.data_ptr(), rvdw=c["rvdw"])
    torch.cuda.synchronize()
    ref = W.features((n, n, n), (c["L"],) * 3, sol, SV, e.kT, c["rvdw"]).reshape(3, -1)
    got = feat.cpu().numpy()
    for ch in range(3):
        assert np.abs(got[ch] - ref[ch]).max() <= 1e-6 * max(1.0, np.abs(ref[ch]).max()), ch


def test_target_and_expand_match_oracle(sys16):
    c, _, e, _, tab = sys16
    n = c["n"]
    vext = e.get_vext()
    rng = np.random.default_rng(14)
    xi = rng.uniform(0.2, 2.5, e.shape)
    xi[vext >= _vmax(e.kT)] = 0.0
    dxi = _dev(xi, torch.float64)
    tgt = torch.empty((4, n ** 3), device="cuda")
    mask = torch.empty((n ** 3,), device="cuda")
    e.warm_target(tgt.data_ptr(), mask.data_ptr(), d_xi=dxi.data_ptr())
    torch.cuda.synchronize()
    rt, rm = W.target(xi, vext, tab, _vmax(e.kT))
    assert np.abs(tgt.cpu().numpy() - rt.reshape(4, -1)).max() < 1e-5
    assert np.array_equal(mask.cpu().numpy(), rm.reshape(-1).astype(np.float32))
    pred = rng.uniform(-2, 2, (4, n ** 3)).astype(np.float32)
    dp = _dev(pred)
    out = torch.empty(e.shape, dtype=torch.float64, device="cuda")
    e.warm_expand(dp.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    rx = W.expand(pred.astype(np.float64).reshape(4, n, n, n), vext, tab, _vmax(e.kT))
    assert np.abs(out.cpu().numpy() - rx).max() <= 1e-12 * rx.max()


def test_projection_form_network_matches_oracle():
    # a network with the projection form's head (2 np outputs at mmax 2: 28): forward and every
    # parameter gradient against torch float64 autograd
    nout = 28
    net = warmstart.WarmNet(N16, seed=15, nout=nout)
    rng = np.random.default_rng(16)
    x = rng.standard_normal((3, N16, N16, N16)).astype(np.float32)
    t = rng.standard_normal((nout, N16, N16, N16)).astype(np.float32)
    m = (rng.random((N16, N16, N16)) > 0.25).astype(np.float32)
    dx, dt, dm = _dev(x), _dev(t), _dev(m)
    out = torch.empty((nout, N16, N16, N16), device="cuda")
    net.forward(dx.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    p = W.bf16_weights(net.get_params(), nout).astype(np.float64)
    pt = torch.tensor(p, requires_grad=True)
    y = W.forward(pt, torch.tensor(x, dtype=torch.float64), torch, nout)
    got = out.cpu().numpy()
    assert np.abs(got - y.detach().numpy()).max() < 1e-5 * np.abs(y.detach().numpy()).max()
    g, loss = net.gradients(dx.data_ptr(), dt.data_ptr(), dm.data_ptr())
    L = W.loss(y, torch.tensor(t, dtype=torch.float64), torch.tensor(m, dtype=torch.float64))
    L.backward()
    assert abs(loss - L.item()) <= 1e-5 * abs(L.item())
    ref = pt.grad.numpy()
    off = 0
    for li, (k, _, _, ci, co, _, _) in enumerate(W.layers(nout)):
        n = int(np.prod(W.weight_shape(k, ci, co)))
        for a, b, what in ((off, off + n, "W"), (off + n, off + n + co, "b")):
            e = np.abs(g[a:b] - ref[a:b]).max() / np.abs(ref[a:b]).max()
            assert e < 2e-4, (li, what, e)
        off += n + co
    net.close()


def test_projection_form_target_and_expand_match_oracle(sys16):
    c, ck, e, _, _ = sys16
    n = c["n"]
    o = O.Oracle(c["n"], c["L"], c["mmax"], ck, SV.kT, SV.n0)
    A, B = W.angular_maps(o)
    nout = 2 * e.np
    vext = e.get_vext()
    rng = np.random.default_rng(17)
    xi = rng.uniform(0.2, 2.5, e.shape)
    xi[vext >= _vmax(e.kT)] = 0.0
    dxi = _dev(xi, torch.float64)
    tgt = torch.empty((nout, n ** 3), device="cuda")
    mask = torch.empty((n ** 3,), device="cuda")
    e.warm_target(tgt.data_ptr(), mask.data_ptr(), d_xi=dxi.data_ptr(), nout=nout)
    torch.cuda.synchronize()
    rt, rm = W.target_proj(xi, vext, A, _vmax(e.kT))
    assert np.abs(tgt.cpu().numpy() - rt.reshape(nout, -1)).max() <= 1e-5 * max(1.0, np.abs(rt).max())
    assert np.array_equal(mask.cpu().numpy(), rm.reshape(-1).astype(np.float32))
    # the start from planes of a real field's projections (the form a trained network predicts)
    raw = rng.uniform(-0.5, 0.5, e.shape)
    pr = raw @ A
    pred = np.moveaxis(np.stack([pr.real, pr.imag], -1).reshape(n, n, n, -1), -1, 0).astype(np.float32)
    dp = _dev(pred.reshape(nout, -1))
    out = torch.empty(e.shape, dtype=torch.float64, device="cuda")
    e.warm_expand(dp.data_ptr(), out.data_ptr(), nout=nout)
    torch.cuda.synchronize()
    rx = W.expand_proj(pred.astype(np.float64), vext, B, _vmax(e.kT))
    assert np.abs(out.cpu().numpy() - rx).max() <= 1e-12 * rx.max()
    o.close()


@pytest.mark.parametrize("precision", [0, PREC_MIXED])
def test_warm_started_solve_reaches_the_cold_result(sys16, precision):
    c, ck, _, sol, _ = sys16
    opts = dict(m=5, pgtol=1e-5, ftol_abs=-1.0, itermax=2000, precision=precision)
    cold = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=precision)
    rc = cold.solve(sol, SV, rvdw=c["rvdw"], **opts)
    warm = Engine(c["n"], c["L"], c["mmax"], ck, temperature=SV.temperature, n0=SV.n0, precision=precision)
    net = warmstart.WarmNet(c["n"], seed=9)
    warm.set_warm_net(net)
    rw = warm.solve(sol, SV, rvdw=c["rvdw"], **opts)
    st = warm.warm_stats()
    assert st["warm_starts"] == 1 and st["fallbacks"] == 0
    assert rw["status"] == 0 and rw["pgnorm"] <= 1e-5
    assert abs(rw["dG"] - rc["dG"]) < 2e-3, (rw["dG"], rc["dG"])
    warm.set_warm_net(None)
    rb = warm.solve(sol, SV, rvdw=c["rvdw"], **opts)
    assert rb["evaluations"] == rc["evaluations"] and abs(rb["dG"] - rc["dG"]) < 1e-9 * abs(rc["dG"])
    for x in (warm, cold):
        x.close()
    net.close()


@pytest.mark.skipif(not os.path.exists(warmstart.WEIGHTS), reason="no trained parameters in the package")
def test_trained_network_against_cold_solves(tmp_path, record_property):
    """Held-out 1-30-site solutes at 64^3 (seeds outside the training set): the trained
    network's start is much closer to the converged density than the bulk guess (masked
    squared error of the m <= 1 log-density projections).  Cold mixed solves with the bench's
    stop rule (max|df| <= 1e-4, |sum w df dv| <= 0.1) and warm-started ones with the learned
    form's tighter rule (5e-5, 0.05; with the bench's rule one held-out warm solve in twelve
    stopped 0.133 kJ/mol off) land within 0.1 kJ/mol of an FP64 solve to max|df| <= 1e-6.
    The warm/cold evaluation ratio is recorded (junit property warm_cold_evaluation_ratio)
    and bounded."""
    params, meta = warmstart.load_params()
    ck = str(tmp_path / "ck.dat")
    synth.make_ck_file(ck, 3, seed=warmstart.CK_SEED, kmax=12.0)
    opts = dict(m=5, pgtol=1e-4, ftol_abs=-1.0, itermax=3000, precision=PREC_MIXED, guni_tol=0.1)
    warm_opts = dict(opts, pgtol=warmstart.LEARNED_PGTOL, guni_tol=warmstart.LEARNED_GUNI_TOL)
    ref_opts = dict(m=5, pgtol=1e-6, ftol_abs=-1.0, itermax=3000, precision=0, guni_tol=0.01)
    e = Engine(64, 32.0, 3, ck, temperature=SV.temperature, n0=SV.n0, precision=PREC_MIXED)
    ref = Engine(64, 32.0, 3, ck, temperature=SV.temperature, n0=SV.n0, precision=0)
    net = warmstart.WarmNet(64, params=params)
    n3 = 64 ** 3
    feat = torch.empty((3, n3), device="cuda")
    tgt = torch.empty((4, n3), device="cuda")
    mask = torch.empty((n3,), device="cuda")
    pred = torch.empty((4, n3), device="cuda")
    rows = []
    for sd in (50000000, 50000001, 50000002):
        sol = warmstart.centred(warmstart.config4_solute(sd), e.box)
        dg_ref = ref.solve(sol, SV, **ref_opts)["dG"]
        e.set_warm_net(None)
        rc = e.solve(sol, SV, **opts)
        e.warm_target(tgt.data_ptr(), mask.data_ptr())
        e.warm_features(sol, SV, feat.data_ptr())
        torch.cuda.synchronize()
        net.forward(feat.data_ptr(), pred.data_ptr())
        torch.cuda.synchronize()
        err_net = float((((pred - tgt) ** 2).sum(0) * mask).sum())
        err_bulk = float(((tgt ** 2).sum(0) * mask).sum())
        assert err_net < 0.1 * err_bulk, (sd, err_net, err_bulk)
        e.set_warm_net(net)
        rw = e.solve(sol, SV, **warm_opts)
        assert rw["status"] == 0 and rw["pgnorm"] <= warmstart.LEARNED_PGTOL
        assert abs(rc["dG"] - dg_ref) <= 0.1, (sd, rc["dG"], dg_ref)
        assert abs(rw["dG"] - dg_ref) <= 0.1, (sd, rw["dG"], dg_ref)
        rows.append((rc["evaluations"] + rc["evaluations_mixed"], rw["evaluations"] + rw["evaluations_mixed"],
                     round(err_net / err_bulk, 4), round(rc["dG"] - dg_ref, 4), round(rw["dG"] - dg_ref, 4)))
    cold = sum(r[0] for r in rows)
    warm = sum(r[1] for r in rows)
    ratio = warm / cold
    record_property("warm_cold_evaluation_ratio", round(ratio, 4))
    record_property("held_out_rows", rows)
    print("held-out (cold evaluations, warm evaluations, start error ratio, cold dG error, warm dG error):", rows,
          "warm/cold evaluations: %.3f" % ratio, "trained:", {k: meta.get(k) for k in ("train", "epochs", "final_val_loss")})
    # measured 1.13 on these seeds (warm at the tighter rule against cold at the bench's): the
    # start gains nothing in evaluations, so the bench keeps the cold start; the bound catches
    # a start that costs more
    assert ratio <= 1.25, rows
    e.set_warm_net(None)
    for x in (e, ref):
        x.close()
    net.close()

"""Learned warm start: the network object, training-set generation by the solver itself,
training, and the parameter file.

The network, its kernels and the solver glue live in libmdft_b200.so (csrc/warmnet.cu,
csrc/k_warmnet.cuh, csrc/warmstart.cuh); this module drives them through the C-ABI.  The
reference has no counterpart: its solves start from guess_density
(src/module_density.f90:267-284), which stays the fallback of every warm-started solve.

Device memory for the training set is held in torch CUDA tensors (plumbing only: every
kernel that touches them is the library's).

    python -m mdft_b200.warmstart --train 2000 --val 50 --epochs 12 [--form proj|m1] [--eval 200]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import threading
import time

import numpy as np

from . import engine as E
from . import synth

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "warmstart_weights.npz")  # m <= 1 form
# all projections of the log-density (56 outputs at mmax 3): the form the solver starts from
WEIGHTS_PROJ = os.path.join(os.path.dirname(os.path.abspath(__file__)), "warmstart_weights_proj.npz")
TRAIN_N, TRAIN_BOX = 48, 24.0   # 0.5 A spacing, as the 64^3 / 32 A evaluation grid
EVAL_N, EVAL_BOX = 64, 32.0
MMAX = 3
CK_SEED = 20260001              # the synthetic c(k) of the 64^3 / mmax 3 workload
# Stop rule of warm-started solves: with the cold solves' max|df| <= 1e-4, |sum w df dv| <= 0.1,
# one held-out warm solve in twelve (64^3, mmax 3, seeds 50000000..50000011) stopped
# 0.133 kJ/mol from the FP64 solve to 1e-6 (a slow mode the started density leaves that the
# uniform-mode bound does not see); at 5e-5 and 0.05 all twelve are within 0.031.
LEARNED_PGTOL = 5e-5
LEARNED_GUNI_TOL = 0.05


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to the nearest BF16 (ties to even), returned as FP32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


class WarmNet:
    """The warm-start network on one GPU for one grid (dimensions multiples of 8)."""

    def __init__(self, n: int, device: int = 0, seed: int | None = 20260401, params: np.ndarray | None = None,
                 nout: int = 4):
        h = C.c_void_p()
        E._check(E.lib().mdft_warm_net_create_n(n, n, n, int(nout), device, C.byref(h)))
        self.h = h.value
        self.n = n
        self.nout = int(nout)
        c = C.c_longlong()
        E._check(E.lib().mdft_warm_net_num_params(self.h, C.byref(c)))
        self.nparam = c.value
        if params is not None:
            self.set_params(params)
        elif seed is not None:
            E._check(E.lib().mdft_warm_net_init(self.h, C.c_ulonglong(seed)))

    def close(self):
        if getattr(self, "h", None):
            E.lib().mdft_warm_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        E._check(E.lib().mdft_warm_net_set_params(self.h, p.ctypes.data_as(E._FP), p.size))

    def get_params(self) -> np.ndarray:
        p = np.empty(self.nparam, dtype=np.float32)
        E._check(E.lib().mdft_warm_net_get_params(self.h, p.ctypes.data_as(E._FP), p.size))
        return p

    def set_stream(self, stream: int | None):
        E._check(E.lib().mdft_warm_net_set_stream(self.h, None if not stream else C.c_void_p(stream)))

    def forward(self, d_in: int, d_out: int | None):
        E._check(E.lib().mdft_warm_net_forward(self.h, C.c_void_p(d_in), None if d_out is None else C.c_void_p(d_out)))

    def gradients(self, d_in: int, d_target: int, d_mask: int | None):
        g = np.empty(self.nparam, dtype=np.float32)
        loss = np.zeros(1)
        E._check(E.lib().mdft_warm_net_gradients(self.h, C.c_void_p(d_in), C.c_void_p(d_target),
                                                 None if d_mask is None else C.c_void_p(d_mask),
                                                 g.ctypes.data_as(E._FP), E._p(loss)))
        return g, float(loss[0])

    def train_step(self, ins, targets, masks, lr: float):
        k = len(ins)
        a = (C.c_void_p * k)(*ins)
        b = (C.c_void_p * k)(*targets)
        m = None if masks is None else (C.c_void_p * k)(*masks)
        E._check(E.lib().mdft_warm_net_train_step(self.h, a, b, m, k, C.c_float(lr)))

    def take_loss(self) -> float:
        v = np.zeros(1)
        E._check(E.lib().mdft_warm_net_take_loss(self.h, E._p(v)))
        return float(v[0])

    @property
    def launch_count(self) -> int:
        c = C.c_longlong()
        E._check(E.lib().mdft_warm_net_launch_count(self.h, C.byref(c)))
        return c.value


def save_params(path: str, params: np.ndarray, meta: dict | None = None):
    """Parameters as BF16 bit patterns (the kernels' precision) plus a JSON note."""
    bits = (bf16_round(params).view(np.uint32) >> 16).astype(np.uint16)
    np.savez_compressed(path, bf16=bits, meta=np.array(json.dumps(meta or {})))


def load_params(path: str = WEIGHTS) -> tuple[np.ndarray, dict]:
    z = np.load(path)
    p = (z["bf16"].astype(np.uint32) << 16).view(np.float32)
    meta = json.loads(str(z["meta"]))
    meta.setdefault("nout", 4)
    return p, meta


def default_weights() -> str | None:
    """The parameter file the solver's learned start uses: the all-projection form when shipped."""
    for p in (WEIGHTS_PROJ, WEIGHTS):
        if os.path.exists(p):
            return p
    return None


def config4_solute(seed: int):
    """A seeded 1-30-site solute drawn as the 24-site bench solute (random walk, 1.4-1.6 A
    bonds inside 6 A, sigma U[2.5,3.8], eps U[0.2,1.0], q ~ N(0, 0.3) shifted to sum 0)."""
    nsite = 1 + int(np.random.default_rng(seed).integers(0, 30))
    return synth.random_walk_solute(nsite, seed)


def centred(sol, box):
    """The solute moved to the box centre (mv_solute_to_center, src/module_solute.f90:146-187)."""
    return synth.Solute(q=sol.q, sig=sol.sig, eps=sol.eps, xyz=synth.center_solute(sol.xyz, box))


def make_training_set(engines, seeds, solvent, rvdw=10.0, pgtol=1e-4, precision=E.PREC_FP64, log=None, nout=4,
                      guni_tol=0.0):
    """Solve every seeded solute with the solver (from the bulk guess) on the given engines,
    one host thread per engine, and keep each one's channels, target (nout x N) and mask on
    the device.  Returns (samples, per-solute results)."""
    n = engines[0].shape[0] * engines[0].shape[1] * engines[0].shape[2]
    box = engines[0].box
    samples = [None] * len(seeds)
    results = [None] * len(seeds)
    nxt = [0]
    lock = threading.Lock()
    errors = []

    def worker(eng):
        import torch as T
        torch_dev = T.device("cuda", eng.device)
        while True:
            with lock:
                i = nxt[0]
                nxt[0] += 1
            if i >= len(seeds):
                return
            try:
                sol = centred(config4_solute(seeds[i]), box)
                r = eng.solve(sol, solvent, rvdw=rvdw, pgtol=pgtol, ftol_abs=-1.0, itermax=5000, precision=precision,
                              guni_tol=guni_tol)
                feat = T.empty((3, n), dtype=T.float32, device=torch_dev)
                tgt = T.empty((nout, n), dtype=T.float32, device=torch_dev)
                mask = T.empty((n,), dtype=T.float32, device=torch_dev)
                eng.warm_features(sol, solvent, feat.data_ptr(), rvdw=rvdw)
                eng.warm_target(tgt.data_ptr(), mask.data_ptr(), nout=nout)
                T.cuda.synchronize(torch_dev)
                samples[i] = (feat, tgt, mask)
                results[i] = dict(seed=seeds[i], nsite=len(sol.q), dG=r["dG"], evaluations=r["evaluations"],
                                  status=r["status"])
                if log and i % 50 == 0:
                    log("sample %d/%d: %d sites, %d evaluations" % (i, len(seeds), len(sol.q), r["evaluations"]))
            except Exception as e:  # noqa: BLE001
                errors.append((seeds[i], repr(e)))
                return

    ts = [threading.Thread(target=worker, args=(e,)) for e in engines]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errors:
        raise E.MdftError("training-set generation failed: %s" % (errors[:3],))
    return samples, results


def train(net: WarmNet, samples, epochs=30, batch=4, lr=2e-3, lr_end=1e-4, seed=7, val=None, log=None):
    """Adam on the masked squared error; cosine decay of the learning rate from lr to lr_end."""
    rng = np.random.default_rng(seed)
    nsteps = epochs * ((len(samples) + batch - 1) // batch)
    step = 0
    hist = []
    for ep in range(epochs):
        order = rng.permutation(len(samples))
        for b0 in range(0, len(order), batch):
            idx = order[b0:b0 + batch]
            frac = step / max(1, nsteps - 1)
            cur = lr_end + 0.5 * (lr - lr_end) * (1.0 + np.cos(np.pi * frac))
            net.train_step([samples[i][0].data_ptr() for i in idx], [samples[i][1].data_ptr() for i in idx],
                           [samples[i][2].data_ptr() for i in idx], cur)
            step += 1
        tl = net.take_loss()
        vl = evaluate_loss(net, val) if val else float("nan")
        hist.append((ep, tl, vl))
        if log:
            log("epoch %d: train loss %.5f, validation loss %.5f" % (ep, tl, vl))
    return hist


def evaluate_loss(net: WarmNet, samples) -> float:
    tot = 0.0
    for f, t, m in samples:
        _, l = net.gradients(f.data_ptr(), t.data_ptr(), m.data_ptr())
        tot += l
    return tot / max(1, len(samples))


def evaluate_heldout(params, seeds, solvent, ck, workers=3, pgtol=1e-4, pgtol_ref=1e-6, log=None, nout=4, guni_tol=0.1):
    """Held-out solutes at 64^3: plain FP64 solves from the bulk guess to max|df| <= pgtol_ref
    (the dG reference), then mixed-precision solves to pgtol (and |sum w df dv| <= guni_tol)
    from the bulk guess and from the network's prediction, each form as one concurrent batch
    over `workers` engines.  Returns per-solute rows and a summary (evaluations, solutes/s by
    wall clock, |dG - FP64|)."""
    sols = [centred(config4_solute(sd), (EVAL_BOX,) * 3) for sd in seeds]
    out = {}
    forms = [("fp64_ref", E.PREC_FP64, pgtol_ref, False, 0.01), ("mixed_cold", E.PREC_MIXED, pgtol, False, guni_tol),
             ("mixed_warm", E.PREC_MIXED, pgtol, True, guni_tol)]
    fallbacks = 0
    for name, prec, tol, warm, gtol in forms:
        engs = [E.Engine(EVAL_N, EVAL_BOX, MMAX, ck, temperature=solvent.temperature, n0=solvent.n0, precision=prec)
                for _ in range(workers)]
        nets = []
        if warm:
            for e in engs:
                net = WarmNet(EVAL_N, device=e.device, params=params, nout=nout)
                e.set_warm_net(net)
                nets.append(net)
        t0 = time.time()
        res = E.solve_batch(engs, sols, solvent, m=5, pgtol=tol, ftol_abs=-1.0, itermax=5000, precision=prec,
                            guni_tol=gtol)
        wall = time.time() - t0
        if warm:
            fallbacks = sum(e.warm_stats()["fallbacks"] for e in engs)
            for e in engs:
                e.set_warm_net(None)
            for net in nets:
                net.close()
        for e in engs:
            e.close()
        out[name] = (res, wall)
        if log:
            log("%s: %d solutes in %.1f s" % (name, len(sols), wall))
    ref = [r["dG"] for r in out["fp64_ref"][0]]
    rows = []
    for i, sd in enumerate(seeds):
        c, w = out["mixed_cold"][0][i], out["mixed_warm"][0][i]
        f = out["fp64_ref"][0][i]
        rows.append(dict(seed=sd, nsite=len(sols[i].q), dG_fp64=ref[i], fp64_evals=f["evaluations"],
                         fp64_status=f["status"], fp64_pgnorm=f["pgnorm"],
                         cold_evals=c["evaluations"] + c["evaluations_mixed"], cold_iters=c["iterations"],
                         cold_status=c["status"], cold_pgnorm=c["pgnorm"],
                         warm_evals=w["evaluations"] + w["evaluations_mixed"], warm_iters=w["iterations"],
                         warm_status=w["status"], warm_pgnorm=w["pgnorm"],
                         cold_err=c["dG"] - ref[i], warm_err=w["dG"] - ref[i]))
    n = len(seeds)
    summ = dict(heldout=n, fallbacks=fallbacks,
                fp64_solutes_per_s=n / out["fp64_ref"][1], cold_solutes_per_s=n / out["mixed_cold"][1],
                warm_solutes_per_s=n / out["mixed_warm"][1],
                cold_mean_evals=float(np.mean([r["cold_evals"] for r in rows])),
                warm_mean_evals=float(np.mean([r["warm_evals"] for r in rows])),
                cold_mean_iters=float(np.mean([r["cold_iters"] for r in rows])),
                warm_mean_iters=float(np.mean([r["warm_iters"] for r in rows])),
                cold_max_dG_err=float(np.max(np.abs([r["cold_err"] for r in rows]))),
                warm_max_dG_err=float(np.max(np.abs([r["warm_err"] for r in rows]))),
                cold_over_0p1=int(np.sum(np.abs([r["cold_err"] for r in rows]) > 0.1)),
                warm_over_0p1=int(np.sum(np.abs([r["warm_err"] for r in rows]) > 0.1)),
                fp64_mean_evals=float(np.mean([r["evaluations"] for r in out["fp64_ref"][0]])))
    return rows, summ


def main(argv=None):
    import torch

    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--train", type=int, default=600, help="training solutes (48^3, plain FP64 solves)")
    ap.add_argument("--val", type=int, default=40, help="validation solutes (48^3)")
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--workers", type=int, default=3)
    ap.add_argument("--pgtol", type=float, default=1e-4)
    ap.add_argument("--seed0", type=int, default=40000000, help="first training seed (held-out seeds start at 50000000)")
    ap.add_argument("--ck", default=None, help="c(k) file (default: the synthetic mmax-3 table)")
    ap.add_argument("--eval", type=int, default=0, help="held-out 64^3 solutes to compare cold and warm solves on")
    ap.add_argument("--eval-seed0", type=int, default=50000000)
    ap.add_argument("--eval-only", default=None, help="parameter file: skip training, only the held-out comparison")
    ap.add_argument("--form", default="proj", choices=["proj", "m1"],
                    help="proj: all projections of the log-density (2 np outputs); m1: the m <= 1 real basis (4)")
    ap.add_argument("--solver", default="mixed", choices=["mixed", "fp64"], help="precision of the training-set solves")
    ap.add_argument("--guni-tol", type=float, default=0.1, help="uniform-mode stop bound of the solves (kJ/mol)")
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)
    t0 = time.time()

    def log(msg):
        print("[%7.1f s] %s" % (time.time() - t0, msg), flush=True)

    import tempfile
    tmp = tempfile.mkdtemp()
    ck = a.ck or os.path.join(tmp, "ck_m3.dat")
    if not a.ck:
        synth.make_ck_file(ck, MMAX, seed=CK_SEED, kmax=12.0)
    solvent = synth.Solvent()
    if a.eval_only:
        params, meta = load_params(a.eval_only)
        rows, summ = evaluate_heldout(params, [a.eval_seed0 + i for i in range(a.eval)], solvent, ck,
                                      workers=a.workers, pgtol=a.pgtol, log=log, nout=meta["nout"], guni_tol=a.guni_tol)
        log("held-out: %s" % json.dumps(summ))
        if a.report:
            with open(a.report, "w") as f:
                json.dump(dict(meta=meta, summary=summ, heldout=rows), f)
        return
    prec = E.PREC_MIXED if a.solver == "mixed" else E.PREC_FP64
    engines = [E.Engine(TRAIN_N, TRAIN_BOX, MMAX, ck, temperature=solvent.temperature, n0=solvent.n0, precision=prec)
               for _ in range(a.workers)]
    nout = 4 if a.form == "m1" else 2 * engines[0].np
    out_path = a.out or (WEIGHTS if a.form == "m1" else WEIGHTS_PROJ)
    seeds = [a.seed0 + i for i in range(a.train + a.val)]
    samples, res = make_training_set(engines, seeds, solvent, pgtol=a.pgtol, log=log, nout=nout, precision=prec,
                                     guni_tol=a.guni_tol)
    tgen = time.time() - t0
    log("training set: %d solutes in %.1f s (%.1f evaluations per solve)" %
        (len(samples), tgen, np.mean([r["evaluations"] for r in res])))
    for e in engines:
        e.close()
    net = WarmNet(TRAIN_N, nout=nout)
    t1 = time.time()
    hist = train(net, samples[:a.train], epochs=a.epochs, batch=a.batch, lr=a.lr, val=samples[a.train:], log=log)
    ttrain = time.time() - t1
    meta = dict(nout=nout, form=a.form, solver=a.solver, guni_tol=a.guni_tol,
                train=a.train, val=a.val, epochs=a.epochs, batch=a.batch, lr=a.lr, pgtol=a.pgtol, seed0=a.seed0,
                grid=[TRAIN_N, TRAIN_BOX], final_train_loss=hist[-1][1], final_val_loss=hist[-1][2],
                gen_seconds=tgen, train_seconds=ttrain)
    params = net.get_params()
    net.close()
    del samples
    torch.cuda.empty_cache()
    rows, summ = [], {}
    if a.eval > 0:
        rows, summ = evaluate_heldout(bf16_round(params), [a.eval_seed0 + i for i in range(a.eval)], solvent, ck,
                                      workers=a.workers, pgtol=a.pgtol, log=log, nout=nout, guni_tol=a.guni_tol)
        meta["heldout"] = summ
        log("held-out: %s" % json.dumps(summ))
    save_params(out_path, params, meta)
    log("saved %s (%d parameters): %s" % (out_path, len(params), json.dumps(meta)))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(dict(meta=meta, history=hist, solves=res, heldout=rows), f)


if __name__ == "__main__":
    main()

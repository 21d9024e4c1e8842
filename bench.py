#!/usr/bin/env python
"""Benchmark of the MDFT engine: solutes/s converged at 64^3, mmax 3, in the headline form
(mixed precision, optionally from the learned warm start) and in the plain FP64 form.

Workload (one "step" = one solute solved end to end): a seeded 24-site neutral
solute (random walk, 1.4-1.6 A bonds inside 6 A, sigma U[2.5,3.8], eps
U[0.2,1.0], q ~ N(0,0.3) shifted to 0) in SPC/E-like 3-site water, 64^3 grid,
32 A box, mmax 3, synthetic c(k); vext (LJ + Poisson) -> guess_density ->
L-BFGS (m=5, stop at max|df| <= 1e-4 and |sum w df dv| <= 0.1 kJ/mol in FP64; the
reference's F-decrease test is off, it stops ~1 kJ/mol short of the converged dG)
-> pressure correction -> dG.  The steps' solutes are solved through mdft_solve_batch
on --workers engine handles (default 3), so that solves overlap on the GPU; each form
is timed over --regions regions (default 3) and the median is reported.  The plain
FP64 form solves the same solutes on as many handles with the same stop rule; its rate
and the ratio are in config.  Every run re-solves its solutes in FP64 to max|df| <= 1e-6
and reports the largest |dG - dG_FP64| of both forms (the metric's 0.1 kJ/mol bar).
Synthetic inputs stand in for the reference's data.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N>1 runs N independent replicas (each rank solves its own solutes; no
collective on the data path, only a barrier and a max of the timings).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "mdft-dev_general_b200")]

METRIC = "solutes/s to |ΔG−FP64|≤0.1 kJ/mol at 64³ mmax3: learned+mixed vs plain FP64"
UNIT = "solutes/s"
N_GRID, BOX, MMAX, NSITE = 64, 32.0, 3, 24
RVDW = 10.0
CK_SEED = 20260001
# Stop rule of the timed solves: max|df| <= 1e-4 in FP64.  On this workload the FP64 dG path
# is within 0.01-0.03 kJ/mol of its max|df| <= 1e-6 value there; every run checks its dG
# against an FP64 solve to 1e-6 (PGTOL_REF) and reports the largest deviation.
PGTOL = 1e-4
PGTOL_REF = 1e-6
# Second stop bound: |sum_{r,io} w df dv| (the gradient along a uniform change of xi), in
# kJ/mol.  Along FP64 L-BFGS paths the dG error at a stopping point is about half of it, and
# it converges more slowly than max|df| for small solutes.
GUNI_TOL = 0.1
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# dram__bytes_read.sum + dram__bytes_write.sum per launch, by (form, stage), from one ncu
# capture of each FP32-phase kernel in a mixed solve of this workload (k_gather_ring<84>,
# k_project_umma<float,4>, k_ozd<3,2>), and of the FP64 form's kernels; absent: null
NCU_TRAFFIC_BYTES = {("mixed", "oz"): 69.2e6, ("mixed", "gather"): 397.8e6, ("mixed", "project"): 113.1e6,
                     ("fp64", "oz"): 186.6e6, ("fp64", "gather"): 803.4e6, ("fp64", "project"): 256.1e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="small grid smoke run (not a bench number)")
    ap.add_argument("--form", default="mixed", choices=["learned", "mixed", "fp64"],
                    help="learned: mixed solves started from the trained warm-start network; mixed: FP32 excess "
                         "pipeline then an FP64 polish, from the bulk guess; fp64: plain FP64 solve")
    ap.add_argument("--pgtol", type=float, default=PGTOL, help="stop at max|df| <= pgtol (FP64 gradient)")
    ap.add_argument("--workers", type=int, default=3,
                    help="concurrent solves per GPU (engine handles, each with its own buffers and stream)")
    ap.add_argument("--pgtol-mixed", type=float, default=0.0, help="FP32-phase stop (<=0: the final pgtol)")
    ap.add_argument("--polish", type=int, default=1, help="mixed: 1 = FP64 iterations until pgtol, 0 = one FP64 evaluation")
    ap.add_argument("--guni-tol", type=float, default=GUNI_TOL,
                    help="also stop only when |sum w df dv| <= this (kJ/mol); <= 0: off")
    ap.add_argument("--regions", type=int, default=5, help="timed regions per form (the median is reported)")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain FP64 form's timing")
    ap.add_argument("--solves", type=int, default=0,
                    help="profiling mode: only N solves of the workload (no timing, no reference solves)")
    ap.add_argument("--evals", type=int, default=0,
                    help="profiling mode: only N energy_and_gradient evaluations of the workload (no solve)")
    ap.add_argument("--prof-grid", type=int, default=0,
                    help="with --evals: evaluations of a config-2-style cluster on this grid (0.375 A spacing) instead")
    ap.add_argument("--prof-mmax", type=int, default=5, help="with --prof-grid: the angular order")
    ap.add_argument("--prof-solve", action="store_true",
                    help="with --prof-grid: full solves of the packed cluster (mixed and FP64 at the bench's stop "
                         "rule, FP64 to max|df| <= 1e-6) and their dG")
    ap.add_argument("--terms-compare", action="store_true",
                    help="time one FP64 evaluation plain, with each bridge term and as a two-species mixture")
    ap.add_argument("--fft-compare", action="store_true",
                    help="timing comparison: the engine's FFT stages against cuFFT (torch.fft) on the same planes")
    return ap.parse_args()


def ck_file(mmax, kmax=12.0):
    from mdft_b200 import synth
    d = os.path.join(tempfile.gettempdir(), "mdft_b200_bench")
    os.makedirs(d, exist_ok=True)
    p = os.path.join(d, "ck_m%d_s%d_k%g.txt" % (mmax, CK_SEED, kmax))
    if not os.path.exists(p):
        tmp = p + ".%d" % os.getpid()
        synth.make_ck_file(tmp, mmax, seed=CK_SEED, kmax=kmax, dk=0.01)
        os.replace(tmp, p)
    return p


def solute(seed, box):
    from mdft_b200 import synth
    s = synth.random_walk_solute(NSITE, seed=seed)
    s.xyz = synth.center_solute(s.xyz, (box,) * 3)
    return s


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    try:
        with open(MEASURED_PEAKS) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def stage_bytes(N, no, np_, c=16, r=8):
    """Algorithmic bytes per evaluation of each stage inside a solve (c = bytes per complex
    projection value, r = bytes per real value of the point, vext, gradient and direction):
    the projection reads xi and writes the planes; each FFT direction and the OZ read and write
    them; the gather reads them, xi, vext and the search direction and writes the gradient."""
    return {"project": N * (no * r + np_ * c), "fft_forward": 2 * np_ * N * c, "oz": 2 * np_ * N * c,
            "fft_inverse": 2 * np_ * N * c, "gather": N * (np_ * c + 4 * no * r)}


def cpu_oracle_eval_seconds(n, box, mmax, ck, nevals, threads, seed=1000):
    """Time nevals oracle evaluations of the workload (solute `seed`, guess density) on the host cores."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as O
    from mdft_b200 import synth
    sv = synth.Solvent()
    o = O.Oracle(n, box, mmax, ck, sv.kT, sv.n0)
    s = solute(seed, box)
    o.compute_vext(s, sv, rvdw=RVDW)
    xi = o.guess_density()
    o.energy_grad(xi)  # first call
    t0 = time.perf_counter()
    for _ in range(nevals):
        o.energy_grad(xi)
    return (time.perf_counter() - t0) / nevals


def replica_seeds(rank, count):
    """Seeds of the solutes one rank solves: replicas work on disjoint solutes."""
    return [10_000 * rank + i for i in range(count)]


def max_over_ranks(t_ms, world, device):
    """The slowest rank's time (every rank calls this once per timed region)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([t_ms], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, steps, t_ms):
    """Solutes/s of the whole job: every rank solves `steps` solutes within t_ms."""
    return world * steps / (t_ms / 1e3)


def reference_arm(args, rank, world):
    """CPU implementation of the path on the host cores (the C restatement; the Fortran
    reference cannot be compiled here): per step one FP64 evaluation of one of the b200 arm's
    timed solutes at its guess density, extrapolated to a solve by the FP64 evaluations per
    solve of this workload and stop rule."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as O
    from mdft_b200 import synth
    sv = synth.Solvent()
    ck = ck_file(MMAX)
    seeds = replica_seeds(0, args.warmup + args.steps)[args.warmup:]
    cache = {}

    def eval_seconds(seed):
        if seed not in cache:  # set-up (vext, guess density) once per solute, not timed
            o = O.Oracle(N_GRID, BOX, MMAX, ck, sv.kT, sv.n0)
            o.compute_vext(solute(seed, BOX), sv, rvdw=RVDW)
            cache.clear()
            cache[seed] = (o, o.guess_density())
        o, xi = cache[seed]
        t0 = time.perf_counter()
        o.energy_grad(xi)
        return time.perf_counter() - t0

    times = []
    for i in range(args.warmup + args.steps):
        t = eval_seconds(seeds[i % len(seeds)])
        if i >= args.warmup:
            times.append(t)
    t_eval = float(np.mean(times))
    ev = EVALS_PER_SOLVE_FP64
    if ev["key"] != (N_GRID, BOX, MMAX, NSITE, CK_SEED, args.pgtol, args.guni_tol):
        raise SystemExit("EVALS_PER_SOLVE_FP64 was measured for another workload or stop rule: %r" % (ev["key"],))
    v = 1.0 / (t_eval * ev["mean"])
    sample = ("one FP64 energy_and_gradient per step of the b200 arm's timed solutes (seeds %d..%d) at their guess "
              "density, %d OpenMP threads, x %.1f evaluations per FP64 solve (%s); the L-BFGS vector work is not "
              "counted" % (seeds[0], seeds[-1], threads, ev["mean"], ev["source"]))
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_eval * 1e3,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                      "data": "synthetic", "config": {"workload": WORKLOAD % (N_GRID, BOX, MMAX, NSITE),
                                                      "form": "CPU FP64 restatement (oracle), OpenMP",
                                                      "extrapolated": "value = 1 / (per-evaluation time x evaluations "
                                                                      "per solve); ms_per_step is the measured time "
                                                                      "of one step's sample (one evaluation)",
                                                      "stop": STOP_TEXT % (PGTOL, GUNI_TOL)},
                      "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
                      "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


WORKLOAD = "%d^3 grid, %g A box, mmax %d, %d-site random-walk solute per step, synthetic c(k)"
STOP_TEXT = ("max|df|<=%g and |sum w df dv|<=%g kJ/mol in FP64 (line-search stall accepted); dG checked against "
             "FP64 solves to max|df|<=1e-6")
# Evaluations per plain FP64 solve of this workload and stop rule (the mean over the bench's
# first 20 solutes on one B200); scales the CPU evaluation time to solutes/s in the reference
# arm, which cannot count them itself.  The b200 arm counts them in every run and reports both.
EVALS_PER_SOLVE_FP64 = {"mean": 190.55, "key": (N_GRID, BOX, MMAX, NSITE, CK_SEED, PGTOL, GUNI_TOL),
                        "source": "mean of 20 plain FP64 GPU solves of seeds 5..24"}


def fft_compare(n, box, ck, sv, sol, rvdw, device):
    """The engine's forward and inverse 3-D FFT stages (np planes of n^3 complex, in place,
    live CUDA-event stage times averaged over one solve) against cuFFT through torch.fft on a
    tensor of the same shape (out of place, plan cached, the same sign conventions, no
    scaling).  A timing comparison only: cuFFT is not on the engine's path."""
    import torch
    from mdft_b200 import Engine, PREC_FP64, PREC_MIXED
    res = {"metric": "3-D FFT stage time, %d planes of %d^3" % (0, n), "unit": "ms", "workload": WORKLOAD % (N_GRID, BOX, MMAX, NSITE)}
    for name, prec, dt in (("fp32", PREC_MIXED, torch.complex64), ("fp64", PREC_FP64, torch.complex128)):
        e = Engine(n, box, MMAX, ck, temperature=sv.temperature, n0=sv.n0, device=device, precision=prec)
        np_ = e.np
        opts = dict(m=5, pgtol=PGTOL, ftol_abs=-1.0, itermax=3000, precision=prec, guni_tol=GUNI_TOL)
        e.solve(sol, sv, rvdw=rvdw, **opts)
        e.set_timing(True)
        e.solve(sol, sv, rvdw=rvdw, **opts)
        st, cnt = e.stage_times()
        e.set_timing(False)
        e.close()
        x = torch.randn(np_, n, n, n, dtype=dt, device=device)
        for _ in range(5):  # plans and warm-up
            torch.fft.fftn(x, dim=(1, 2, 3))
            torch.fft.ifftn(x, dim=(1, 2, 3), norm="forward")
        t = {}
        for key, fn in (("forward", lambda: torch.fft.fftn(x, dim=(1, 2, 3))),
                        ("inverse", lambda: torch.fft.ifftn(x, dim=(1, 2, 3), norm="forward"))):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record()
            for _ in range(20):
                fn()
            b.record()
            torch.cuda.synchronize()
            t[key] = a.elapsed_time(b) / 20
        res["metric"] = "3-D FFT stage time, %d planes of %d^3" % (np_, n)
        res[name] = {"engine_forward_ms": st["fft_forward"] / cnt, "engine_inverse_ms": st["fft_inverse"] / cnt,
                     "cufft_forward_ms": t["forward"], "cufft_inverse_ms": t["inverse"], "engine_evaluations": cnt}
    print(json.dumps(res))


def terms_compare(n, box, ck, sv, sol, rvdw, device, evals=20):
    """Device time of one FP64 evaluation (energy and gradient) of the bench workload at a
    perturbed bulk density: plain, with bridge = cgb ('sla'), with bridge = hard_sphere (PY,
    R = 1.4 A), and as a mixture of two species (x = 0.5 each) through mdft_mixture_*.
    CUDA events on species 0's stream around `evals` evaluations after 3 untimed ones; each
    evaluation ends with the host reading its sums, so the gaps between them are included."""
    import torch
    from mdft_b200 import Engine, Mixture, PREC_FP64

    def timed(stream_ptr, fn):
        st = torch.cuda.ExternalStream(stream_ptr)
        for _ in range(3):
            fn()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        for _ in range(evals):
            fn()
        b.record(st)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / evals

    res = {"metric": "FP64 evaluation time with the optional terms", "unit": "ms per evaluation",
           "workload": WORKLOAD % (N_GRID, BOX, MMAX, NSITE), "evaluations": evals}
    e = Engine(n, box, MMAX, ck, temperature=sv.temperature, n0=sv.n0, device=device, precision=PREC_FP64)
    e.compute_vext(sol, sv, rvdw=rvdw)
    rng = np.random.default_rng(5)
    xi_h = np.clip(1.0 + 0.1 * rng.standard_normal(e.shape), 0.0, None)
    xi = torch.from_numpy(xi_h).to(device)
    df = torch.empty_like(xi)
    run = lambda: e.energy_and_gradient_device(xi.data_ptr(), df.data_ptr())
    res["plain_ms"] = timed(e.stream, run)
    e.set_bridge_cgb(1, B6=5.0, sigma=1.0, c00=-13.665)
    res["cgb_sla_ms"] = timed(e.stream, run)
    e.set_bridge_fmt(1, 1.4)
    res["hard_sphere_py_ms"] = timed(e.stream, run)
    e.set_bridge_fmt(0)
    e.close()
    sp = [Engine(n, box, MMAX, ck, temperature=sv.temperature, n0=sv.n0 * 0.5, device=device, precision=PREC_FP64)
          for _ in range(2)]
    for h in sp:
        h.compute_vext(sol, sv, rvdw=rvdw)
    xm = torch.cat([xi.reshape(-1), xi.reshape(-1)])
    dm = torch.empty_like(xm)
    with Mixture(sp, [0.5, 0.5]) as mix:
        res["mixture_2_species_ms"] = timed(sp[0].stream, lambda: mix.energy_and_gradient_device(xm.data_ptr(), dm.data_ptr()))
    for h in sp:
        h.close()
    print(json.dumps(res))


def median(xs):
    return float(np.median(np.asarray(xs, dtype=np.float64)))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    import torch
    import torch.distributed as dist
    from mdft_b200 import Engine, PREC_FP64, PREC_MIXED, solve_batch, synth

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=180))
    n, box = (N_GRID, BOX) if not args.quick else (32, 16.0)
    rvdw = RVDW if not args.quick else 7.9
    ck = ck_file(MMAX)
    sv = synth.Solvent()
    W = max(1, args.workers)
    R = max(1, args.regions)
    warm_params, warm_meta, warm_note = None, None, None
    if args.form == "learned":
        from mdft_b200 import warmstart
        wpath = warmstart.default_weights()
        if wpath:
            warm_params, warm_meta = warmstart.load_params(wpath)
        else:
            warm_note = "no trained parameters in the package: solves start from the bulk guess"
    nets = []

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def opts_of(prec):
        return dict(m=5, pgtol=args.pgtol, ftol_abs=-1.0, itermax=3000, precision=prec, pgtol_mixed=args.pgtol_mixed,
                    polish=args.polish, guni_tol=args.guni_tol)

    class Form:
        """W engine handles of one precision solving the steps' solutes concurrently."""

        def __init__(self, name):
            self.name = name
            self.prec = PREC_FP64 if name == "fp64" else PREC_MIXED
            self.opts = opts_of(self.prec)
            if name == "learned" and warm_params is not None:
                # warm-started solves need the tighter stop rule to stay within 0.1 kJ/mol
                from mdft_b200 import warmstart
                self.opts.update(pgtol=min(args.pgtol, warmstart.LEARNED_PGTOL), guni_tol=min(args.guni_tol, warmstart.LEARNED_GUNI_TOL))
            self.engines = []
            for _ in range(W):
                e = Engine(n, box, MMAX, ck, temperature=sv.temperature, n0=sv.n0, device=local, precision=self.prec)
                if name == "learned" and warm_params is not None:
                    from mdft_b200 import warmstart
                    net = warmstart.WarmNet(n, device=local, params=warm_params, nout=warm_meta["nout"])
                    e.set_warm_net(net)
                    nets.append(net)
                self.engines.append(e)
            self.streams = [torch.cuda.ExternalStream(e.stream) for e in self.engines]

        def warm(self, idx):
            # every handle solves at least one solute (first-solve allocations happen here)
            solve_batch(self.engines, [sols[i] for i in idx], sv, rvdw=rvdw, handles=[k % W for k in range(len(idx))],
                        **self.opts)
            barrier()

        def timed(self, idx, xi_bufs=None):
            """solve sols[idx]; device time from an event before every stream's first kernel to
            one after every stream's last, the slowest rank's."""
            master = torch.cuda.current_stream()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(master)
            for st in self.streams:
                st.wait_event(ev0)
            res = solve_batch(self.engines, [sols[i] for i in idx], sv, rvdw=rvdw, xi_out=xi_bufs, **self.opts)
            for st in self.streams:
                e = torch.cuda.Event()
                e.record(st)
                master.wait_event(e)
            ev1.record(master)
            barrier()
            return res, max_over_ranks(ev0.elapsed_time(ev1), world, "cuda")

        def launches(self):
            return sum(e.launch_count for e in self.engines)

        def close(self):
            for e in self.engines:
                e.close()

    sols = [solute(sd, box) for sd in replica_seeds(rank, args.warmup + args.steps)]
    warm_idx = list(range(args.warmup))
    steps_idx = list(range(args.warmup, args.warmup + args.steps))

    if args.fft_compare:
        fft_compare(n, box, ck, sv, sols[0], rvdw, local)
        return
    if args.terms_compare:
        terms_compare(n, box, ck, sv, sols[0], rvdw, local)
        return

    if args.prof_solve and args.prof_grid:
        # the packed cluster of the profiling mode, solved: the mixed form and plain FP64 at the
        # bench's stop rule, and FP64 to max|df| <= 1e-6 as the reference dG
        pn, pbox = args.prof_grid, 0.375 * args.prof_grid
        rad = min(20.0, 0.4 * pbox)
        cl = synth.packed_cluster_solute(max(20, int(540 * (rad / 20.0) ** 3)), seed=2026, radius=rad)
        cl.xyz = synth.center_solute(cl.xyz, (pbox,) * 3)
        ckp = ck_file(args.prof_mmax, kmax=15.0)
        out = {"grid": pn, "box": pbox, "mmax": args.prof_mmax, "sites": len(cl.q)}
        forms = (("mixed", PREC_MIXED, dict(pgtol=PGTOL, guni_tol=GUNI_TOL)),
                 ("fp64", PREC_FP64, dict(pgtol=PGTOL, guni_tol=GUNI_TOL)),
                 ("fp64_ref", PREC_FP64, dict(pgtol=PGTOL_REF, guni_tol=0.01)))
        for name, prec, stop in forms:
            eng = Engine(pn, pbox, args.prof_mmax, ckp, temperature=sv.temperature, n0=sv.n0, device=local, precision=prec)
            t0 = time.time()
            r = eng.solve(cl, sv, rvdw=min(RVDW, 0.45 * pbox), m=5, ftol_abs=-1.0, itermax=3000, precision=prec, **stop)
            out[name] = {"dG": r["dG"], "evaluations": r["evaluations"], "status": r["status"], "pgnorm": r["pgnorm"],
                         "guni": r["guni"], "seconds": time.time() - t0}
            eng.close()
        out["dG_error_mixed"] = abs(out["mixed"]["dG"] - out["fp64_ref"]["dG"])
        out["dG_error_fp64"] = abs(out["fp64"]["dG"] - out["fp64_ref"]["dG"])
        print(json.dumps(out))
        return

    if args.evals and args.prof_grid:
        # profiling mode: the general kernels (np = 88, no = 330 at mmax 5) on a packed cluster
        # (600 sites in a 48 A box, proportionally fewer in a smaller one), mixed precision, N
        # evaluations at its guess density
        pn, pbox = args.prof_grid, 0.375 * args.prof_grid
        eng = Engine(pn, pbox, args.prof_mmax, ck_file(args.prof_mmax, kmax=15.0), temperature=sv.temperature, n0=sv.n0,
                     device=local, precision=PREC_MIXED)
        rad = min(20.0, 0.4 * pbox)  # 600 sites at >= 3 A fill a 20 A sphere; fewer in a smaller box
        cl = synth.packed_cluster_solute(max(20, int(540 * (rad / 20.0) ** 3)), seed=2026, radius=rad)
        cl.xyz = synth.center_solute(cl.xyz, (pbox,) * 3)
        eng.compute_vext(cl, sv, rvdw=min(RVDW, 0.45 * pbox))
        xi0 = eng.guess_density()
        for _ in range(args.evals):
            f, _, terms = eng.energy_and_gradient(xi0)
        print(json.dumps({"evals": args.evals, "grid": pn, "mmax": args.prof_mmax, "np": eng.np, "no": eng.no, "f": f}))
        eng.close()
        return

    if args.evals or args.solves:
        # profiling modes: N evaluations at the first solute's guess density, or N solves
        F = Form(args.form)
        eng = F.engines[0]
        if args.evals:
            eng.compute_vext(sols[0], sv, rvdw=rvdw)
            xi0 = eng.guess_density()
            for _ in range(args.evals):
                f, _, terms = eng.energy_and_gradient(xi0)
            print(json.dumps({"evals": args.evals, "f": f, "terms": list(map(float, terms))}))
        else:
            for i in range(args.solves):
                r = eng.solve(sols[args.warmup + i % args.steps], sv, rvdw=rvdw, **F.opts)
            print(json.dumps({"solves": args.solves, "dG": r["dG"], "evaluations": r["evaluations"],
                              "evaluations_mixed": r["evaluations_mixed"], "guni": r["guni"]}))
        F.close()
        for net in nets:
            net.close()
        return

    # ---- the headline form: R regions of solute in -> dG out (density resident in HBM),
    # each followed by one region of the same call returning the densities to pinned host memory ----
    H = Form(args.form)
    H.warm(warm_idx)
    xi_pinned = [torch.empty(int(np.prod(H.engines[0].shape)), dtype=torch.float64, pin_memory=True) for _ in steps_idx]
    xi_host = [b.numpy().reshape(H.engines[0].shape) for b in xi_pinned]
    rates, rates_e2e, launches = [], [], None
    with Clocks(local) as clk:
        for r in range(R):
            l0 = H.launches()
            timed, t_ms = H.timed(steps_idx)
            if launches is None:
                launches = H.launches() - l0
            rates.append(whole_job_rate(world, args.steps, t_ms))
            _, te_ms = H.timed(steps_idx, xi_bufs=xi_host)
            rates_e2e.append(whole_job_rate(world, args.steps, te_ms))
    value, e2e_value = median(rates), median(rates_e2e)
    evals = [r["evaluations"] + r.get("evaluations_mixed", 0) for r in timed]
    s0 = sols[0]
    h2d = 8 * (4 * s0.nsite + 4 * 3 * 2)  # solute q, sig, eps, xyz + solvent sites
    d2h = xi_host[0].nbytes + 8 * 6
    warm_stats = None
    if args.form == "learned" and warm_params is not None:
        warm_stats = {"starts": sum(e.warm_stats()["warm_starts"] for e in H.engines),
                      "fallbacks_to_bulk_guess": sum(e.warm_stats()["fallbacks"] for e in H.engines)}

    # ---- roofline of the dominant stage: per-stage CUDA events over every evaluation of one
    # solve of the first timed solute (the FP32 phase's kernels in the mixed forms) ----
    eng = H.engines[0]
    eng.set_timing(True)
    eng.solve(sols[steps_idx[0]], sv, rvdw=rvdw, **H.opts)
    st, cnt = eng.stage_times()
    eng.set_timing(False)
    per = {k: v / cnt for k, v in st.items()}
    sb = stage_bytes(n ** 3, eng.no, eng.np, 16, 8) if H.prec == PREC_FP64 else stage_bytes(n ** 3, eng.no, eng.np, 8, 4)
    dom = max(per, key=per.get)
    peak, peak_kind = measured_peak_hbm()
    achieved = sb[dom] / (per[dom] * 1e-3) / 1e9
    traffic = NCU_TRAFFIC_BYTES.get(("fp64" if H.prec == PREC_FP64 else "mixed", dom)) if n == N_GRID else None
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_source": peak_kind, "stage_ms": per, "algorithmic_bytes": sb[dom],
            "timed": "every evaluation of one solve (%d), per-stage CUDA events on the handle's stream" % cnt}
    H.close()

    # ---- the plain FP64 form on the same solutes, handles and stop rule (the metric's divisor) ----
    fp64 = None
    if args.form != "fp64" and not args.no_compare:
        P = Form("fp64")
        P.warm(warm_idx)
        rates64 = []
        for r in range(R):
            timed64, t64 = P.timed(steps_idx)
            rates64.append(whole_job_rate(world, args.steps, t64))
        P.close()
        fp64 = {"value": median(rates64), "regions": rates64,
                "evaluations_per_solve": [r["evaluations"] for r in timed64], "dG": [r["dG"] for r in timed64]}
    evals64 = fp64["evaluations_per_solve"] if fp64 else evals

    # ---- FP64 reference dG of the timed solutes, converged to PGTOL_REF (outside the timed regions) ----
    ref = Engine(n, box, MMAX, ck, temperature=sv.temperature, n0=sv.n0, device=local, precision=PREC_FP64)
    dg_ref = [ref.solve(sols[i], sv, rvdw=rvdw, **dict(opts_of(PREC_FP64), pgtol=PGTOL_REF, guni_tol=0.01))["dG"]
              for i in steps_idx]
    ref.close()
    dg_err = [abs(r["dG"] - d) for r, d in zip(timed, dg_ref)]
    if fp64:
        err64 = [abs(a - d) for a, d in zip(fp64["dG"], dg_ref)]
        fp64["dG_error_vs_fp64_max"] = max(err64)
        fp64["all_within_0.1"] = bool(max(err64) <= 0.1)
        del fp64["dG"]

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and not args.quick:
            threads = os.cpu_count() or 1
            te_cpu = cpu_oracle_eval_seconds(n, box, MMAX, ck, 2, threads, seed=replica_seeds(0, args.warmup + 1)[-1])
            epsolve = float(np.mean(evals64))
            cpu = {"value": 1.0 / (te_cpu * epsolve), "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": "2 FP64 evaluations of the first timed solute at its guess density on the host (oracle, "
                             "%d OpenMP threads) x %.1f evaluations per FP64 solve (this run's plain FP64 GPU solves); "
                             "the L-BFGS vector work is not counted" % (threads, epsolve)}
        clocks = clk.summary()
        form_text = ("plain FP64 from the bulk guess" if H.prec == PREC_FP64 else
                     ("learned warm start + " if warm_params is not None else "") +
                     "mixed: FP32 projections, FFTs, OZ, angular transforms, ideal/external terms and "
                     "L-BFGS vectors (BF16 history) with FP64 sums, then an FP64 check/polish")
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 / value * world, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if H.prec == PREC_FP64 else "f32+f64",
                "data": "synthetic",
                "config": {"workload": WORKLOAD % (n, box, MMAX, NSITE),
                           "form": form_text + " (vext + start + L-BFGS m=5 + pressure correction)",
                           "fp64_form": fp64,
                           "speedup_vs_fp64": (value / fp64["value"]) if fp64 else None,
                           "speedup_target": 5.0,
                           "warm_start": (
                               {"used": False, "note": "the learned warm start (--form learned) is built and trained; "
                                                       "this form starts from the bulk guess"}
                               if args.form == "mixed" else None) if args.form != "learned" else (
                               {"note": warm_note} if warm_params is None else
                               dict({"network": "periodic 3-D conv encoder-decoder, BF16 weights, %d outputs (%s)"
                                                % (warm_meta["nout"], "m <= 1 real basis" if warm_meta["nout"] == 4
                                                   else "all projections of the log-density"),
                                     "trained": {k: warm_meta.get(k) for k in ("train", "epochs", "final_val_loss",
                                                                               "solver")}},
                                    **warm_stats)),
                           "stop": STOP_TEXT % (args.pgtol, args.guni_tol),
                           "l2": "inputs larger than L2 (176 MB per field)",
                           "parallelism": ("replicas" if world > 1 else "single GPU") + ", %d concurrent solves per GPU" % W,
                           "workers": W,
                           "regions": {"value": rates, "e2e": rates_e2e, "statistic": "median of %d timed regions" % R},
                           "evaluations_per_solve": evals,
                           "fp32_evaluations_per_solve": [r.get("evaluations_mixed", 0) for r in timed],
                           "fp64_evaluations_per_solve": [r["evaluations"] for r in timed],
                           "evals_per_fp64_solve_constant": EVALS_PER_SOLVE_FP64["mean"],
                           "dG": [r["dG"] for r in timed], "dG_fp64": dg_ref,
                           "dG_error_vs_fp64_max": max(dg_err), "all_within_0.1": bool(max(dg_err) <= 0.1)},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks}
        print(json.dumps(line))
    for net in nets:
        net.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

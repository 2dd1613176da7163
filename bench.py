#!/usr/bin/env python3
"""bench.py -- timeslices/s of the per-timeslice LapH eigensystem path on B200.

Workload (one "step"): every timeslice of a seeded synthetic 32^3 x 64 gauge
field (U = exp(i*0.3*H), stout-smeared 5 x rho=0.1 on the device in FP64),
solved for the lowest nev = 120 eigenpairs of -Delta to a residual
||(-Delta)v - lambda v|| / (||v|| lambda_max) <= 1e-9 by the batched block
solver (FP32 filter matvecs on FP32 links, FP64 Gram / Cholesky /
Rayleigh-Ritz / residuals), phase-fixed.  All 64 timeslices run as one batch,
one CUDA graph launch per solve; the solver's degree, column block, guard and
filter tile are tuned on 4 timeslices first (--autotune 0: the defaults).

value : timeslices/s with links resident in HBM (device-timed, CUDA events on
        the solver's stream, K steps between barriers, max over ranks).
e2e   : the same through the public C ABI with host buffers: each step copies
        the links from pinned host memory and reads every eigenpair back
        (laph_solver_get_async into pinned buffers, overlapping the next step;
        the last step waits for its copies).
roofline: lap_cheb_mrhs (the FP32 multi-RHS Chebyshev stencil), the solver's
        own count of algorithmic bytes / its device-timed duration, against
        the measured HBM copy peak; frac on the correction form's bytes and
        frac_s8d on the plain recurrence's 72 B + links per site-vector-step.
parity: timeslice 0 of the timed batch against the CPU FP64 oracle's run.
cpu_baseline: the CPU FP64 oracle (restated reference ev_ts path: stout
        smearing + Krylov-Schur on T_DEG(B)) on one timeslice of the same
        workload, all host cores.
Also reported: the plain GPU form (MatShell + Krylov-Schur, its one-launch
MatMult event-timed), the learned window against the non-learned one on the
headline batch (window_ab), sub-records of the other benchmark configurations
(C1 with parity, C2 with parity, C3 with BF16 links, a wave of C4's mixed
volumes, a wave of C5), the source shape and displacement kernels on the
solved eigenvectors with an FP64 peak measured in place, the LIME reader's
throughput (lime_io), and the autotuner's choice.

--impl reference runs that CPU path as the reference arm without loading the
product library (inputs from the oracle's generator), plus one round of the
reference's MPI layout (one single-threaded timeslice per core) recorded
beside it; --cpu-layout per-core times that layout as the arm itself.
Multi-GPU (torchrun): timeslices are independent; each rank solves its own
64-timeslice batch (weak scaling), no collective on the data path.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # 32^3 x 64, eps 0.3, stout 5 x 0.1, nev 120 (+16 guard), FP32 filter links
    "c3": dict(L=32, T=64, eps=0.3, seed=1229, smear="stout", p1=0.1, p2=0.0, iters=5, compat=1, nev=120,
               guard=16, link_prec="fp32", tol=1e-9, deg=60),
    # 24^3 x 48, eps 0.3, HYP 0.62/0.62 x 1, nev 120
    "c2": dict(L=24, T=48, eps=0.3, seed=1228, smear="hyp", p1=0.62, p2=0.62, iters=1, compat=0, nev=120,
               guard=16, link_prec="fp32", tol=1e-9, deg=60),
    # 8^3 x 16, eps 0.4, stout 3 x 0.1, nev 60
    "c1": dict(L=8, T=16, eps=0.4, seed=1227, smear="stout", p1=0.1, p2=0.0, iters=3, compat=1, nev=60,
               guard=16, link_prec="fp32", tol=1e-9, deg=32,
               lam_c_ref=2.07),  # the reference's window must lie above lambda_60 (1.88 here); 0.65 suits the rest
    # one launch mixing 16^3 x 32 (nev 60), 24^3 x 48 (nev 120), 32^3 x 64 (nev 180), APE 0.5 x 10
    "c4": dict(mixed=[(16, 32, 60, 1230), (24, 48, 120, 1231), (32, 64, 180, 1232)], eps=0.3, smear="ape", p1=0.5,
               p2=0.0, iters=10, compat=1, guard=16, link_prec="fp32", tol=1e-9, deg=48, L=32, T=144, nev=180),
    # 48^3 x 96, eps 0.25, stout 6 x 0.1, nev 220, solved in memory-bounded waves
    "c5": dict(L=48, T=96, eps=0.25, seed=1233, smear="stout", p1=0.1, p2=0.0, iters=6, compat=1, nev=220,
               guard=16, link_prec="fp32", tol=1e-9, deg=48, wave=16),
}
def hyp_scan_grid(a1i, a1f, a2i, a2f):
    """tune_hyp's (alpha_1, alpha_2) grid with its own loops (src/tune_hyp.cpp:116-117)."""
    out, a1 = [], a1i
    while a1 <= a1f:
        a2 = a2i
        while a2 <= a2f:
            out.append((a1, a2))
            a2 += 0.05
        a1 += 0.05
    return out


# 32^3, HYP x 3, nev 120: timeslice 0 of seed 1234 under a 4 x 4 (alpha_1, alpha_2) grid in one batch
CONFIGS["c6"] = dict(L=32, T=16, eps=0.3, seed=1234, smear="hyp", p1=0.4, p2=0.4, iters=3, compat=1, nev=120,
                     guard=16, link_prec="fp32", tol=1e-9, deg=56, scan=hyp_scan_grid(0.4, 0.56, 0.4, 0.56))
HBM_FALLBACK = 6650.0
# DRAM bytes (read + write) of one k_cheb_mrhs2 launch over its algorithmic bytes, from an ncu capture of the same
# kernel on 32^3 x 4 timeslices (2.125 GB / 2.155 GB); the filter's traffic grows with the site-vectors processed,
# so a bench launch's traffic is this ratio times its algorithmic bytes
NCU_TRAFFIC_RATIO = 0.986


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def generate_links(cfg, seed_offset=0, oracle_generator=False):
    """Spatial links of one batch: list of (L, nev, links (V3, 3, 3, 3)).  oracle_generator: the oracle's
    restatement of the seeded generator (same field to rounding), for the reference arm, which must not load the
    library."""
    if oracle_generator:
        import oracle as gen
    else:
        import laph_eigsys_b200 as gen
    out = []
    if cfg.get("scan"):
        conf = gen.gauge_random(cfg["L"], 1, cfg["eps"], cfg["seed"] + seed_offset)
        return [(cfg["L"], cfg["nev"], np.ascontiguousarray(conf[0, :, 1:4])) for _ in cfg["scan"]]
    for L, T, nev, seed in cfg.get("mixed") or [(cfg["L"], cfg.get("wave") or cfg["T"], cfg["nev"], cfg["seed"])]:
        conf = gen.gauge_random(L, T, cfg["eps"], seed + seed_offset)
        for t in range(T):
            out.append((L, nev, np.ascontiguousarray(conf[t, :, 1:4])))
    return out


def make_opts(cfg):
    import laph_eigsys_b200 as lb
    kinds = {"stout": lb.SMEAR_STOUT, "ape": lb.SMEAR_APE, "hyp": lb.SMEAR_HYP, "none": lb.SMEAR_NONE}
    return lb.solve_opts(smear_kind=kinds[cfg["smear"]], smear_p1=cfg["p1"], smear_p2=cfg["p2"],
                         smear_iters=cfg["iters"], smear_compat=cfg["compat"], guard=cfg["guard"],
                         link_prec=lb.LINKS_BF16 if cfg["link_prec"] == "bf16" else lb.LINKS_FP32, tol=cfg["tol"],
                         max_it=400, deg=cfg["deg"], phase_fix=1, seed=1227, block=cfg.get("block", 0),
                         filter_kernel=cfg.get("filter_kernel", 1), jacobi_sweeps=cfg.get("sweeps", 0),
                         filter_tile=cfg.get("tile", 0), host_loop=cfg.get("host_loop", 0),
                         **({"direct_resid": cfg["direct_resid"]} if cfg.get("direct_resid") is not None else {}),
                         lam_cut=cfg.get("lam_cut0", 0.0),
                         window={"mlp": lb.WINDOW_MLP, "lanczos": lb.WINDOW_LANCZOS, "fixed": lb.WINDOW_FIXED}[
                             cfg.get("window", "mlp")])


def autotune_cfg(cfg, batch, device, nsample, cache):
    """laph_solver_autotune on the first nsample timeslices of the batch; the chosen deg / block / guard replace
    the configuration's before the measured solver is built."""
    import laph_eigsys_b200 as lb
    model = None
    if cfg.get("window", "mlp") == "mlp":
        from laph_eigsys_b200 import window as lw
        model = lw.load_model()
    t0 = time.perf_counter()
    opts, res = lb.autotune([(L, nev) for L, nev, _ in batch], [U for _, _, U in batch], nsample=nsample,
                            opts=make_opts(cfg), model=model, device=device, cache=cache)
    res["seconds"] = time.perf_counter() - t0
    res["sample_timeslices"] = min(nsample, len(batch))
    res["before"] = {"deg": cfg["deg"], "block": cfg.get("block", 0) or 32, "guard": cfg["guard"],
                     "tile": cfg.get("tile", 0) or 128}
    cfg["deg"], cfg["block"], cfg["guard"], cfg["tile"] = opts.deg, opts.block, opts.guard, opts.filter_tile
    return res


def make_solver(cfg, device, batch):
    import laph_eigsys_b200 as lb
    probs = [(L, nev) for L, nev, _ in batch]
    s = lb.Solver(probs, opts=make_opts(cfg), device=device)
    for i, (a1, a2) in enumerate(cfg.get("scan") or []):
        s.set_smear(i, a1, a2)  # the batched tune_hyp scan: one copy of the timeslice per grid point
    return s


def cpu_reference_step(cfg, links_ts, lam_c, deg_ref, threads, L=None, nev=None, keep=False):
    """One timeslice of the reference ev_ts path on the CPU oracle: smear + Krylov-Schur on T_DEG(B)."""
    import oracle as orc
    orc.set_threads(threads)
    L = L or cfg["L"]
    nev = nev or cfg["nev"]
    t0 = time.perf_counter()
    if cfg["smear"] == "stout":
        Us = orc.smear_stout(links_ts, L, cfg["p1"], cfg["iters"], cfg["compat"])
    elif cfg["smear"] == "ape":
        Us = orc.smear_ape(links_ts, L, cfg["p1"], cfg["iters"], cfg["compat"])
    elif cfg["smear"] == "hyp":
        Us = orc.smear_hyp(links_ts, L, cfg["p1"], cfg["p2"], cfg["iters"])
    else:
        Us = links_ts
    st, theta, V, nconv, its, nmv = orc.eps_solve(Us, L, 12.0, lam_c, deg_ref, nev, tol=1e-10, max_it=100)
    Vf, ph = orc.fix_phase(V)
    dt = time.perf_counter() - t0
    info = dict(status=st, nconv=nconv, restarts=its, matvecs=nmv)
    if keep:
        info["_solution"] = (Us, Vf)
    return dt, info


def plain_gpu(cfg, batch, lam_c, ntimeslices, device, deg_ref=12):
    """The plain GPU form of the same workload: per timeslice, links into a
    MatShell context, smearing on the device, SLEPc-style Krylov-Schur on
    T_DEG(B) with the Krylov basis in device memory driving the GPU MatMult,
    then recover_spectrum and fix_phase -- the reference's ev_ts loop body with
    the MatShell product on the GPU."""
    import torch
    import laph_eigsys_b200 as lb
    kinds = {"stout": lb.SMEAR_STOUT, "ape": lb.SMEAR_APE, "hyp": lb.SMEAR_HYP, "none": lb.SMEAR_NONE}
    L, nev = batch[0][0], batch[0][1]
    ctx = lb.Context(L, 12.0, lam_c, deg_ref, device=device)
    out = {"unit": "timeslices/s", "timeslices": ntimeslices, "basis": "device", "deg": deg_ref, "lam_l": 12.0,
           "lam_c": lam_c, "tol": 1e-10, "ncv": "max(2 nev, nev+15)"}
    t0 = time.perf_counter()
    nmv, rs = 0, 0
    for t in range(ntimeslices):
        ctx.set_links(batch[t][2])
        ctx.smear(kinds[cfg["smear"]], cfg["p1"], cfg["p2"], cfg["iters"], cfg["compat"])
        st, theta, V, nconv, its, nm = ctx.eps_solve(nev, tol=1e-10, max_it=100, device_basis=True)
        if st != 0:
            out["status"] = f"not converged on timeslice {t}"
        lb.recover_spectrum(theta, deg_ref, 12.0, lam_c)
        lb.fix_phase(V)
        nmv += nm
        rs += its
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    ctx.close()
    out.update({"value": ntimeslices / dt, "seconds": dt, "matvecs": nmv, "restarts": rs})
    return out


def _per_core_step(job):
    """One single-threaded timeslice of the reference path (a worker of the per-core layout)."""
    cfg, U, lam_c, deg_ref, L, nev = job
    return cpu_reference_step(cfg, U, lam_c, deg_ref, 1, L, nev)


def run_reference_per_core(args, cfg, batch, lam_c, deg_ref, threads):
    """The reference's MPI layout (src/ev_ts.cpp:103-119): one single-threaded timeslice per core at once; a step is
    one such round of `threads` timeslices, timed by the wall clock around it."""
    import multiprocessing as mp
    jobs = [(cfg, batch[i % len(batch)][2], lam_c, deg_ref, batch[0][0], batch[0][1]) for i in range(threads)]
    with mp.get_context("spawn").Pool(threads) as pool:
        for _ in range(args.warmup):
            pool.map(_per_core_step, jobs)
        tot, info = 0.0, None
        for _ in range(args.steps):
            t0 = time.perf_counter()
            out = pool.map(_per_core_step, jobs)
            tot += time.perf_counter() - t0
            info = out[0][1]
    return args.steps * threads / tot, tot, info


def run_reference(args, cfg):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    batch = generate_links(cfg, oracle_generator=True)
    lam_c = cfg.get("lam_c_ref", 0.65)
    deg_ref = 12
    if args.cpu_layout == "per-core":
        value, tot, info = run_reference_per_core(args, cfg, batch, lam_c, deg_ref, threads)
        sample = (f"{threads} single-threaded timeslices at once per step ({batch[0][0]}^3, nev {batch[0][1]}, "
                  f"smear + Krylov-Schur on T_{deg_ref}(B), LAM_L 12, LAM_C {lam_c}, tol 1e-10)")
        line = {"impl": "reference", "metric": "timeslices/s to nev pairs @resid<=1e-9", "value": value,
                "unit": "timeslices/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "c128", "data": "synthetic", "config": workload_config(cfg),
                "cpu_baseline": {"value": value, "unit": "timeslices/s", "cores": threads, "kind": "port",
                                 "layout": "one timeslice per core", "sample": sample, "last": info},
                "e2e": {"value": value, "unit": "timeslices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    for _ in range(args.warmup):
        cpu_reference_step(cfg, batch[0][2], lam_c, deg_ref, threads, batch[0][0], batch[0][1])
    tot = 0.0
    info = None
    for k in range(args.steps):
        L, nev, U = batch[k % len(batch)]
        dt, info = cpu_reference_step(cfg, U, lam_c, deg_ref, threads, L, nev)
        tot += dt
    value = args.steps / tot
    sample = (f"1 timeslice per step ({batch[0][0]}^3, nev {batch[0][1]}, smear + Krylov-Schur on T_{deg_ref}(B), "
              f"LAM_L 12, LAM_C {lam_c}, tol 1e-10)")
    cpu = {"value": value, "unit": "timeslices/s", "cores": threads, "kind": "port",
           "layout": "OpenMP inside one timeslice", "sample": sample, "last": info,
           "inputs": "seeded field from the oracle's generator (the library is not loaded in this arm)"}
    if not args.no_per_core:
        # the reference's MPI layout (src/ev_ts.cpp:103-119): one round of one single-threaded timeslice per core,
        # wall clock around the round, no warm-up round (a round is minutes at 32^3)
        import multiprocessing as mp
        jobs = [(cfg, batch[i % len(batch)][2], lam_c, deg_ref, batch[0][0], batch[0][1]) for i in range(threads)]
        with mp.get_context("spawn").Pool(threads) as pool:
            t0 = time.perf_counter()
            out = pool.map(_per_core_step, jobs)
            wall = time.perf_counter() - t0
        cpu["per_core"] = {"value": threads / wall, "unit": "timeslices/s", "cores": threads,
                           "layout": "one single-threaded timeslice per core (the reference's MPI layout)",
                           "sample": f"one round of {threads} timeslices, wall clock", "seconds": wall,
                           "last": out[0][1]}
        cpu["value_best_layout"] = max(value, threads / wall)
    line = {"impl": "reference", "metric": "timeslices/s to nev pairs @resid<=1e-9", "value": value,
            "unit": "timeslices/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic", "config": workload_config(cfg),
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": "timeslices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def solve_config(cfg, device, reps=1, window=None, link_prec=None, wave=None, parity=None, no_cpu=False):
    """One benchmark configuration as a compact sub-record: its batch (or one memory-bounded wave of it) solved
    once untimed (graph capture) and `reps` times timed with CUDA events on the solver's stream, with iterations,
    residual, the filter's algorithmic bandwidth and, where asked, parity of timeslice 0 (or all timeslices of a
    small lattice) against the oracle.  Everything here runs outside the headline's timed region."""
    import torch
    import laph_eigsys_b200 as lb
    cfg = dict(cfg)
    if window:
        cfg["window"] = window
    if link_prec:
        cfg["link_prec"] = link_prec
    if wave:
        if cfg.get("mixed"):
            cfg["mixed"] = [(L, wave[i], nev, seed) for i, (L, T, nev, seed) in enumerate(cfg["mixed"])]
        else:
            cfg["wave"] = wave
    batch = generate_links(cfg)
    solver = make_solver(cfg, device, batch)
    if cfg.get("window", "mlp") == "mlp":
        from laph_eigsys_b200 import window as lw
        lw.set_model(solver, lw.load_model())
    for i, (_, _, U) in enumerate(batch):
        solver.set_links(i, U)
    stream = torch.cuda.ExternalStream(solver.stream())
    st, res = solver.run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    filt_ms, fb = 0.0, [0.0, 0.0]
    e0.record(stream)
    for _ in range(reps):
        st, res = solver.run()
        filt_ms += solver.timings()[1]
        b = solver.filter_bytes()
        fb[0] += b[0]
        fb[1] += b[1]
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    hbm, src = peaks()
    kb = cfg.get("block") or 32
    out = {"workload": workload_config(cfg)["workload"], "timeslices": len(batch), "status": st,
           "value": len(batch) / (ms / 1e3), "unit": "timeslices/s", "ms_per_solve": ms,
           "outer_iterations": max(r["iters"] for r in res), "max_resid": max(r["max_resid"] for r in res),
           "window": cfg.get("window", "mlp"), "links": cfg["link_prec"], "deg": cfg["deg"],
           "window_fallbacks": sum(r["window_fallback"] for r in res),
           "filter": {"ms_per_solve": filt_ms / reps, "achieved_gbs": fb[0] / (filt_ms / 1e3) / 1e9,
                      "frac": fb[0] / (filt_ms / 1e3) / 1e9 / hbm,
                      "frac_s8d": fb[1] / (filt_ms / 1e3) / 1e9 / hbm, "peak_gbs": hbm, "peak_source": src,
                      "bytes_model_s8d": f"72 + {112 if cfg['link_prec'] == 'bf16' else 216}/{kb} B"}}
    if parity and not no_cpu:
        import oracle as orc
        orc.set_threads(os.cpu_count() or 1)
        worst = {}
        for t in parity["timeslices"]:
            L, nev, U = batch[t]
            Us = smear_oracle(cfg, U, L)
            if parity["kind"] == "dense":
                w, Vd = np.linalg.eigh(orc.neglap_dense(Us, L))
                Vo, _ = orc.fix_phase(Vd[:, :nev])
            else:
                lam = -solver.get(t, vectors=False)[0]
                sto, _, Vk, _, _, _ = orc.eps_solve(Us, L, 12.0, float(1.1 * lam[-1]), 12, nev, tol=1e-12,
                                                     max_it=200)
                Vo, _ = orc.fix_phase(Vk)
            r = orc.compare_eigensystems(Us, L, solver.get(t)[1], Vo)
            for k_, v in r.items():
                if isinstance(v, float) and (k_.startswith("max") or k_ == "block_proj"):
                    worst[k_] = max(worst.get(k_, 0.0), v)
            g = r["gap_min_isolated"]
            if g is not None:
                worst["gap_min_isolated"] = min(worst.get("gap_min_isolated", g), g)
        worst["against"] = ("oracle smearing + dense eigh of the assembled -Delta" if parity["kind"] == "dense" else
                            "oracle smearing + FP64 Krylov-Schur on T_12(B), tol 1e-12")
        worst["timeslices"] = list(parity["timeslices"])
        out["parity"] = worst
    solver.close()
    del batch
    return out


def smear_oracle(cfg, U, L):
    import oracle as orc
    if cfg["smear"] == "stout":
        return orc.smear_stout(U, L, cfg["p1"], cfg["iters"], cfg["compat"])
    if cfg["smear"] == "ape":
        return orc.smear_ape(U, L, cfg["p1"], cfg["iters"], cfg["compat"])
    if cfg["smear"] == "hyp":
        return orc.smear_hyp(U, L, cfg["p1"], cfg["p2"], cfg["iters"])
    return U


def workload_config(cfg):
    if cfg.get("mixed"):
        shape = " + ".join(f"{L}^3x{T} (nev {nev})" for L, T, nev, _ in cfg["mixed"]) + " in one batch"
    elif cfg.get("scan"):
        a1 = sorted({round(a, 6) for a, _ in cfg["scan"]})
        a2 = sorted({round(b, 6) for _, b in cfg["scan"]})
        shape = (f"{cfg['L']}^3 timeslice 0 x {len(cfg['scan'])} HYP (alpha_1, alpha_2) grid points "
                 f"(alpha_1 {a1[0]}..{a1[-1]}, alpha_2 {a2[0]}..{a2[-1]}, step 0.05) in one batch, nev {cfg['nev']}")
    elif cfg.get("wave"):
        shape = f"{cfg['L']}^3x{cfg['T']} in waves of {cfg['wave']} timeslices (one wave per step), nev {cfg['nev']}"
    else:
        shape = f"{cfg['L']}^3x{cfg['T']}, nev {cfg['nev']}"
    return {"workload": f"{shape}, eps {cfg['eps']} {cfg['smear']} {cfg['iters']}x{cfg['p1']}, "
                        f"+{cfg['guard']} guard, resid<=1e-9",
            "L": cfg["L"], "timeslices": cfg["T"], "nev": cfg["nev"], "guard": cfg["guard"], "deg": cfg["deg"],
            "block": cfg.get("block") or 32, "tile": cfg.get("tile") or 128,
            "window": cfg.get("window", "mlp"),
            "links": cfg["link_prec"], "filter": "fp32", "rayleigh_ritz": "fp64",
            "l2": "inputs larger than L2 (each 64-timeslice block of vectors is 8 GB)"}


def sourceshape_flops(L, nev):
    """FP64 flops of the source-shape kernel: per parity class the upper 32-site tile pairs of V_c V_c^dag,
    9 nev complex FMAs per site pair."""
    nc = (L // 2) ** 3
    t = (nc + 31) // 32
    return 8 * (t * (t + 1) // 2) * 32 * 32 * 9 * nev * 8.0


def measure_displacement(solver, stream, batch, reps=4):
    """Covariant displacement of the solved eigenvectors along x, y, z in place on the device (CUDA events on the
    solver's stream); HBM roofline: 48 B read + 48 B written per site and eigenvector plus the forward links."""
    import torch
    L, nev, _ = batch[0]
    n = min(reps, len(batch))
    W = torch.empty(3 * L ** 3 * nev, dtype=torch.complex128, device="cuda")
    solver.displace_device(0, 0, W.data_ptr())  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(n):
        for d in range(3):
            solver.displace_device(i, d, W.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / (3 * n)
    byts = L ** 3 * nev * 96.0 + L ** 3 * 144.0 * ((nev + 15) // 16)
    hbm, src = peaks()
    del W
    return {"workload": f"{L}^3 x nev {nev} eigenvectors, one direction per launch, FP64", "ms_per_launch": ms,
            "bytes_per_launch": byts, "achieved_gbs": byts / (ms / 1e3) / 1e9, "peak_gbs": hbm, "peak_source": src,
            "frac": byts / (ms / 1e3) / 1e9 / hbm, "launches": 3 * n}


def measure_matvec_fp64(cfg, batch, device, deg=12, reps=20):
    """The plain form's MatShell MatMult y = T_deg(B) x (FP64, one vector, device pointers), CUDA events around
    each of `reps` products on the context's stream.  Algorithmic bytes per site and B application: the 6 links a site
    reads once (its 3 forward links; the backward ones are other sites' forward links) = 432, plus x read,
    z read, y written = 3 x 48."""
    import torch
    import laph_eigsys_b200 as lb
    L = batch[0][0]
    ctx = lb.Context(L, 12.0, 0.6, deg, device=device)
    ctx.set_links(batch[0][2])
    dim = 3 * L ** 3
    x = torch.randn(dim, dtype=torch.complex128, device="cuda")
    y = torch.empty_like(x)
    for _ in range(3):
        ctx.matmult_device(x.data_ptr(), y.data_ptr(), deg)  # warm-up
    stream = torch.cuda.ExternalStream(ctx.stream())
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for a, b in evs:
        a.record(stream)
        ctx.matmult_device(x.data_ptr(), y.data_ptr(), deg)
        b.record(stream)
    torch.cuda.synchronize()
    host_ms = (time.perf_counter() - t0) * 1e3 / reps
    ms = sum(a.elapsed_time(b) for a, b in evs) / reps
    ctx.close()
    byts = deg * L ** 3 * (432.0 + 3 * 48.0)
    hbm, src = peaks()
    return {"workload": f"T_{deg}(B) x on one {L}^3 vector, FP64 (laph_matmult, device pointers)",
            "ms_per_matmult": ms, "bytes_per_matmult": byts, "achieved_gbs": byts / (ms / 1e3) / 1e9,
            "peak_gbs": hbm, "peak_source": src, "frac": byts / (ms / 1e3) / 1e9 / hbm,
            "kernel": "k_cheb64_fused (one cooperative launch per product)",
            "timing": "CUDA events on the context's stream around each call (device time of the product and its "
                      "error-flag read), mean of the calls", "host_ms_per_matmult": host_ms}


def measure_lime_io(L=32, T=16, no_cpu=False):
    """The LIME/ILDG gauge reader on the host: a seeded L^3 x T FP64 configuration written to a scratch directory
    beside this file, then read whole with laph_lime_read_gauge once after dropping the file from the page cache
    (fsync + POSIX_FADV_DONTNEED) and once warm; beside it the oracle's restatement of the reference's reader
    (read_lime_gauge_field_doubleprec_timeslices: one thread, the whole file) on the warm file.  Bytes = the
    binary record, V3 T 72 8."""
    import tempfile
    import laph_eigsys_b200 as lb
    nbytes = L ** 3 * T * 72 * 8
    out = {"workload": f"{L}^3 x {T} FP64 ILDG file, all timeslices", "bytes": nbytes, "threads": os.cpu_count()}
    with tempfile.TemporaryDirectory(dir=os.path.dirname(os.path.abspath(__file__)), prefix="_lime_") as tmp:
        path = os.path.join(tmp, "conf.1227")
        conf = lb.gauge_random(L, T, 0.3, 1227)
        lb.lime_write_gauge(path, conf, L, T)
        fd = os.open(path, os.O_RDONLY)
        try:
            os.fsync(fd)
            os.posix_fadvise(fd, 0, 0, os.POSIX_FADV_DONTNEED)
            out["cold_cache"] = "dropped (fsync + POSIX_FADV_DONTNEED)"
        except OSError as e:
            out["cold_cache"] = f"not dropped: {e}"
        finally:
            os.close(fd)
        t0 = time.perf_counter()
        got = lb.lime_read_gauge(path, T, L, 0, T - 1)
        t1 = time.perf_counter()
        out["cold_gbs"] = nbytes / (t1 - t0) / 1e9
        t0 = time.perf_counter()
        got = lb.lime_read_gauge(path, T, L, 0, T - 1)
        t1 = time.perf_counter()
        out["warm_gbs"] = nbytes / (t1 - t0) / 1e9
        out["matches_written"] = bool(np.array_equal(got, conf))
        del got
        if not no_cpu:
            import oracle as orc
            t0 = time.perf_counter()
            st, ref = orc.lime_read_gauge(path, T, L, 0, T - 1)
            t1 = time.perf_counter()
            out["oracle_reader_warm_gbs"] = nbytes / (t1 - t0) / 1e9
            out["oracle_matches"] = bool(st == 0 and np.array_equal(ref, conf))
    return out


def measure_sourceshape(solver, stream, batch, no_cpu, reps=4):
    """psi(r) of the first solved timeslices in place on the device (CUDA events on the solver's stream), and the
    oracle's restatement on one 16^3 eigensystem beside the device kernel on the same input."""
    import torch
    import laph_eigsys_b200 as lb
    L, nev, _ = batch[0]
    n = min(reps, len(batch))
    fma_peak, dmma_peak = lb.probe_fp64(torch.cuda.current_device())
    solver.sourceshape(0)  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(n):
        solver.sourceshape(i)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n
    fl = sourceshape_flops(L, nev)
    out = {"workload": f"psi(r) of {L}^3 x nev {nev}, (L/2)^3 = {(L // 2) ** 3} displacements, FP64",
           "kernel": "k_ss_tile, FP64 tensor path (mma.sync m8n8k4.f64)",
           "ms_per_timeslice": ms, "tflops": fl / (ms / 1e3) / 1e12, "bound": "fp64 tensor (DMMA)",
           "fp64_peak_tflops": dmma_peak, "fp64_fma_tflops": fma_peak,
           "peak_source": "laph_probe_fp64 in this run (saturating mma.sync.m8n8k4.f64 loop)",
           "frac": fl / (ms / 1e3) / 1e12 / dmma_peak, "timeslices": n}
    if not no_cpu:
        import oracle as orc
        Ls, nevs = 16, min(nev, 120)
        rng = np.random.default_rng(16)
        V, _ = np.linalg.qr(rng.normal(size=(3 * Ls ** 3, nevs)) + 1j * rng.normal(size=(3 * Ls ** 3, nevs)))
        V = np.asfortranarray(V)
        orc.set_threads(os.cpu_count() or 1)
        t0 = time.perf_counter()
        ref = orc.sourceshape(V, Ls)
        cpu_s = time.perf_counter() - t0
        lb.sourceshape(V, Ls)
        t1 = time.perf_counter()
        got = lb.sourceshape(V, Ls)
        gpu_s = time.perf_counter() - t1
        out["cpu_sample"] = {"workload": f"16^3 x nev {nevs} (random orthonormal block)", "cpu_seconds": cpu_s,
                             "cores": os.cpu_count() or 1, "kind": "port",
                             "gpu_seconds_host_api": gpu_s,
                             "max_rel_diff": float(np.abs(got - ref).max() / np.abs(ref).max())}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(CONFIGS))
    ap.add_argument("--deg", type=int, default=None)
    ap.add_argument("--link-prec", default=None, choices=["bf16", "fp32"])
    ap.add_argument("--timeslices", type=int, default=None)
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--filter-kernel", type=int, default=1, choices=[0, 1, 2, 3, 4, 5])
    ap.add_argument("--direct-resid", type=float, default=None,
                    help="passes above this largest wanted residual filter V directly in FP32 (< 0: never; "
                         "default: the library's)")
    ap.add_argument("--guard", type=int, default=None)
    ap.add_argument("--sweeps", type=int, default=0)
    ap.add_argument("--lam-cut0", type=float, default=0.0)
    ap.add_argument("--window", default="mlp", choices=["mlp", "lanczos", "fixed"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-shape", action="store_true")
    ap.add_argument("--no-io", action="store_true")
    ap.add_argument("--host-loop", action="store_true",
                    help="drive the outer iteration from the host (same kernels; ncu cannot profile kernels inside "
                         "a graph with conditional nodes)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the learned-window A/B and the sub-records of the other benchmark configurations")
    ap.add_argument("--autotune", type=int, default=4, metavar="NSAMPLE",
                    help="tune deg / block / guard on the first NSAMPLE timeslices before measuring (0: off, the "
                         "configuration's own settings)")
    ap.add_argument("--tune-cache", default=None, help="autotuner cache file")
    ap.add_argument("--cpu-layout", default="omp", choices=["omp", "per-core"],
                    help="reference arm: OpenMP inside one timeslice (default) or one single-threaded timeslice per "
                         "core (the reference's MPI layout; a step is one round over all cores, minutes at 32^3)")
    ap.add_argument("--plain-timeslices", type=int, default=2)
    ap.add_argument("--no-per-core", action="store_true",
                    help="reference arm: skip the extra per-core round recorded beside the OpenMP figure")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    cfg = dict(CONFIGS[args.config])
    if args.deg:
        cfg["deg"] = args.deg
    if args.link_prec:
        cfg["link_prec"] = args.link_prec
    if args.timeslices:
        cfg["T"] = args.timeslices
    cfg["block"] = args.block
    cfg["sweeps"] = args.sweeps
    cfg["lam_cut0"] = args.lam_cut0
    cfg["window"] = args.window
    if args.guard is not None:
        cfg["guard"] = args.guard
    cfg["filter_kernel"] = args.filter_kernel
    cfg["direct_resid"] = args.direct_resid
    cfg["host_loop"] = int(args.host_loop)
    if args.impl == "reference":
        return run_reference(args, cfg)

    import torch
    import laph_eigsys_b200 as lb
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    batch = generate_links(cfg, seed_offset=rank * 1000)
    T = len(batch)
    tune = autotune_cfg(cfg, batch, local, args.autotune, args.tune_cache) if args.autotune > 0 else None
    solver = make_solver(cfg, local, batch)
    if cfg.get("window", "mlp") == "mlp":
        from laph_eigsys_b200 import window as lw
        lw.set_model(solver, lw.load_model())
    for i in range(T):
        solver.set_links(i, batch[i][2])
    stream = torch.cuda.ExternalStream(solver.stream())

    results = None
    for _ in range(args.warmup):
        st, results = solver.run()
        if st != 0:
            raise RuntimeError(f"solver did not converge: {results[:2]}")

    # ---- value: links resident in HBM --------------------------------------
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    filt_ms, fsv, flaunch, launches, iters = 0.0, 0, 0, 0, []
    fbytes_tot = [0.0, 0.0]
    window_fallbacks = 0
    e0.record(stream)
    for _ in range(args.steps):
        st, results = solver.run()
        if st != 0:
            raise RuntimeError("solver did not converge in a timed step")
        tm = solver.timings()
        cn = solver.counters()
        filt_ms += tm[1]
        fsv += cn[0]
        fb = solver.filter_bytes()
        fbytes_tot[0] += fb[0]
        fbytes_tot[1] += fb[1]
        flaunch += cn[1]
        launches += cn[2]
        iters.append(max(r["iters"] for r in results))
        loop_info = solver.loop_info()
        window_fallbacks = sum(r["window_fallback"] for r in results)
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms)
    value = world * T * args.steps / (ms_max / 1000.0)
    max_resid = max(r["max_resid"] for r in results)

    # ---- roofline of lap_cheb_mrhs -----------------------------------------
    # algorithmic bytes of the timed filter passes, counted by the solver pass by pass (each pass's own degree,
    # its unlocked columns and column blocks): what the correction-form recurrence moves, and the unit
    # of one step Y = 2BX - Z (72 B per site-vector-step + links once per column block)
    kb = cfg["block"] or 32
    link_b = 112 if cfg["link_prec"] == "bf16" else 216
    alg_bytes, alg_s8d = fbytes_tot
    hbm, src = peaks()
    achieved = alg_bytes / (filt_ms / 1000.0) / 1e9 if filt_ms > 0 else None
    achieved_s8d = alg_s8d / (filt_ms / 1000.0) / 1e9 if filt_ms > 0 else None
    fk = cfg.get("filter_kernel", 1)
    kname = ({2: "k_cheb_mrhs3", 3: "k_cheb_mrhs4", 4: "k_cheb_mrhs5", 5: "k_cheb_mrhs6"}.get(fk, "k_cheb_mrhs2")) if fk >= 1 and kb <= 64 else "k_cheb_mrhs"
    roofline = {"kernel": f"{kname} (lap_cheb_mrhs)", "bound": "hbm", "achieved": achieved, "peak": hbm,
                "unit": "GB/s", "frac": achieved / hbm if achieved else None, "peak_source": src,
                "traffic": NCU_TRAFFIC_RATIO * alg_bytes / max(flaunch, 1) if kname == "k_cheb_mrhs2" else None,
                "traffic_source": "ncu capture of 32^3 x 4, scaled by site-vectors",
                "avg_launch_ms": filt_ms / max(flaunch, 1),
                "bytes_per_launch": alg_bytes / max(flaunch, 1),
                "filter_share_of_step": filt_ms / ms if ms > 0 else None,
                "achieved_s8d": achieved_s8d, "frac_s8d": achieved_s8d / hbm if achieved_s8d else None,
                "bytes_model_s8d": f"72 + {link_b}/{kb} B per site-vector-step"}

    # ---- e2e through the public API with host buffers ----------------------
    e2e = None
    if not args.no_e2e:
        hl = []
        for L_, nev_, U_ in batch:
            pin = torch.empty(U_.shape, dtype=torch.complex128, pin_memory=True)
            pin.numpy()[...] = U_
            hl.append(pin.numpy())
        # every timeslice's results land in their own pinned buffers: a run's read-back (laph_solver_get_async)
        # overlaps the next step's link upload and solve; the last step waits for its copies
        vout = [torch.empty(3 * L_ ** 3 * nev_, dtype=torch.complex128, pin_memory=True).numpy()
                for L_, nev_, _ in batch]
        eout = [torch.empty(nev_, dtype=torch.float64, pin_memory=True).numpy() for _, nev_, _ in batch]
        pout = [torch.empty(nev_, dtype=torch.float64, pin_memory=True).numpy() for _, nev_, _ in batch]

        def e2e_step():
            for i in range(T):
                solver.set_links(i, hl[i])
            st_, _ = solver.run()
            if st_ != 0:
                raise RuntimeError("solver did not converge in an e2e step")
            for i in range(T):
                solver.get_async(i, eout[i], vout[i], pout[i])

        e2e_step()  # untimed: allocates the read-back staging pool
        solver.wait()
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        solver.wait()
        f1.record(stream)
        barrier()
        e2e_ok = bool(np.array_equal(eout[0], solver.get(0, vectors=False)[0]))
        ems = max_over_ranks(f0.elapsed_time(f1))
        e2e = {"value": world * T * args.steps / (ems / 1000.0), "unit": "timeslices/s",
               "h2d_bytes_per_step": int(sum(L_ ** 3 * 27 * 16 for L_, _, _ in batch)),
               "d2h_bytes_per_step": int(sum(nev_ * 16 + 3 * L_ ** 3 * nev_ * 16 for L_, nev_, _ in batch)),
               "ms_per_step": ems / args.steps, "read_back": "laph_solver_get_async into pinned buffers",
               "last_values_match": e2e_ok}

    # ---- plain GPU form: MatShell MatMult + Krylov-Schur, one timeslice at a time
    plain = None
    if rank == 0 and world == 1 and not args.no_plain:
        ev0, _, _ = solver.get(0, vectors=False)
        plain = plain_gpu(cfg, batch, float(1.1 * (-ev0)[-1]), args.plain_timeslices, local)
        plain["matvec_fp64"] = measure_matvec_fp64(cfg, batch, local)
        plain["chosen_over_plain"] = value / plain["value"] if plain.get("value") else None

    # ---- source shape of the solved eigenvectors (next row of the path) ------
    shape = disp = None
    if rank == 0 and world == 1 and not args.no_shape and all(L_ % 2 == 0 for L_, _, _ in batch):
        shape = measure_sourceshape(solver, stream, batch, args.no_cpu)
        disp = measure_displacement(solver, stream, batch)

    # ---- the gauge reader (host, rank 0, N = 1) --------------------------------
    lime_io = None
    if rank == 0 and world == 1 and not args.no_io:
        try:
            lime_io = measure_lime_io(no_cpu=args.no_cpu)
        except Exception as e:  # a host file-system problem must not cost the headline line
            lime_io = {"error": f"{type(e).__name__}: {e}"}

    # ---- CPU baseline (rank 0, N = 1) ----------------------------------------
    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        ev0, _, _ = solver.get(0, vectors=False)
        lam = -ev0
        lam_c = float(1.1 * lam[-1])
        threads = os.cpu_count() or 1
        dt, info = cpu_reference_step(cfg, batch[0][2], lam_c, 12, threads, batch[0][0], batch[0][1], keep=True)
        Us_orc, V_orc = info.pop("_solution")
        cpu = {"value": 1.0 / dt, "unit": "timeslices/s", "cores": threads, "kind": "port",
               "sample": f"timeslice 0 of the workload: {cfg['smear']} smearing + Krylov-Schur on T_12(B), "
                         f"LAM_L 12, LAM_C {lam_c:.4f} (1.1 x lambda_nev from this run), tol 1e-10",
               "seconds": dt, "detail": info}
        # parity of the timed run's timeslice-0 eigenpairs against that FP64 oracle run (outside every timed region)
        import oracle as orc
        _, V_gpu, _ = solver.get(0)
        parity = orc.compare_eigensystems(Us_orc, batch[0][0], V_gpu, V_orc)
        parity["what"] = ("timeslice 0 of the timed batch (FP32 filter, FP64 Rayleigh-Ritz, tol 1e-9) against the "
                          "oracle's FP64 smearing + Krylov-Schur on T_12(B) (tol 1e-10), both phase-fixed; "
                          "eigenvalues as FP64 Rayleigh quotients on -Delta")
        del V_gpu, V_orc

    timings_last = solver.timings()
    solver.close()
    # ---- learned window A/B and the other benchmark configurations (rank 0, N = 1, untimed for the headline) --
    window_ab = configs = None
    if rank == 0 and world == 1 and not args.no_configs and args.config == "c3":
        torch.cuda.synchronize()
        try:
            lanc = solve_config(cfg, local, reps=1, window="lanczos")
            window_ab = {"workload": "the headline batch, same settings", "mlp": {
                "value": value, "outer_iterations": max(iters), "window_fallbacks": window_fallbacks},
                "lanczos": {k: lanc[k] for k in ("value", "outer_iterations", "ms_per_solve", "status")},
                "gain": value / lanc["value"] if lanc["value"] else None}
        except Exception as e:  # the A/B must not cost the headline line
            window_ab = {"error": f"{type(e).__name__}: {e}"}
        configs = {}
        for name, kw in (("c1", dict(parity={"kind": "dense", "timeslices": range(16)})),
                         ("c2", dict(wave=16, parity={"kind": "ks", "timeslices": [0]})),
                         ("c3_bf16", dict(link_prec="bf16", parity={"kind": "ks", "timeslices": [0]})),
                         ("c4_wave", dict(wave=[8, 12, 16])),
                         ("c5_wave", dict(wave=16))):
            base = CONFIGS[name.split("_")[0]]
            try:
                configs[name] = solve_config(base, local, no_cpu=args.no_cpu, **kw)
            except Exception as e:  # one configuration's failure must not cost the headline line
                configs[name] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.synchronize()
    if rank == 0:
        line = {"metric": "timeslices/s to nev pairs @resid<=1e-9", "value": value, "unit": "timeslices/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32 filter / fp64 RR",
                "data": "synthetic (seeded U = exp(i eps H) gauge field)", "config": workload_config(cfg),
                "roofline": roofline, "cpu_baseline": cpu, "parity": parity, "plain_gpu": plain, "e2e": e2e,
                "gpu_launches": launches,
                "graph_launches_per_solve": loop_info[1], "device_loop": bool(loop_info[0]),
                "clocks": clk, "sourceshape": shape, "displacement": disp, "lime_io": lime_io, "autotune": tune,
                "window_ab": window_ab, "configs": configs,
                "detail": {"outer_iterations": iters, "max_resid": max_resid,
                           "filter_ms_per_step": filt_ms / args.steps,
                           "timings_last_ms": dict(zip(["smear+setup", "filter", "dense+stencil64", "total"],
                                                       timings_last))}}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

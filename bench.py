#!/usr/bin/env python
"""Benchmark: fitted stars/s of the simultaneous PSF fit on the 2048^2 crowded field.

Workload (one "step" = one fit_all_stars_simultaneous call over one field):
  2048 x 2048 Float32 image, 50,000 stars (uniform positions, power-law
  fluxes dN/dF ~ F^-1.5 on [1e1, 1e6]), Moffat beta=3 FWHM 2.8 ePSF tabulated
  101 x 101 at 4x oversampling (single-node GriddedPSFModel{ImagePSF}),
  25 x 25 fit boxes (fit_rad = model_rad = 12), background 50-200 counts,
  Poisson + Gaussian read noise 5, inverse-variance weights, initial guesses
  perturbed by N(0, 0.3 px) and x U(0.9, 1.1) in flux; fixed = (bkg = 0).
  Synthetic, seeded; the reference publishes no dataset for this path.

value: fitted (valid and converged) stars per second with inputs resident in
HBM, device-timed (CUDA events on the library's stream), whole job over all
GPUs.  e2e: the same through the public API with host buffers (host->device
copies and the result readback inside the timed region).  Multi-GPU runs are
independent replicas (one field per GPU, no collective on the data path).

--impl reference times the CPU restatement of the reference algorithm (the
oracle; the Julia reference cannot run on the box) on bounded samples of the
same field across all host cores.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "crowdphot.jl_b200")]

import numpy as np  # noqa: E402

METRIC = "fitted stars/s on 1 B200 (served+mixed vs plain, flux err\u22641e-5); p50/p99 ms"
NY = NX = 2048
N_STARS = 50_000
FIT_RAD = 12
SEED = 1002
SAMPLE = 512  # CPU sample side (same star density)
# DRAM bytes moved per algorithmic byte by the FP64 J v gather (read 816.8 MB + write
# 5.9 MB against 818.3 MB algorithmic: 50,000 live stars x (3 x 625 x 8 + 24) B + two
# 2048^2 FP64 pixel vectors), from an ncu capture of the first launch of the kernel on
# this 2048^2 field (every star live; one metric pass, no replay)
JV_TRAFFIC_RATIO = (816.78 + 5.90) / 818.3


def workload_config(ny=NY, nx=NX, n=N_STARS):
    return {"workload": f"crowded field {ny}x{nx} Float32, {n} stars, Moffat ePSF 101x101 os4, 25x25 boxes",
            "form": "plain (FP64 device arithmetic)", "image": [ny, nx], "n_stars": n, "fit_rad": FIT_RAD,
            "model_rad": FIT_RAD, "psf": "GriddedPSFModel{ImagePSF} single node", "seed": SEED,
            "l2": "intermediate stamp arrays exceed L2 (375-750 MB); a 256 MiB buffer is written between steps"}


def make_field(ny, nx, n, seed):
    from crowdphot_b200.simulate import crowded_field, moffat_epsf
    psf = moffat_epsf()
    img, bkg, iv, truth, init = crowded_field(ny, nx, n, seed=seed, psf=psf, dtype=np.float32)
    return psf, img, bkg, iv, truth, init


def fit_kwargs():
    return dict(fixed={"bkg": 0.0}, model_rad=FIT_RAD)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def max_and_sum_over_ranks(values, device="cpu"):
    """Whole-job aggregates of per-rank values: (max over the ranks, sum over the
    ranks), each a list in the order of `values`.  Times take the max (the job ends
    with its slowest replica), counts the sum.  A single process gets its own values
    back twice."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    mx, sm = t.clone(), t.clone()
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return mx.tolist(), sm.tolist()


def replica_seed(base, rank):
    """The seed of one replica's synthetic input: every rank fits its own field."""
    return base + rank


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        mx = [float(r[2]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip().lower() == "active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU: the oracle on bounded samples (cpu_baseline and the reference arm)
# ---------------------------------------------------------------------------
def _cpu_sample_fit(seed):
    from oracle import orc_fit_simultaneous
    n = int(round(N_STARS * SAMPLE * SAMPLE / (NY * NX)))
    psf, img, bkg, iv, truth, init = make_field(SAMPLE, SAMPLE, n, seed)
    t = time.perf_counter()
    r = orc_fit_simultaneous(img, psf, init, FIT_RAD, inv_var=iv, background=bkg, residual=False, **fit_kwargs())
    dt = time.perf_counter() - t
    return int((r.valid & r.converged).sum()), dt, n


def cpu_baseline_single():
    fitted, dt, n = _cpu_sample_fit(SEED + 1)
    return {"value": fitted / dt, "unit": "stars/s", "cores": 1, "kind": "port",
            "sample": f"{SAMPLE}x{SAMPLE} crop at the same star density ({n} stars), one fit, FP64 oracle, "
                      f"{dt:.1f} s"}


def _full_field_oracle(ny, nx, n, seed):
    """The FP64 oracle on the whole bench field (the C2-size parity check); runs in
    a spawned process while the GPU legs are timed."""
    from oracle import orc_fit_simultaneous
    psf, img, bkg, iv, truth, init = make_field(ny, nx, n, seed)
    t = time.perf_counter()
    r = orc_fit_simultaneous(img, psf, init, FIT_RAD, inv_var=iv, background=bkg, residual=False, **fit_kwargs())
    dt = time.perf_counter() - t
    return dict(y=r.y, x=r.x, flux=r.flux, flux_err=r.flux_err, valid=r.valid, converged=r.converged,
                n_iter=r.n_iter, n_passes=r.n_passes, n_active=r.stats["n_active"], n_union=r.stats["n_union"],
                seconds=dt)


FLUX_GATE, POS_GATE = 1e-5, 1e-4


def deviation(a, b, mask):
    """Per-output deviation of fit a from fit b over `mask`: relative flux, position
    (max of |dy|, |dx|) and flux in units of b's flux error."""
    if not mask.any():
        return None
    dfl = np.abs(a["flux"][mask] / b["flux"][mask] - 1)
    dpos = np.maximum(np.abs(a["y"][mask] - b["y"][mask]), np.abs(a["x"][mask] - b["x"][mask]))
    dsig = np.abs(a["flux"][mask] - b["flux"][mask]) / b["flux_err"][mask]
    q = lambda v: {"median": float(np.median(v)), "p99": float(np.percentile(v, 99)), "max": float(v.max())}
    bad = (dfl > FLUX_GATE) | (dpos > POS_GATE)
    return {"stars": int(mask.sum()), "flux_rel": dict(q(dfl), frac_within_gate=float(np.mean(dfl <= FLUX_GATE))),
            "pos_px": dict(q(dpos), frac_within_gate=float(np.mean(dpos <= POS_GATE))),
            "flux_in_sigma": q(dsig), "violators": int(bad.sum())}


def fitted_mask(*rs):
    m = np.ones_like(rs[0]["valid"], dtype=bool)
    for r in rs:
        m &= r["valid"].astype(bool) & r["converged"].astype(bool)
    return m


def run_reference(args):
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    times = []
    total_fitted = 0
    with ctx.Pool(cores) as pool:
        for step in range(args.warmup + args.steps):
            t = time.perf_counter()
            res = pool.map(_cpu_sample_fit, [SEED + 100 + step * cores + k for k in range(cores)])
            dt = time.perf_counter() - t
            if step >= args.warmup:
                times.append(dt)
                total_fitted += sum(r[0] for r in res)
    total = sum(times)
    value = total_fitted / total
    n = int(round(N_STARS * SAMPLE * SAMPLE / (NY * NX)))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "stars/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload_config(), sample=f"{cores} x {SAMPLE}x{SAMPLE} samples per step"),
            "cpu_baseline": {"value": value, "unit": "stars/s", "cores": cores, "kind": "port",
                             "sample": f"each step: {cores} independent {SAMPLE}x{SAMPLE} fields at the workload's "
                                       f"star density ({n} stars each), one process per core, FP64 oracle "
                                       "(single-threaded restatement of the reference fitter)"},
            "e2e": {"value": value, "unit": "stars/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args):
    import ctypes as C

    import torch
    import torch.distributed as dist

    import crowdphot_b200 as cpb
    from crowdphot_b200 import _abi
    from crowdphot_b200.photometry import SimOutputs, sim_params

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])
        torch.cuda.synchronize()

    ny, nx, n = args.ny, args.nx, args.n_stars
    oracle_job = pool = None
    if world == 1 and not args.quick and not args.no_cpu:
        import multiprocessing as mp
        pool = mp.get_context("spawn").Pool(1)
        oracle_job = pool.apply_async(_full_field_oracle, (ny, nx, n, replica_seed(SEED, rank)))
    psf, img, bkg, iv, truth, init = make_field(ny, nx, n, replica_seed(SEED, rank))
    ctx = cpb.get_context(local)
    hp = ctx.psf_handle(psf)
    # the timed form: the plain FP64 form, or (--quick only, for profiler captures) the mixed form
    P = sim_params(psf, FIT_RAD, {"bkg": 0.0}, inv_var_given=True, model_rad=FIT_RAD,
                   precision=args.precision if args.quick else "fp64")

    # device-resident inputs (column-major images = torch (nx, ny) contiguous)
    t_img = torch.from_numpy(np.ascontiguousarray(img.T)).to(dev)
    t_iv = torch.from_numpy(np.ascontiguousarray(iv.T)).to(dev)
    t_bkg = torch.from_numpy(np.ascontiguousarray(bkg.T)).to(dev)
    t_y = torch.from_numpy(np.asarray(init["y"], np.float64)).to(dev)
    t_x = torch.from_numpy(np.asarray(init["x"], np.float64)).to(dev)
    t_f = torch.from_numpy(np.asarray(init["flux"], np.float64)).to(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2
    R = FIT_RAD
    S2 = (2 * R + 1) ** 2
    outs = SimOutputs(n, ny, nx, S2, residual=False)
    vp = lambda t: C.c_void_p(t.data_ptr())

    def step_resident(Pp=None, o=None):
        Pp = Pp if Pp is not None else P
        o = o if o is not None else outs
        rc = ctx.lib.cpb_fit_simultaneous_device(ctx.handle, hp, C.byref(Pp), vp(t_img), _abi.CPB_F32, ny, nx,
                                                 vp(t_iv), vp(t_bkg), n, vp(t_y), vp(t_x), vp(t_f), C.byref(o.c))
        ctx.raise_for(rc, "cpb_fit_simultaneous_device")
        fitted = int((o.valid[:n].astype(bool) & o.converged[:n].astype(bool)).sum())
        return fitted, float(o.c.device_seconds)

    for _ in range(args.warmup):
        step_resident()
        flush.fill_(1.0)
    ctx.kernel_stats(reset=True)
    barrier()
    clocks = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    fitted_total, dev_times = 0, []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        f, s = step_resident()
        fitted_total += f
        dev_times.append(s)
    barrier()
    clk = clocks.stop() if clocks else None
    _, launches = ctx.kernel_stats(reset=True)
    total_s = float(sum(dev_times))
    def kernel_table(Pf):
        ctx.set_profiling(True)
        flush.fill_(1.0)
        torch.cuda.synchronize()
        _, secs = step_resident(Pf, SimOutputs(n, ny, nx, S2, residual=False))
        ctx.set_profiling(False)
        kst_, _ = ctx.kernel_stats(reset=True)
        return kst_, secs, {k: {"launches": v["launches"], "ms": 1e3 * v["seconds"],
                                "GB_s": v["bytes"] / max(v["seconds"], 1e-12) / 1e9} for k, v in sorted(kst_.items())}

    if args.quick:
        # one more step with per-launch events (not timed above): the kernel table and
        # the render-path kernels' algorithmic bandwidth
        _, _, ktab = kernel_table(P)
        peak = peaks()[0]
        render = {k: dict(v, frac=v["GB_s"] / peak) for k, v in ktab.items()
                  if k in ("k_gather_resid", "k_gather_cost", "k_gather_freeze", "k_eval_model", "k_gather_Jv",
                           "k_JT_lsqr", "k_JT", "k_eval_fill")}
        if rank == 0:
            print(json.dumps({"quick": True, "precision": args.precision, "value": fitted_total / total_s,
                              "unit": "stars/s",
                              "ms_per_step": 1e3 * total_s / args.steps, "gpu_launches": launches,
                              "config": workload_config(ny, nx, n), "kernels": ktab,
                              "roofline_by_kernel": render, "peak_gbs": peak}))
        if world > 1:
            dist.destroy_process_group()
        return
    mx, sm = max_and_sum_over_ranks([total_s, fitted_total, launches], dev)
    total_s, fitted_all, launches_all = mx[0], sm[1], int(sm[2])
    value = fitted_all / total_s

    # the other precision forms, same protocol: the mixed-precision form (FP32
    # stamps, model values and LSQR pixel vectors, FP64 sums and solver) and the
    # same followed by two FP64 refinement iterations
    def take(o):
        return {k: getattr(o, k)[:n].copy() for k in ("y", "x", "flux", "flux_err", "valid", "converged", "n_iter")}

    def timed_form(Pf, steps):
        o = SimOutputs(n, ny, nx, S2, residual=False)
        for _ in range(args.warmup):
            step_resident(Pf, o)
            flush.fill_(1.0)
        barrier()
        fitted, times = 0, []
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            f, s_ = step_resident(Pf, o)
            fitted += f
            times.append(s_)
        barrier()
        mx_, sm_ = max_and_sum_over_ranks([sum(times), fitted], dev)
        ms = [1e3 * t for t in times]
        return o, {"value": sm_[1] / mx_[0], "unit": "stars/s", "ms_per_step": float(np.mean(ms)),
                   "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99))}

    Pm = sim_params(psf, FIT_RAD, {"bkg": 0.0}, inv_var_given=True, model_rad=FIT_RAD, precision="mixed")
    outs_m, mixed = timed_form(Pm, args.steps)
    mixed["kernels"] = kernel_table(Pm)[2]
    Pr = sim_params(psf, FIT_RAD, {"bkg": 0.0}, inv_var_given=True, model_rad=FIT_RAD, precision="mixed",
                    refine_iters=2)
    outs_r, refined = timed_form(Pr, max(1, min(args.steps, 5)))
    # How far the FP64 form itself moves when the input moves by its own rounding:
    # two fits of the image times (1 + 1e-7 N(0, 1)), rounded to the Float32 input
    # (about one ulp on half of the pixels).  Stars that both move by less than a
    # tenth of the gates (1e-6 relative flux, 1e-5 px) form the stable set, on which
    # the other forms are held to the gates.
    ref = take(outs)
    pert = []
    for k in range(2):
        g = np.random.default_rng(SEED + 700 + k)
        ip = (img.astype(np.float64) * (1 + 1e-7 * g.standard_normal(img.shape))).astype(img.dtype)
        t_ip = torch.from_numpy(np.ascontiguousarray(ip.T)).to(dev)
        o = SimOutputs(n, ny, nx, S2, residual=False)
        rc = ctx.lib.cpb_fit_simultaneous_device(ctx.handle, hp, C.byref(P), vp(t_ip), _abi.CPB_F32, ny, nx,
                                                 vp(t_iv), vp(t_bkg), n, vp(t_y), vp(t_x), vp(t_f), C.byref(o.c))
        ctx.raise_for(rc, "cpb_fit_simultaneous_device")
        pert.append(take(o))
        del t_ip
    fit_all = fitted_mask(ref, *pert)
    stable = fit_all.copy()
    for pr in pert:
        dfl = np.abs(pr["flux"] / ref["flux"] - 1)
        dpos = np.maximum(np.abs(pr["y"] - ref["y"]), np.abs(pr["x"] - ref["x"]))
        stable &= (dfl <= 0.1 * FLUX_GATE) & (dpos <= 0.1 * POS_GATE)
    conditioning = {
        "perturbation": "image x (1 + 1e-7 N(0,1)) rounded to Float32, two draws, FP64 form",
        "fitted_in_all": int(fit_all.sum()), "stable_set": int(stable.sum()),
        "fp64_vs_perturbed": deviation(pert[0], ref, fitted_mask(ref, pert[0]))}
    for name, o, blk in (("mixed", outs_m, mixed), ("mixed_refine2", outs_r, refined)):
        r = take(o)
        blk["vs_fp64_all_fitted"] = deviation(r, ref, fitted_mask(ref, r))
        blk["vs_fp64_stable_set"] = deviation(r, ref, stable & fitted_mask(r))
    refined["note"] = ("two FP64 iterations after the mixed fit with every star live again and the damping "
                       "restarted: they continue toward the field's minimum, which the FP64 form at the default "
                       "tolerances stops short of, so this form does not reproduce the FP64 form's output (run to "
                       "the minimum it reaches the oracle's: tests/test_gpu_sim.py)")

    # profiling pass (not timed): per-kernel event timing and algorithmic bytes
    ctx.set_profiling(True)
    flush.fill_(1.0)
    torch.cuda.synchronize()
    f_prof, s_prof = step_resident()
    ctx.set_profiling(False)
    kst, _ = ctx.kernel_stats(reset=True)
    top = max(kst.items(), key=lambda kv: kv[1]["seconds"])
    peak, peak_kind = peaks()
    ach = top[1]["bytes"] / top[1]["seconds"] / 1e9
    roof = {"kernel": top[0], "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_source": peak_kind, "traffic": None,
            "launches": top[1]["launches"], "share_of_step": top[1]["seconds"] / max(s_prof, 1e-12)}
    if top[0] == "k_gather_Jv":
        roof["traffic"] = JV_TRAFFIC_RATIO * top[1]["bytes"] / max(top[1]["launches"], 1)
        roof["traffic_note"] = ("bytes per launch: this run's algorithmic bytes per launch times the DRAM / "
                                f"algorithmic ratio of an ncu capture of one launch of the kernel on this "
                                f"2048^2 field ({JV_TRAFFIC_RATIO:.3f})")
    kernels = {k: {"launches": v["launches"], "ms": 1e3 * v["seconds"],
                   "GB_s": v["bytes"] / max(v["seconds"], 1e-12) / 1e9} for k, v in sorted(kst.items())}

    # end to end through the public API with pinned host buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a.T)).pin_memory().numpy().T
    h_img, h_iv, h_bkg = pin(img), pin(iv), pin(bkg)
    e_times, e_fitted = [], 0
    for i in range(args.warmup + args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        r = cpb.fit_all_stars_simultaneous(h_img, psf, init, FIT_RAD, inv_var=h_iv, background=h_bkg, ctx=ctx,
                                           residual=True, **fit_kwargs())
        ev1.record()
        torch.cuda.synchronize()
        if i >= args.warmup:
            e_times.append(ev0.elapsed_time(ev1) * 1e-3)
            e_fitted += int((r.valid & r.converged).sum())
    mx, sm = max_and_sum_over_ranks([sum(e_times), e_fitted], dev)
    e_value = sm[1] / mx[0]
    h2d = 3 * img.nbytes + 3 * 8 * n
    d2h = n * (12 * 8 + 2 + 4) + ny * nx * 8

    # the comparison the headline metric names: the served stream (C5) through the
    # served mixed form against the plain FP64 form, same requests (one GPU; it runs
    # while the spawned oracle fit is still going)
    served = None
    if world == 1 and not args.no_serve:
        out_s, acc_s, specs_s, _, _ = serve_stream(args.n_requests, args.max_inflight, 1, rank, local,
                                                   sample_clocks=False)
        keep = ("value", "fitted", "makespan_s", "p50_ms", "p99_ms", "slots_used")
        served = {"workload": serve_config(args.n_requests, specs_s)["workload"],
                  "served_mixed": {k: out_s["served_mixed"][k] for k in keep},
                  "plain": {k: out_s["plain"][k] for k in keep},
                  "speedup_vs_plain": out_s["served_mixed"]["value"] / out_s["plain"]["value"],
                  "accuracy": acc_s, "unit": "stars/s",
                  "timer": "host wall clock from the first arrival to the last result"}

    if rank == 0:
        ms = sorted(1e3 * t for t in dev_times)
        line = {"metric": METRIC, "value": value, "unit": "stars/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(workload_config(ny, nx, n), parallelism=f"replicas x{world}"),
                "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
                "fitted_per_step": fitted_all / args.steps / world,
                "model_px_evals_per_s": float(outs.c.model_px_evals) / s_prof,
                "roofline": roof, "kernels": kernels, "gpu_launches": launches_all, "clocks": clk,
                "forms": {"plain_fp64": {"value": value, "ms_per_step": 1e3 * total_s / args.steps},
                          "mixed": mixed, "mixed_refine2": refined, "conditioning": conditioning,
                          "served_stream": served},
                "e2e": {"value": e_value, "unit": "stars/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}}
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline_single()
        if oracle_job is not None:
            orc = oracle_job.get(timeout=1800)
            pool.close()
            both = fitted_mask(ref, orc)
            same = both & (ref["n_iter"] == orc["n_iter"])
            line["parity_full_field"] = {
                "what": "FP64 form vs the FP64 oracle on the whole bench field, same inputs",
                "n_active_equal": int(outs.c.n_active) == int(orc["n_active"]),
                "n_union_equal": int(outs.c.n_union) == int(orc["n_union"]),
                "n_passes": [int(outs.c.n_passes), int(orc["n_passes"])],
                "fitted_in_both": int(both.sum()), "same_freeze_iteration": int(same.sum()),
                "same_freeze": deviation(ref, orc, same),
                "freeze_differs": deviation(ref, orc, both & ~same),
                "stable_set": deviation(ref, orc, both & stable)}
            fitted_cpu = int((orc["valid"] & orc["converged"]).sum())
            line["cpu_baseline"]["full_field"] = {
                "value": fitted_cpu / orc["seconds"], "unit": "stars/s", "cores": 1,
                "sample": f"the whole {ny}x{nx} field ({n} stars), one FP64 oracle fit, {orc['seconds']:.0f} s"}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Batched per-star LM workload (--workload lm-cutouts)
# ---------------------------------------------------------------------------
LM_CUTOUTS = 200_000
LM_SEED = 1004
LM_METRIC = "fitted stars/s on 1 B200, batched fit_star over isolated cutouts"


def lm_config(n):
    return {"workload": f"{n} isolated-star cutouts, side U{{9..41}} (mean 716 px), SNR log-uniform 5-1000, "
                        "Float32 pixels, Moffat ePSF 101x101 os4, fit_star(fixed=(bkg=0), inv_var), LM defaults",
            "n_cutouts": n, "seed": LM_SEED, "psf": "GriddedPSFModel{ImagePSF} single node",
            "l2": "cutout pixels + weights are 1.15 GB (> L2); a 256 MiB buffer is written between steps"}


def _lm_packed(n, seed):
    from crowdphot_b200.simulate import lm_cutouts, moffat_epsf
    return moffat_epsf(), lm_cutouts(n, seed=seed)


def _lm_oracle(psf, d, lo, hi, threads):
    from oracle.ffi import orc_fit_star_packed
    off = d["offsets"][lo:hi]
    end = int(off[-1] + d["ny"][hi - 1] * d["nx"][hi - 1])
    base = int(off[0])
    t = time.perf_counter()
    out, used = orc_fit_star_packed(psf, d["pix"][base:end], off - base, d["ny"][lo:hi], d["nx"][lo:hi],
                                    d["y1"][lo:hi], d["x1"][lo:hi], d["init"][lo:hi], inv_var=d["inv_var"][base:end],
                                    fixed={"bkg": 0.0}, threads=threads)
    dt = time.perf_counter() - t
    return int(((out["status"] == 0) & (out["converged"] != 0)).sum()), dt, used


def run_reference_lm(args):
    psf, d = _lm_packed(args.n_cutouts, LM_SEED)
    n = len(d["ny"])
    times, fitted, used = [], 0, 1
    for step in range(args.warmup + args.steps):
        f, dt, used = _lm_oracle(psf, d, 0, n, 0)
        if step >= args.warmup:
            times.append(dt)
            fitted += f
    value = fitted / sum(times)
    print(json.dumps({"impl": "reference", "metric": LM_METRIC, "value": value, "unit": "stars/s",
                      "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": lm_config(n),
                      "cpu_baseline": {"value": value, "unit": "stars/s", "cores": used, "kind": "port",
                                       "sample": f"all {n} cutouts per step, FP64 oracle fit_star, {used} threads"},
                      "e2e": {"value": value, "unit": "stars/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_gpu_lm(args):
    import torch

    import crowdphot_b200 as cpb
    from crowdphot_b200 import _abi
    from crowdphot_b200.photometry import _lm_outputs, _lm_result_struct, lm_params

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    psf, d = _lm_packed(args.n_cutouts, replica_seed(LM_SEED, rank))
    n = len(d["ny"])
    ctx = cpb.get_context(local)
    hp = ctx.psf_handle(psf)
    fixed = {"bkg": 0.0}
    P = lm_params(psf, fixed)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    dpix, div, doff = t(d["pix"]), t(d["inv_var"]), t(d["offsets"])
    dny, dnx, dy1, dx1, dinit = t(d["ny"]), t(d["nx"]), t(d["y1"]), t(d["x1"]), t(d["init"])
    outs = {k: torch.from_numpy(v).to(dev) for k, v in _lm_outputs(n, 4, 3).items()}
    r = _lm_result_struct(outs, lambda a: a.data_ptr())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    vp = lambda a: a.data_ptr()

    def step():
        rc = ctx.lib.cpb_fit_lm_batch_device(ctx.handle, hp, P, n, vp(doff), vp(dny), vp(dnx), vp(dy1), vp(dx1),
                                             vp(dpix), _abi.CPB_F32, vp(div), vp(dinit), d["pix"].size, r)
        ctx.raise_for(rc, "cpb_fit_lm_batch_device")
        return float(r.device_seconds)

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
        flush.fill_(1.0)
    ctx.kernel_stats(reset=True)
    barrier()
    clocks = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    times, fitted = [], 0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        times.append(step())
        fitted += int(((outs["status"] == 0) & (outs["converged"] != 0)).sum().item())
    barrier()
    clk = clocks.stop() if clocks else None
    _, launches = ctx.kernel_stats(reset=True)
    if args.quick:
        if rank == 0:
            print(json.dumps({"quick": True, "value": fitted / sum(times), "unit": "stars/s",
                              "ms_per_step": 1e3 * sum(times) / args.steps, "gpu_launches": launches,
                              "config": lm_config(n)}))
        if world > 1:
            dist.destroy_process_group()
        return
    mx, sm = max_and_sum_over_ranks([sum(times), fitted, launches], dev)
    total_s, fitted_all, launches_all = mx[0], sm[1], int(sm[2])
    value = fitted_all / total_s
    iters = outs["iterations"].cpu().numpy()

    ctx.set_profiling(True)
    flush.fill_(1.0)
    torch.cuda.synchronize()
    s_prof = step()
    ctx.set_profiling(False)
    kst, _ = ctx.kernel_stats(reset=True)
    k = kst["k_lm"]
    peak, peak_kind = peaks()
    ach = k["bytes"] / k["seconds"] / 1e9
    px_evals = float(np.sum((iters + 1).astype(np.int64) * (d["ny"].astype(np.int64) * d["nx"])))
    roof = {"kernel": "k_lm", "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_source": peak_kind, "traffic": None, "launches": k["launches"],
            "share_of_step": k["seconds"] / max(s_prof, 1e-12),
            "note": "k_lm re-reads each cutout from L1/L2 once per LM iteration; its DRAM floor is one read of "
                    "pixels+weights, so this fraction shows how far the FP64 evaluation is from that floor"}

    # end to end: host buffers through the public packed API
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    hpix, hiv = pin(d["pix"]), pin(d["inv_var"])
    e_times, e_fitted = [], 0
    for i in range(args.warmup + args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = cpb.fit_star_packed(psf, hpix, d["offsets"], d["ny"], d["nx"], d["y1"], d["x1"], d["init"],
                                  inv_var=hiv, fixed=fixed, ctx=ctx)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e_times.append(dt)
            e_fitted += int(((out["status"] == 0) & (out["converged"] != 0)).sum())
    mx, sm = max_and_sum_over_ranks([sum(e_times), e_fitted], dev)
    e_value = sm[1] / mx[0]
    h2d = 2 * d["pix"].nbytes + n * (8 + 16 + 32)
    d2h = n * (8 * 4 + 8 * 9 + 8 * 4 + 4 + 8)
    if rank == 0:
        ms = sorted(1e3 * x for x in times)
        line = {"metric": LM_METRIC, "value": value, "unit": "stars/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(lm_config(n), parallelism=f"replicas x{world}"),
                "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
                "fitted_per_step": fitted_all / args.steps / world, "mean_iterations": float(iters.mean()),
                "model_px_evals_per_s": px_evals / s_prof, "roofline": roof, "gpu_launches": launches_all,
                "clocks": clk,
                "e2e": {"value": e_value, "unit": "stars/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "timer": "host wall clock around the public call (it synchronises before returning)"}}
        if world == 1 and not args.no_cpu:
            m = min(n, 100_000)
            f, dt, used = _lm_oracle(psf, d, 0, m, 0)
            line["cpu_baseline"] = {"value": f / dt, "unit": "stars/s", "cores": used, "kind": "port",
                                    "sample": f"first {m} cutouts of the workload, FP64 oracle fit_star on {used} "
                                              f"host threads, {dt:.2f} s"}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Mixed batch (--workload c4): 200,000 fit_star cutouts + 20,000 blended groups
# in one captured CUDA graph whose two persistent kernels run concurrently
# ---------------------------------------------------------------------------
C4_GROUPS = 20_000
C4_GROUP_SEED = 1104
C4_METRIC = "fitted stars/s on 1 B200, one CUDA-graph launch of fit_star cutouts + simultaneous group fits"
C4_GKW = dict(fixed={"bkg": 0.0}, model_rad=12)


def c4_config(n_cut, n_grp, n_grp_stars):
    return {"workload": f"{n_cut} isolated fit_star cutouts (side U{{9..41}}, SNR 5-1000) + {n_grp} blended groups "
                        f"of 2-12 stars ({n_grp_stars} stars, (8k+17)^2 cutouts, fit_rad 5, model_rad 12), Float32 "
                        "pixels, Moffat ePSF 101x101 os4, one CUDA-graph launch with tuned launch shapes",
            "n_cutouts": n_cut, "n_groups": n_grp, "n_group_stars": n_grp_stars, "seeds": [LM_SEED, C4_GROUP_SEED],
            "psf": "GriddedPSFModel{ImagePSF} single node",
            "l2": "inputs are 1.25 GB (> L2); a 256 MiB buffer is written between steps"}


def _group_oracle_chunk(items):
    from crowdphot_b200.simulate import moffat_epsf
    from oracle import orc_fit_simultaneous
    psf = moffat_epsf()
    fitted, t = 0, 0.0
    for img, iv, cat in items:
        t0 = time.perf_counter()
        r = orc_fit_simultaneous(img, psf, cat, 5, inv_var=iv, residual=False, **C4_GKW)
        t += time.perf_counter() - t0
        fitted += int((r.valid & r.converged).sum())
    return fitted, t


def c4_cpu(n_cut, n_grp, cores, lm_sample, grp_sample, dg=None):
    """The oracle on a bounded sample of both halves: the first `lm_sample`
    cutouts over the oracle's host threads, the first `grp_sample` groups over
    `cores` processes.  Returns (stars/s of the whole mix at the measured
    rates, description)."""
    import multiprocessing as mp
    from crowdphot_b200.simulate import lm_groups
    psf, d = _lm_packed(n_cut, LM_SEED)
    m = min(n_cut, lm_sample)
    f_lm, t_lm, used = _lm_oracle(psf, d, 0, m, cores)
    dg = dg if dg is not None else lm_groups(n_grp, seed=C4_GROUP_SEED, psf=psf)
    k = min(n_grp, grp_sample)
    items = []
    for g in range(k):
        off, ny, nx = int(dg["offsets"][g]), int(dg["ny"][g]), int(dg["nx"][g])
        s0, s1 = int(dg["star_offsets"][g]), int(dg["star_offsets"][g + 1])
        items.append((dg["pix"][off:off + ny * nx].reshape((ny, nx), order="F"),
                      dg["inv_var"][off:off + ny * nx].reshape((ny, nx), order="F"),
                      dict(y=dg["y"][s0:s1], x=dg["x"][s0:s1], flux=dg["flux"][s0:s1])))
    chunks = [items[k * i // cores:k * (i + 1) // cores] for i in range(cores)]
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_group_oracle_chunk, [c for c in chunks if c])
    t_g = max(r[1] for r in res)  # the processes fit in parallel; their start-up is not counted
    f_g = sum(r[0] for r in res)
    # whole mix at the measured rates: time = lm time scaled + group time scaled
    total_time = t_lm * (n_cut / m) + t_g * (n_grp / k)
    total_fitted = f_lm * (n_cut / m) + f_g * (n_grp / k)
    desc = (f"first {m} cutouts on {used} threads ({t_lm:.2f} s) + first {k} groups over {cores} processes "
            f"({t_g:.2f} s, slowest process), FP64 oracle, rates scaled to the whole mix")
    return total_fitted / total_time, desc


def run_reference_c4(args):
    cores = os.cpu_count() or 1
    from crowdphot_b200.simulate import lm_groups, moffat_epsf
    dg = lm_groups(args.n_groups, seed=C4_GROUP_SEED, psf=moffat_epsf())
    times, vals = [], []
    desc = ""
    for step in range(args.warmup + args.steps):
        t = time.perf_counter()
        v, desc = c4_cpu(args.n_cutouts, args.n_groups, cores, 40_000, 40 * cores, dg=dg)
        if step >= args.warmup:
            times.append(time.perf_counter() - t)
            vals.append(v)
    value = float(np.mean(vals))
    print(json.dumps({"impl": "reference", "metric": C4_METRIC, "value": value, "unit": "stars/s",
                      "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                      "config": c4_config(args.n_cutouts, args.n_groups, None),
                      "cpu_baseline": {"value": value, "unit": "stars/s", "cores": cores, "kind": "port",
                                       "sample": desc},
                      "e2e": {"value": value, "unit": "stars/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_gpu_c4(args):
    import tempfile as _tf

    import torch

    import crowdphot_b200 as cpb
    from crowdphot_b200.photometry import _lm_outputs, group_outputs
    from crowdphot_b200.simulate import lm_groups

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    psf, dl = _lm_packed(args.n_cutouts, replica_seed(LM_SEED, rank))
    dg = lm_groups(args.n_groups, seed=replica_seed(C4_GROUP_SEED, rank), psf=psf)
    n_cut, n_grp = len(dl["ny"]), len(dg["ny"])
    ns = int(dg["star_offsets"][-1])
    ctx = cpb.get_context(local)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    lm = {k: t(dl[k]) for k in ("offsets", "ny", "nx", "y1", "x1", "pix", "inv_var", "init")}
    lm["out"] = {k: torch.from_numpy(v).to(dev) for k, v in _lm_outputs(n_cut, 4, 3).items()}
    gr = {k: t(dg[k]) for k in ("offsets", "ny", "nx", "pix", "inv_var", "star_offsets")}
    gr.update(y=t(dg["y"]), x=t(dg["x"]), flux=t(dg["flux"]))
    gr["out"] = {k: torch.from_numpy(v).to(dev) for k, v in group_outputs(ns, n_grp).items()}
    cache = os.path.join(_tf.gettempdir(), f"cpb_tune_{os.getuid()}.txt")
    graph = cpb.BatchGraph(psf, lm=lm, lm_fixed={"bkg": 0.0}, groups=gr, fit_rad=5, group_kw=C4_GKW,
                           autotune=0 if args.quick else 1, cache_path=cache, ctx=ctx)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def fitted_now():
        a = int(((lm["out"]["status"] == 0) & (lm["out"]["converged"] != 0)).sum().item())
        b = int(((gr["out"]["valid"][:ns] != 0) & (gr["out"]["converged"][:ns] != 0)).sum().item())
        return a, b

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        graph.launch()
        flush.fill_(1.0)
    ctx.kernel_stats(reset=True)
    barrier()
    clocks = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    times, f_lm, f_g = [], 0, 0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        times.append(graph.launch())
        a, b = fitted_now()
        f_lm += a
        f_g += b
    barrier()
    clk = clocks.stop() if clocks else None
    _, launches = ctx.kernel_stats(reset=True)
    if args.quick:
        if rank == 0:
            print(json.dumps({"quick": True, "value": (f_lm + f_g) / sum(times), "unit": "stars/s",
                              "ms_per_step": 1e3 * sum(times) / args.steps, "gpu_launches": launches,
                              "config": c4_config(n_cut, n_grp, ns)}))
        graph.close()
        if world > 1:
            dist.destroy_process_group()
        return
    mx, sm = max_and_sum_over_ranks([sum(times), f_lm + f_g, launches], dev)
    total_s, fitted_all, launches_all = mx[0], sm[1], int(sm[2])
    value = fitted_all / total_s
    info = graph.tune_info()
    # profiling pass (not timed): each kernel alone through the direct device entries
    from crowdphot_b200 import _abi
    from crowdphot_b200.photometry import _lm_result_struct, group_result_struct, lm_params, sim_params
    ctx.set_profiling(True)
    P = lm_params(psf, {"bkg": 0.0})
    r = _lm_result_struct(lm["out"], lambda a: a.data_ptr())
    vp = lambda a: a.data_ptr()
    flush.fill_(1.0)
    torch.cuda.synchronize()
    rc = ctx.lib.cpb_fit_lm_batch_device(ctx.handle, ctx.psf_handle(psf), P, n_cut, vp(lm["offsets"]), vp(lm["ny"]),
                                         vp(lm["nx"]), vp(lm["y1"]), vp(lm["x1"]), vp(lm["pix"]), _abi.CPB_F32,
                                         vp(lm["inv_var"]), vp(lm["init"]), dl["pix"].size, r)
    ctx.raise_for(rc, "cpb_fit_lm_batch_device")
    SP = sim_params(psf, 5, {"bkg": 0.0}, inv_var_given=True, model_rad=12)
    gres = group_result_struct(gr["out"], lambda a: a.data_ptr())
    flush.fill_(1.0)
    torch.cuda.synchronize()
    rc = ctx.lib.cpb_fit_simultaneous_batch_device(ctx.handle, ctx.psf_handle(psf), C_byref(SP), n_grp,
                                                   vp(gr["offsets"]), vp(gr["ny"]), vp(gr["nx"]), vp(gr["pix"]),
                                                   _abi.CPB_F32, vp(gr["inv_var"]), None, vp(gr["star_offsets"]),
                                                   vp(gr["y"]), vp(gr["x"]), vp(gr["flux"]), dg["pix"].size,
                                                   C_byref(gres))
    ctx.raise_for(rc, "cpb_fit_simultaneous_batch_device")
    ctx.set_profiling(False)
    kst, _ = ctx.kernel_stats(reset=True)
    peak, peak_kind = peaks()
    kernels = {k: {"launches": v["launches"], "ms": 1e3 * v["seconds"], "GB_s": v["bytes"] / max(v["seconds"], 1e-12) / 1e9}
               for k, v in kst.items()}
    top = max(kst.items(), key=lambda kv: kv[1]["seconds"])
    ach = top[1]["bytes"] / top[1]["seconds"] / 1e9
    roof = {"kernel": top[0], "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "peak_source": peak_kind, "traffic": None, "launches": top[1]["launches"],
            "note": "both kernels are FP64-arithmetic bound: each input pixel is read from DRAM once and re-read from "
                    "L1 / shared memory once per iteration; the fraction shows the distance from the one-read floor"}
    # end to end: pinned host inputs -> bound device buffers, one graph launch, results back
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    h_in = {("lm", k): pin(dl[k]) for k in ("pix", "inv_var", "init")}
    h_in.update({("gr", k): pin(dg[k]) for k in ("pix", "inv_var")})
    h_in.update({("gr", "y"): pin(dg["y"]), ("gr", "x"): pin(dg["x"]), ("gr", "flux"): pin(dg["flux"])})
    outs = [lm["out"][k] for k in ("params", "cov", "cost", "converged", "iterations", "status")] + \
           [gr["out"][k] for k in ("y", "x", "flux", "y_err", "x_err", "flux_err", "converged", "valid", "n_iter",
                                   "n_passes", "status")]
    h_out = [torch.empty(o.shape, dtype=o.dtype).pin_memory() for o in outs]
    e_times, e_fitted = [], 0
    for i in range(args.warmup + args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for (half, k), h in h_in.items():
            (lm if half == "lm" else gr)[k].copy_(h, non_blocking=True)
        torch.cuda.synchronize()
        graph.launch()
        for h, o in zip(h_out, outs):
            h.copy_(o, non_blocking=True)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e_times.append(dt)
            st_lm, cv_lm = h_out[5].numpy(), h_out[3].numpy()
            e_fitted += int(((st_lm == 0) & (cv_lm != 0)).sum() + ((h_out[13].numpy()[:ns] != 0) &
                                                                   (h_out[12].numpy()[:ns] != 0)).sum())
    h2d = sum(h.numel() * h.element_size() for h in h_in.values())
    d2h = sum(h.numel() * h.element_size() for h in h_out)
    mx, sm = max_and_sum_over_ranks([sum(e_times), e_fitted], dev)
    e_value = sm[1] / mx[0]
    graph.close()
    if rank == 0:
        ms = sorted(1e3 * x for x in times)
        line = {"metric": C4_METRIC, "value": value, "unit": "stars/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(c4_config(n_cut, n_grp, ns), parallelism=f"replicas x{world}"),
                "p50_ms": float(np.percentile(ms, 50)), "p99_ms": float(np.percentile(ms, 99)),
                "fitted_per_step": {"cutouts": f_lm / args.steps, "group_stars": f_g / args.steps},
                "tuning": info, "roofline": roof, "kernels": kernels, "gpu_launches": launches_all, "clocks": clk,
                "e2e": {"value": e_value, "unit": "stars/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "timer": "host wall clock: pinned H2D of every input, one graph launch, D2H of the results"}}
        if world == 1 and not args.no_cpu:
            cores = os.cpu_count() or 1
            v, desc = c4_cpu(n_cut, n_grp, cores, 50_000, 40 * cores, dg=dg)
            line["cpu_baseline"] = {"value": v, "unit": "stars/s", "cores": cores, "kind": "port", "sample": desc}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Served request stream (--workload serve): Poisson arrivals of fields of
# mixed sizes into the continuous-batching server
# ---------------------------------------------------------------------------
SERVE_SIDES = (256, 512, 1024, 2048, 4096)
SERVE_RATE = 200.0
SERVE_METRIC = "fitted stars/s on 1 B200, served request stream (continuous batching, mixed precision); p50/p99 ms"


def serve_requests(n, seed=5000):
    """Arrival times (Poisson, mean SERVE_RATE / s) and per-request (side, density, seed)."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / SERVE_RATE, n))
    out = []
    for i in range(n):
        r = np.random.default_rng(seed + i)
        out.append((int(r.choice(SERVE_SIDES)), float(r.uniform(0.002, 0.02)), seed + i))
    return arrivals - arrivals[0], out


def serve_config(n, specs):
    stars = sum(int(round(d * s * s)) for s, d, _ in specs)
    return {"workload": f"{n} requests, Poisson arrivals at {SERVE_RATE:.0f}/s, sides uniform in {list(SERVE_SIDES)}, "
                        f"density U[0.002, 0.02] px^-2 ({stars} stars in all), crowded-field PSF / noise model, "
                        "fit_rad = model_rad = 12",
            "n_requests": n, "seeds": "5000 + i", "sides": [s for s, _, _ in specs], "n_stars_total": stars,
            "l2": "fields up to 4096^2 (stamp arrays up to 4 GB) exceed L2; requests run back to back"}


def _run_stream(sv, psf, reqs, arrivals, precision):
    """Submits the requests at their arrival times; returns (results, infos, makespan)."""
    handles = []
    t0 = time.perf_counter()
    for (img, bkg, iv, init), at in zip(reqs, arrivals):
        dt = t0 + at - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        handles.append(sv.submit(img, psf, init, FIT_RAD, inv_var=iv, background=bkg, precision=precision,
                                 **fit_kwargs()))
    results = [h.result(timeout=3600) for h in handles]
    infos = [h.poll() for h in handles]
    makespan = time.perf_counter() - t0
    return results, infos, makespan


def serve_stream(n_requests, max_inflight, warmup, rank, local, sample_clocks=True):
    """The served stream (C5) run twice on one GPU: the plain FP64 form one request
    at a time and the served mixed form with `max_inflight` slots.  Returns the
    per-form summaries (with the results), the accuracy of the served form against
    the plain one, the request specs and inputs, and the clock record."""
    import torch

    import crowdphot_b200 as cpb
    from crowdphot_b200.simulate import moffat_epsf, served_field

    psf = moffat_epsf()
    arrivals, specs = serve_requests(n_requests, 5000 + 1000 * rank)
    reqs = []
    for side, dens, sd in specs:
        img, bkg, iv, truth, init = served_field(side, dens, seed=sd, psf=psf)
        reqs.append((img, bkg, iv, init))
    # warm-up: one small request per form (contexts, PSF upload, kernels loaded)
    warm = reqs[int(np.argmin([s for s, _, _ in specs]))]
    clocks, clk = None, None
    out = {}
    for form, slots, prec in (("plain", 1, "fp64"), ("served_mixed", max_inflight, "mixed")):
        with cpb.Server(device=local, max_inflight=slots) as sv:
            for _ in range(max(warmup, 1)):
                sv.submit(warm[0], psf, warm[3], FIT_RAD, inv_var=warm[2], background=warm[1], precision=prec,
                          **fit_kwargs()).result(timeout=600)
            if form == "served_mixed" and rank == 0 and sample_clocks:
                clocks = ClockSampler(torch.cuda.current_device())
            res, infos, makespan = _run_stream(sv, psf, reqs, arrivals, prec)
            if form == "served_mixed" and clocks is not None:
                clk = clocks.stop()
        fitted = sum(int((r.valid & r.converged).sum()) for r in res)
        lat = np.array([i["latency_seconds"] for i in infos]) * 1e3
        out[form] = dict(results=res, value=fitted / makespan, fitted=fitted, makespan_s=makespan,
                         p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                         device_seconds=float(sum(i["device_seconds"] for i in infos)),
                         slots_used=len({i["slot"] for i in infos}))
    # accuracy of the served mixed form against the plain FP64 form, per output
    dfl, dpos = [], []
    for a, b in zip(out["served_mixed"]["results"], out["plain"]["results"]):
        ok = a.valid & a.converged & b.valid & b.converged & (a.n_iter == b.n_iter)
        dfl.append(np.abs(a.flux[ok] / b.flux[ok] - 1))
        dpos.append(np.maximum(np.abs(a.y[ok] - b.y[ok]), np.abs(a.x[ok] - b.x[ok])))
    dfl, dpos = np.concatenate(dfl), np.concatenate(dpos)
    acc = {"compared_stars": int(dfl.size),
           "flux_rel_dev_vs_fp64": {"median": float(np.median(dfl)), "p99": float(np.percentile(dfl, 99)),
                                    "frac_within_1e-5": float(np.mean(dfl <= 1e-5))},
           "pos_dev_px_vs_fp64": {"median": float(np.median(dpos)), "p99": float(np.percentile(dpos, 99)),
                                  "frac_within_1e-4": float(np.mean(dpos <= 1e-4))}}
    return out, acc, specs, reqs, clk


def run_gpu_serve(args):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    out, acc, specs, reqs, clk = serve_stream(args.n_requests, args.max_inflight, args.warmup, rank, local)
    sm, pl = out["served_mixed"], out["plain"]
    h2d = sum(r[0].nbytes * 3 + 24 * r[3]["y"].size for r in reqs)
    d2h = sum(r[3]["y"].size * (12 * 8 + 2 + 4) for r in reqs)
    if rank == 0:
        line = {"metric": SERVE_METRIC, "value": sm["value"], "unit": "stars/s", "n_gpus": 1,
                "steps": args.n_requests, "warmup": max(args.warmup, 1),
                "ms_per_step": 1e3 * sm["makespan_s"] / args.n_requests, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 mixed", "data": "synthetic",
                "config": dict(serve_config(args.n_requests, specs), max_inflight=args.max_inflight),
                "p50_ms": sm["p50_ms"], "p99_ms": sm["p99_ms"],
                "forms": {k: {kk: vv for kk, vv in v.items() if kk != "results"} for k, v in out.items()},
                "speedup_vs_plain": sm["value"] / pl["value"], "accuracy": acc, "clocks": clk,
                "gpu_launches": None,
                "e2e": {"value": sm["value"], "unit": "stars/s", "h2d_bytes_per_step": h2d // args.n_requests,
                        "d2h_bytes_per_step": d2h // args.n_requests,
                        "timer": "host wall clock from the first arrival to the last result: every request is "
                                 "submitted with host buffers and its results read back"},
                "note": "a step is one request; value is the served stream's fitted stars over its makespan"}
        print(json.dumps(line))


# ---------------------------------------------------------------------------
# Sequential multi-pass photometry (--workload multipass): fit_all_stars
# ---------------------------------------------------------------------------
MP_PASSES = 3
MP_METRIC = "fitted stars/s on 1 B200, fit_all_stars (3 brightness-ordered passes of fit_star)"


def mp_config(ny, nx, n):
    return {"workload": f"fit_all_stars on the crowded field {ny}x{nx} Float32, {n} stars, Moffat ePSF 101x101 "
                        f"os4, fit_rad {FIT_RAD} (25x25 boxes), {MP_PASSES} passes, fixed=(bkg=0), inv_var",
            "image": [ny, nx], "n_stars": n, "fit_rad": FIT_RAD, "n_passes": MP_PASSES, "seed": SEED,
            "psf": "GriddedPSFModel{ImagePSF} single node",
            "l2": "the image, weights and residual (50 MB) stay L2-resident; each pass is a chain of dependent "
                  "batches, so no flush is applied between the batches of one call; 256 MiB written between calls"}


def _mp_field(ny, nx, n, seed):
    psf, img, bkg, iv, truth, init = make_field(ny, nx, n, seed)
    return psf, (img - bkg).astype(np.float32), iv, init


def _mp_cpu(seed):
    from oracle import orc_fit_all_stars
    n = int(round(N_STARS * SAMPLE * SAMPLE / (NY * NX)))
    psf, data, iv, init = _mp_field(SAMPLE, SAMPLE, n, seed)
    t = time.perf_counter()
    r = orc_fit_all_stars(data, psf, init, FIT_RAD, n_passes=MP_PASSES, fixed={"bkg": 0.0}, inv_var=iv,
                          residual=False)
    dt = time.perf_counter() - t
    return int((r.valid & r.converged).sum()), dt, n


def run_reference_mp(args):
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    times, fitted = [], 0
    with mp.get_context("spawn").Pool(cores) as pool:
        for step in range(args.warmup + args.steps):
            t = time.perf_counter()
            res = pool.map(_mp_cpu, [SEED + 300 + step * cores + k for k in range(cores)])
            dt = time.perf_counter() - t
            if step >= args.warmup:
                times.append(dt)
                fitted += sum(r[0] for r in res)
    value = fitted / sum(times)
    n = int(round(N_STARS * SAMPLE * SAMPLE / (NY * NX)))
    print(json.dumps({"impl": "reference", "metric": MP_METRIC, "value": value, "unit": "stars/s",
                      "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                      "config": dict(mp_config(NY, NX, N_STARS), sample=f"{cores} x {SAMPLE}x{SAMPLE} per step"),
                      "cpu_baseline": {"value": value, "unit": "stars/s", "cores": cores, "kind": "port",
                                       "sample": f"each step: {cores} independent {SAMPLE}x{SAMPLE} fields at the "
                                                 f"workload's star density ({n} stars each), one process per core, "
                                                 "FP64 oracle fit_all_stars (one star at a time)"},
                      "e2e": {"value": value, "unit": "stars/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_gpu_mp(args):
    import ctypes as C

    import torch

    import crowdphot_b200 as cpb
    from crowdphot_b200.photometry import MultipassOutputs, lm_params, params_matrix, spread_fwhm_arg

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ny, nx, n = args.ny, args.nx, args.n_stars
    psf, data, iv, init = _mp_field(ny, nx, n, replica_seed(SEED, rank))
    ctx = cpb.get_context(local)
    hp = ctx.psf_handle(psf)
    P = lm_params(psf, {"bkg": 0.0})
    pinit = params_matrix(psf, init)
    outs = MultipassOutputs(n, pinit.shape[1], ny, nx, residual=False)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a.T)).pin_memory().numpy().T
    h_data, h_iv = pin(data), pin(iv)

    def step():
        rc = ctx.lib.cpb_fit_all_stars(ctx.handle, hp, C.byref(P), float(FIT_RAD), MP_PASSES,
                                       spread_fwhm_arg(None), h_data.ctypes.data_as(C.c_void_p), 1, ny, nx,
                                       h_iv.ctypes.data_as(C.c_void_p), n,
                                       pinit.ctypes.data_as(C.POINTER(C.c_double)), C.byref(outs.c))
        ctx.raise_for(rc, "cpb_fit_all_stars")
        return int((outs.valid[:n].astype(bool) & outs.converged[:n].astype(bool)).sum()), float(outs.c.device_seconds)

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
        flush.fill_(1.0)
    ctx.kernel_stats(reset=True)
    barrier()
    clocks = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    times, walls, fitted = [], [], 0
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f, s = step()
        walls.append(time.perf_counter() - t0)
        times.append(s)
        fitted += f
    barrier()
    clk = clocks.stop() if clocks else None
    _, launches = ctx.kernel_stats(reset=True)
    mx, sm = max_and_sum_over_ranks([sum(times), fitted, launches, sum(walls)], dev)
    total_s, fitted_all, launches_all, wall_s = mx[0], sm[1], int(sm[2]), mx[3]
    value = fitted_all / total_s
    e_value = fitted_all / wall_s
    ctx.set_profiling(True)
    flush.fill_(1.0)
    torch.cuda.synchronize()
    _, s_prof = step()
    ctx.set_profiling(False)
    kst, _ = ctx.kernel_stats(reset=True)
    kernels = {k: {"launches": v["launches"], "ms": 1e3 * v["seconds"],
                   "GB_s": v["bytes"] / max(v["seconds"], 1e-12) / 1e9} for k, v in sorted(kst.items())}
    roof = None
    if kst:
        top = max(kst.items(), key=lambda kv: kv[1]["seconds"])
        peak, peak_kind = peaks()
        ach = top[1]["bytes"] / top[1]["seconds"] / 1e9
        roof = {"kernel": top[0], "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "peak_source": peak_kind, "traffic": None, "launches": top[1]["launches"],
                "share_of_step": top[1]["seconds"] / max(s_prof, 1e-12),
                "note": "each batch's fit_star launch reads its cutouts once; the kernels are FP64-pipe and "
                        "launch bound, the share of the step they cover shows the host batching overhead"}
    h2d = 2 * data.nbytes + pinit.nbytes
    d2h = n * (2 * pinit.shape[1] * 8 + 2 + 7 * 8 + 4)
    if rank == 0:
        line = {"metric": MP_METRIC, "value": value, "unit": "stars/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(mp_config(ny, nx, n), parallelism=f"replicas x{world}"),
                "fitted_per_step": fitted_all / args.steps / world, "n_batches_per_call": int(outs.c.n_levels),
                "fits_per_call": int(outs.c.n_fits), "roofline": roof, "kernels": kernels,
                "gpu_launches": launches_all, "clocks": clk,
                "e2e": {"value": e_value, "unit": "stars/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "timer": "host wall clock around cpb_fit_all_stars with pinned host buffers (the call "
                                 "uploads the image and weights and returns every result on the host)"},
                "value_timer": "CUDA events on the library stream from the first device step after the upload "
                               "to the last result (host batching inside)"}
        if world == 1 and not args.no_cpu:
            f, dt, m = _mp_cpu(SEED + 1)
            line["cpu_baseline"] = {"value": f / dt, "unit": "stars/s", "cores": 1, "kind": "port",
                                    "sample": f"{SAMPLE}x{SAMPLE} crop at the same star density ({m} stars), FP64 "
                                              f"oracle fit_all_stars, one core, {dt:.1f} s"}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# The plain CPU-runnable configuration (--workload c1): 256^2 Float64, 200 stars,
# CircularGaussianPSF FWHM 2.5, 15 x 15 boxes, 20 iterations, linear_tol 1e-8
# ---------------------------------------------------------------------------
C1_METRIC = "fitted stars/s on 1 B200, simultaneous fit of the 256^2 Gaussian field"
C1_SEED = 1001


def c1_config():
    return {"workload": "256x256 Float64, 200 stars, CircularGaussianPSF FWHM 2.5, 15x15 boxes, max_iter 20, "
                        "linear_tol 1e-8", "image": [256, 256], "n_stars": 200, "fit_rad": 7, "model_rad": 7,
            "seed": C1_SEED, "l2": "the whole problem is L2-resident; launch and latency bound"}


def _c1_kwargs(iv, bkg):
    return dict(fixed={"fwhm": 2.5, "bkg": 0.0}, inv_var=iv, background=bkg, model_rad=7, max_iter=20,
                linear_tol=1e-8)


def _c1_cpu(seconds=10.0):
    """The FP64 oracle on the C1 field, repeated for about `seconds` (one core)."""
    from crowdphot_b200.simulate import c1_field
    from oracle import orc_fit_simultaneous
    img, bkg, iv, psf, src, init = c1_field(C1_SEED)
    fits, fitted, t0 = 0, 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds or fits == 0:
        r = orc_fit_simultaneous(img, psf, init, 7, residual=False, **_c1_kwargs(iv, bkg))
        fits += 1
        fitted += int((r.valid & r.converged).sum())
    dt = time.perf_counter() - t0
    return fitted / dt, fits, dt


def run_reference_c1(args):
    rate, fits, dt = _c1_cpu(max(5.0, 0.5 * (args.steps + args.warmup)))
    line = {"impl": "reference", "metric": C1_METRIC, "value": rate, "unit": "stars/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / fits, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": c1_config(),
            "cpu_baseline": {"value": rate, "unit": "stars/s", "cores": 1, "kind": "port",
                             "sample": f"{fits} fits of the whole C1 field, FP64 oracle, one core"},
            "e2e": {"value": rate, "unit": "stars/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_gpu_c1(args):
    import torch

    import crowdphot_b200 as cpb
    from crowdphot_b200.simulate import c1_field
    img, bkg, iv, psf, src, init = c1_field(C1_SEED)
    ctx = cpb.get_context(0)
    kw = _c1_kwargs(iv, bkg)
    for _ in range(args.warmup):
        cpb.fit_all_stars_simultaneous(img, psf, init, 7, ctx=ctx, residual=False, **kw)
    ctx.kernel_stats(reset=True)
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    dev_s, walls, fitted = [], [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = cpb.fit_all_stars_simultaneous(img, psf, init, 7, ctx=ctx, residual=False, **kw)
        walls.append(time.perf_counter() - t0)
        dev_s.append(r.stats["device_seconds"])
        fitted += int((r.valid & r.converged).sum())
    clk = clocks.stop()
    _, launches = ctx.kernel_stats(reset=True)
    line = {"metric": C1_METRIC, "value": fitted / sum(dev_s), "unit": "stars/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(dev_s)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": c1_config(),
            "gpu_launches": launches, "clocks": clk, "n_passes": int(r.n_passes),
            "e2e": {"value": fitted / sum(walls), "unit": "stars/s", "h2d_bytes_per_step": 3 * img.nbytes + 3 * 8 * 200,
                    "d2h_bytes_per_step": 200 * (12 * 8 + 2 + 4)}}
    if not args.no_cpu:
        rate, fits, dt = _c1_cpu()
        line["cpu_baseline"] = {"value": rate, "unit": "stars/s", "cores": 1, "kind": "port",
                                "sample": f"{fits} fits of the whole C1 field, FP64 oracle, one core, {dt:.1f} s"}
    print(json.dumps(line))


def C_byref(x):
    import ctypes
    return ctypes.byref(x)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--ny", type=int, default=NY)
    ap.add_argument("--nx", type=int, default=NX)
    ap.add_argument("--n-stars", type=int, default=N_STARS)
    ap.add_argument("--workload", choices=["crowded-field", "lm-cutouts", "c4", "serve", "multipass", "c1"],
                    default="crowded-field",
                    help="crowded-field: the simultaneous fit (headline); lm-cutouts: batched fit_star; "
                         "c4: fit_star cutouts + blended groups in one CUDA-graph launch; "
                         "serve: a Poisson request stream through the continuous-batching server; "
                         "multipass: fit_all_stars (sequential passes run as batches of disjoint boxes); "
                         "c1: the 256^2 Gaussian field of the CPU-runnable configuration")
    ap.add_argument("--n-groups", type=int, default=C4_GROUPS)
    ap.add_argument("--n-requests", type=int, default=24)
    ap.add_argument("--max-inflight", type=int, default=4)
    ap.add_argument("--n-cutouts", type=int, default=LM_CUTOUTS)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-serve", action="store_true",
                    help="default workload: skip the served-stream comparison in forms.served_stream")
    ap.add_argument("--quick", action="store_true",
                    help="only the warm-up and timed resident steps (for profiler captures); prints a short line")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="with --quick: the form the resident steps run")
    args = ap.parse_args()
    ref = {"crowded-field": run_reference, "lm-cutouts": run_reference_lm, "c4": run_reference_c4,
           "serve": run_reference, "multipass": run_reference_mp, "c1": run_reference_c1}
    gpu = {"crowded-field": run_gpu, "lm-cutouts": run_gpu_lm, "c4": run_gpu_c4, "serve": run_gpu_serve,
           "multipass": run_gpu_mp, "c1": run_gpu_c1}
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return
        ref[args.workload](args)
    else:
        gpu[args.workload](args)


if __name__ == "__main__":
    main()

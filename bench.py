"""Benchmark: placement jobs/s of the B200 ElectroPlace path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload electro_200k_1024]

A step is one complete placement job of the workload (seeded synthetic
netlist with the benchmark configuration's shapes): initial placement, the
Nesterov loop run to overflow <= 0.10 (or max_iters), legalisation of every
checkpoint and the final binding.

  value  jobs/s with the netlist resident in HBM (context created before the
         timed region), timed with CUDA events around the K jobs.
  e2e    jobs/s through the C ABI's one-shot eplace_place with host buffers:
         upload, run and result download inside the timed region.

Multi-GPU: one placement job does not shard (every iteration needs the whole
bin map and global dot products), so N ranks run N independent replicas
(seed + rank), no data-path collective; value = jobs of all ranks / max rank
time ("weak" scaling).

`--impl reference` times the reference algorithm's CPU form (the FP64 C
restatement in oracle/, one thread per job like the reference loop) on whole
jobs of the same workload, K jobs spread over all host cores, and prints the
same metric.  It loads only oracle/liboracle.so.
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

METRIC = "placement jobs/s (run to overflow <= 0.10)"
UNIT = "jobs/s"
L2_BYTES = 126 * 1024 * 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="electro_200k_1024")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-reps", type=int, default=30)
    ap.add_argument("--dct", default="fft", choices=["fp32", "bf16x3", "fft"],
                    help="fft: FP32 FFTs (the plain form; power-of-two bin grids, else the FP32 GEMMs); "
                         "fp32: FP32 SIMT DCT-matrix GEMMs; bf16x3: tcgen05 three-term split GEMMs")
    ap.add_argument("--profile-only", action="store_true",
                    help="only run the per-kernel stage profiler (for ncu captures)")
    ap.add_argument("--field-mode", default="potential_gradient", choices=["reference", "potential_gradient"],
                    help="reference: the reference's field formula (default, parity); potential_gradient: the "
                         "opt-in extension that spreads cells")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched (64 mixed-size jobs) arm")
    ap.add_argument("--no-precision-form", action="store_true",
                    help="skip the per-kernel roofline of the 800k precision form (BF16x3 transform)")
    ap.add_argument("--no-served", action="store_true", help="skip the served (Poisson stream) arm")
    ap.add_argument("--batched-jobs", type=int, default=64)
    ap.add_argument("--served-jobs", type=int, default=2000,
                    help="jobs of the served stream (the configuration's 2,000; fewer for a subsample)")
    ap.add_argument("--served-rate", type=float, default=600.0,
                    help="offered rate of the served stream, jobs/s (above both forms' capacity, so the "
                         "throughput of each is measured)")
    ap.add_argument("--served-rate-2", type=float, default=0.0,
                    help="a second offered rate, e.g. 100 jobs/s, within the engine's capacity (0: skip)")
    ap.add_argument("--max-jobs", type=int, default=16, help="jobs the engine keeps on the GPU at once")
    ap.add_argument("--engine-dct", default="bf16x3", choices=["bf16x3", "fft"],
                    help="transform of the engine's jobs: bf16x3 (the mixed-precision form; FP32 FFT where the "
                         "grid is below 128 bins) or fft")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------
class Dist:
    def __init__(self, args):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, v):
        if not self.pg:
            return v
        import torch

        dev = "cuda" if torch.cuda.is_available() else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v):
        if not self.pg:
            return v
        import torch

        dev = "cuda" if torch.cuda.is_available() else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
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
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# roofline bookkeeping
# ---------------------------------------------------------------------------
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    return 6650.0, 1590.0, "fallback"


def algorithmic(nl, chip, dct="fp32"):
    """Algorithmic bytes / flops per launch of each iteration kernel.
    B_wl = 4(Nn+1) + 4P + 8P + 8N, B_sc = 8N + 8 n_macro + 4WH,
    B_fin = 8WH (read map) + 4WH (write charge), GEMM = 2 M N K flops,
    B_step = 68N + 8WH.  FFT form (dct "fft"), three stages: the first
    takes the finalise in and moves 8WH (map) + 4WH (T); the second 12WH (T
    in; U, V out: forward and back along y with the spectral step between);
    the third 16WH (U, V in; Ex, Ey out)."""
    N, Nn, P = nl.num_cells, nl.num_nets, nl.num_pins
    W = chip.bins_x or chip.width
    H = chip.bins_y or chip.height
    nmac = 0 if nl.cell_w is None else int((nl.cell_w.astype(np.int32) * nl.cell_h > 1).sum())
    return {
        "wa_grad": ("hbm", 4 * (Nn + 1) + 12 * P + 8 * N),
        "density_scatter": ("hbm", 8 * N + 8 * nmac + 4 * W * H),
        "density_final": ("hbm", 12 * W * H),
        "dct_gemm1": ("flops", 2 * H * W * W),
        "dct_gemm2_spectral": ("flops", 2 * H * W * H),
        "dct_gemm3": ("flops", 2 * 2 * H * W * W),
        "dct_gemm4": ("flops", 2 * 2 * H * W * H),
        "gather_step": ("hbm", 68 * N + 8 * W * H),
    } if dct != "fft" else {
        "wa_grad": ("hbm", 4 * (Nn + 1) + 12 * P + 8 * N),
        "density_scatter": ("hbm", 8 * N + 8 * nmac + 4 * W * H),
        "density_final": ("hbm", 0),
        "dct_gemm1": ("hbm", 12 * W * H),
        "dct_gemm2_spectral": ("hbm", 12 * W * H),
        "dct_gemm3": ("hbm", 16 * W * H),
        "dct_gemm4": ("hbm", 0),
        "gather_step": ("hbm", 68 * N + 8 * W * H),
    }


def precision_form_roofline(E, args, hbm, bf16, peak_src, workload="electro_800k_2048"):
    """Per-kernel CUDA-event times (one graph-replayed iteration) and their
    fractions of the measured peaks on the 800k-cell precision form."""
    w = E.WORKLOADS[workload]
    nl, chip = E.synth_netlist(w["spec"])
    cfg = E.ElectroPlaceCfg(**w["cfg"])
    opts = E.RunOptions(field_mode=1, dct_mode=1)
    with E.PlacementContext(nl, chip) as ctx:
        ms = ctx.profile_stages(cfg, reps=args.profile_reps, opts=opts)
    algo = algorithmic(nl, chip)
    out = {"workload": workload, "dct": "bf16x3 tcgen05",
           "peak_source": "measured (MEASURED_PEAKS.json)" if peak_src == "measured" else
           "fallback (%.0f GB/s, %.0f TFLOP/s)" % (hbm, bf16), "stages": {}}
    for k, t in ms.items():
        kd, am = algo[k]
        d = {"ms": t}
        if kd == "hbm":
            d.update({"algorithmic_bytes": am, "GB/s": am / (t / 1e3) / 1e9, "frac_hbm": am / (t / 1e3) / 1e9 / hbm,
                      "traffic": ncu_traffic(k, workload)})
        else:
            d.update({"algorithmic_flops": am, "TFLOP/s": am / (t / 1e3) / 1e12,
                      "frac_bf16": am / (t / 1e3) / 1e12 / bf16})
        out["stages"][k] = d
    return out


def field_fp64(density, field_mode=1, target_density=1.0, device="cpu"):
    """FP64 reference of the field solve (density.rs:96-166, with the
    potential-gradient extension for field_mode 1) as dense DCT-matrix
    products in torch float64: the yardstick for the precision report of the
    two FP32-accumulating transforms.  Conventions (rustdct, unnormalised):
    DCT-II C2[k,n] = cos(pi k (n+1/2)/N); DCT-III C3[k,n] = cos(pi n (k+1/2)/N)
    with input 0 halved; DST-III S3[k,n] = sin(pi (n+1)(k+1/2)/N) with input
    N-1 halved.  Returns (ex, ey, phi_hat) as [H, W] float64 tensors."""
    import torch

    d = torch.as_tensor(np.asarray(density, np.float64), device=device)
    H, W = d.shape

    def mats(N):
        k = torch.arange(N, dtype=torch.float64, device=device)[:, None]
        n = torch.arange(N, dtype=torch.float64, device=device)[None, :]
        c2 = torch.cos(np.pi * k * (n + 0.5) / N)
        c3 = torch.cos(np.pi * n * (k + 0.5) / N)
        c3[:, 0] *= 0.5
        s3 = torch.sin(np.pi * (n + 1) * (k + 0.5) / N)
        s3[:, N - 1] *= 0.5
        return c2, c3, s3

    c2w, c3w, s3w = mats(W)
    c2h, c3h, s3h = mats(H)
    rho = d - target_density * max(float(d.mean()), 1e-30)
    a = c2h @ (rho @ c2w.T)
    a = a * (4.0 / (W * H))
    a[:, 0] *= 0.5
    a[0, :] *= 0.5
    wx = (np.pi * torch.arange(W, dtype=torch.float64, device=device) / W)[None, :]
    wy = (np.pi * torch.arange(H, dtype=torch.float64, device=device) / H)[:, None]
    den = 2.0 * (1.0 - torch.cos(wx)) + 2.0 * (1.0 - torch.cos(wy))
    phi = torch.where(den < 1e-30, torch.zeros_like(a), a / torch.where(den < 1e-30, torch.ones_like(den), den))
    exh, eyh = phi * wx, phi * wy
    if field_mode == 1:
        exh = torch.cat([-exh[:, 1:], torch.zeros_like(exh[:, :1])], dim=1)
        eyh = torch.cat([-eyh[1:, :], torch.zeros_like(eyh[:1, :])], dim=0)
    ex = c3h @ (exh @ s3w.T)
    ey = s3h @ (eyh @ c3w.T)
    return ex, ey, phi


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s) if s > 0 else float(np.abs(a).max())


def precision_report(E, dev, workload="electro_800k_2048", state_iters=30):
    """The precision form's report: field and potential-spectrum error of the
    BF16x3 tensor-core transform, the FP32 SIMT transform and the FP32 FFT
    form against an FP64 solve of the same density map (taken from the
    workload's own run after `state_iters` iterations), and the whole job in
    each: HPWL trajectory, final legalised HPWL and overflow, beside the FP64
    oracle's committed run of the same job."""
    import torch

    nl, chip, cfg = E.workload(workload)
    out = {"workload": workload, "fields": {}, "jobs": {}}
    with E.PlacementContext(nl, chip, device=dev) as ctx:
        c = E.ElectroPlaceCfg(**E.WORKLOADS[workload]["cfg"])
        c.max_iters = state_iters
        st = ctx.run(c, E.RunOptions(field_mode=1, dct_mode=0))
        d, _ = ctx.density(st.x, st.y)
        rex, rey, rphi = (t.cpu().numpy() for t in field_fp64(d, 1, cfg.target_density, "cuda:%d" % dev))
        out["state"] = "density map of the best positions after %d iterations" % state_iters
        for name, mode in (("bf16x3_tcgen05", 1), ("fp32_simt", 0), ("fp32_fft", 2)):
            ex, ey, phi = ctx.field(d, dct_mode=mode, want_phi=True, field_mode=1)
            out["fields"][name] = {"field_x_rel_err": _rel(ex, rex), "field_y_rel_err": _rel(ey, rey),
                                   "potential_spectrum_rel_err": _rel(phi, rphi)}
        for name, mode in (("bf16x3_tcgen05", 1), ("fp32_simt", 0), ("fp32_fft", 2)):
            r = ctx.run(cfg, E.RunOptions(field_mode=1, dct_mode=mode))
            out["jobs"][name] = {"iters": r.iters, "converged": r.converged, "overflow": r.overlap,
                                 "final_hpwl": r.hpwl,
                                 "trajectory": [[t["iter"], int(t["hpwl"]), round(t["overlap"], 5)]
                                                for t in r.trajectory]}
    gp = os.path.join(ROOT, "tests", "golden", "job_summaries.json")
    key = workload + ":stable_wa"
    if os.path.exists(gp):
        with open(gp) as f:
            g = json.load(f).get(key)
        if g:
            out["jobs"]["fp64_oracle"] = {
                "iters": g["iters"], "converged": g["converged"], "final_hpwl": g["hpwl"],
                "source": "tests/golden/job_summaries.json %s (committed FP64 CPU run)" % key,
                "trajectory": [[c["iter"], int(c["hpwl"]), c["overlap"]] for c in g["checkpoints"]]}
            for name in ("bf16x3_tcgen05", "fp32_simt", "fp32_fft"):
                j = out["jobs"][name]
                j["final_hpwl_vs_fp64"] = j["final_hpwl"] / g["hpwl"] - 1.0
    out["error_definition"] = "max|x - x_fp64| / max|x_fp64| over the bin grid"
    return out


def ncu_traffic(kernel, workload):
    """dram bytes per launch from a committed ncu summary, if one exists."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for ln in f:
            if ln.startswith("#") or "=" not in ln:
                continue
            kv = dict(t.split("=", 1) for t in ln.split())
            if kv.get("stage") == kernel and kv.get("workload") == workload:
                return float(kv["dram_bytes_per_launch"])
    return None


# ---------------------------------------------------------------------------
# Batched and served forms: the job engine against the plain single-instance
# form on the same jobs.
# ---------------------------------------------------------------------------
def _mixed_jobs(E, specs, rank):
    """The jobs' netlists, generated on all host cores (the generator runs in
    C and releases the interpreter lock); not timed."""
    import concurrent.futures as cf

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        return list(ex.map(lambda sp: E.synth_netlist(replica_spec(sp, rank)), specs))


def _plain(E, jobs, cfg, opts, reuse, arrivals=None):
    """One job at a time through the single-instance API: a fresh context
    per job (reuse=False), or one context re-loaded per job (reuse=True).
    With arrivals, a job starts at max(its arrival, the previous job's end).
    Returns (seconds, results, latencies)."""
    ctx = None
    res, lat = [], []
    t0 = time.perf_counter()
    for k, (nl, chip) in enumerate(jobs):
        if arrivals is not None:
            wait = arrivals[k] - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        if reuse:
            if ctx is None:
                ctx = E.PlacementContext(nl, chip)
            else:
                ctx.load(nl, chip)
            res.append(ctx.run(cfg, opts))
        else:
            with E.PlacementContext(nl, chip) as c:
                res.append(c.run(cfg, opts))
        if arrivals is not None:
            lat.append(time.perf_counter() - t0 - arrivals[k])
    dt = time.perf_counter() - t0
    if ctx is not None:
        ctx.close()
    return dt, res, lat


def _engine(E, srv, jobs, cfg, arrivals=None):
    """All jobs through the engine (submitted at their arrival times when
    given).  Returns (seconds from the first submit to the last result,
    results, latencies)."""
    t0 = time.perf_counter()
    ids = []
    for k, (nl, chip) in enumerate(jobs):
        if arrivals is not None:
            wait = arrivals[k] - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        ids.append(srv.submit(nl, chip, cfg))
    out = [srv.wait(i) for i in ids]
    dt = time.perf_counter() - t0
    return dt, [r for r, _ in out], [info.latency_seconds for _, info in out]


def _agree(a, b):
    """Largest relative final-HPWL difference, jobs within 0.5 %, converged
    counts; and, for jobs whose two forms stop at different iterations (the
    stopping test overlap < 0.1 is discrete, so a last-digit difference can
    move it by one interval), the legalised HPWL at the last checkpoint both
    forms reached."""
    rel = [abs(x.hpwl - y.hpwl) / max(1, y.hpwl) for x, y in zip(a, b)]
    same_iter = []
    for x, y in zip(a, b):
        ty = {t["iter"]: t["hpwl"] for t in y.trajectory}
        common = [t for t in x.trajectory if t["iter"] in ty]
        if common:
            t = common[-1]
            same_iter.append(abs(t["hpwl"] - ty[t["iter"]]) / max(1.0, ty[t["iter"]]))
    return {"max_rel_hpwl_diff": max(rel), "within_0.5pct": int(sum(r <= 0.005 for r in rel)),
            "jobs_stopping_at_other_iteration": int(sum(x.iters != y.iters for x, y in zip(a, b))),
            "max_rel_hpwl_diff_at_last_common_checkpoint": max(same_iter) if same_iter else None,
            "converged": int(sum(x.converged for x in a)), "converged_plain": int(sum(y.converged for y in b)),
            "max_overflow": max(x.overlap for x in a)}


ENGINE_DCT = {"bf16x3": "bf16x3 tcgen05 (fp32 fft where bins < 128)", "fft": "fp32 fft"}


def batched_arm(args, dist, E, cfg):
    """64 instances, 2k..200k cells (log-uniform), mixed precision (BF16x3
    tensor-core transform where the bin grid allows it) through the engine,
    against the plain FP32 form one job at a time on the same jobs."""
    jobs = _mixed_jobs(E, E.batched_specs(args.batched_jobs), dist.rank)
    eng_opts = E.RunOptions(field_mode=1, dct_mode=1 if args.engine_dct == "bf16x3" else 2)
    plain_opts = E.RunOptions(field_mode=1, dct_mode=2)
    with E.JobServer(device=dist.local, max_jobs=args.max_jobs, opts=eng_opts) as srv:
        # Warm-up: one untimed pass over the same jobs (contexts created and
        # grown, process-wide device and pinned pools filled, kernels loaded).
        _engine(E, srv, jobs, cfg)
        # Three timed passes each (the engine's rate moves with the host
        # cores' scheduling of the legaliser threads); the median is reported.
        eng_passes = []
        for _ in range(3):
            dist.barrier()
            t, r_eng, _ = _engine(E, srv, jobs, cfg)
            eng_passes.append(dist.max(t))
        stats = srv.stats()
    dist.barrier()
    _plain(E, jobs, cfg, plain_opts, reuse=True)  # the same untimed pass for the plain form
    reuse_passes = []
    for _ in range(3):
        t, r_reuse, _ = _plain(E, jobs, cfg, plain_opts, reuse=True)
        reuse_passes.append(dist.max(t))
    t_fresh, _, _ = _plain(E, jobs, cfg, plain_opts, reuse=False)
    n = dist.sum(len(jobs))
    t_eng, t_reuse, t_fresh = float(np.median(eng_passes)), float(np.median(reuse_passes)), dist.max(t_fresh)
    cells = [nl.num_cells for nl, _ in jobs]
    return {
        "workload": "batched_%d_jobs_2k_200k" % len(jobs), "jobs": n,
        "cells_total": int(sum(cells)), "cells_min": int(min(cells)), "cells_max": int(max(cells)),
        "engine": {"jobs_per_s": n / t_eng, "seconds": t_eng, "max_jobs": args.max_jobs,
                   "passes_jobs_per_s": [n / t for t in eng_passes],
                   "dct": ENGINE_DCT[args.engine_dct], "contexts": stats["contexts"],
                   "device_bytes": stats["device_bytes"],
                   "scheduler_s": {k: round(stats[k + "_seconds"], 3) for k in ("admit", "pump", "idle")}},
        "plain_fp32_reused_ctx": {"jobs_per_s": n / t_reuse, "seconds": t_reuse, "dct": "fp32 fft",
                                  "passes_jobs_per_s": [n / t for t in reuse_passes]},
        "plain_fp32_fresh_ctx": {"jobs_per_s": n / t_fresh, "seconds": t_fresh},
        "speedup_vs_plain_reused_ctx": t_reuse / t_eng,
        "speedup_vs_plain_fresh_ctx": t_fresh / t_eng,
        "results_vs_plain": _agree(r_eng, r_reuse),
        "time_to_overflow_s_mean": float(np.mean([r.total_seconds for r in r_eng])),
        "warmup": "one untimed pass over the same jobs, each form",
        "timing": "median of three timed passes (engine, plain re-loaded context); one pass with fresh contexts",
    }


def served_arm(args, dist, E, cfg, rate):
    """A Poisson stream (fixed offered rate) of 1k..300k-cell jobs: the
    engine (continuous batching) against the plain form, which serves the
    same stream one job at a time in arrival order."""
    specs, arrivals = E.served_stream(args.served_jobs, rate)
    jobs = _mixed_jobs(E, specs, dist.rank)
    eng_opts = E.RunOptions(field_mode=1, dct_mode=1 if args.engine_dct == "bf16x3" else 2)
    plain_opts = E.RunOptions(field_mode=1, dct_mode=2)
    with E.JobServer(device=dist.local, max_jobs=args.max_jobs, opts=eng_opts) as srv:
        _engine(E, srv, jobs[: args.max_jobs], cfg)  # warm-up
        dist.barrier()
        t_eng, r_eng, lat_eng = _engine(E, srv, jobs, cfg, arrivals)
    dist.barrier()
    t_pl, r_pl, lat_pl = _plain(E, jobs, cfg, plain_opts, reuse=True, arrivals=arrivals)
    n = dist.sum(len(jobs))
    t_eng, t_pl = dist.max(t_eng), dist.max(t_pl)

    def pct(v, q):
        return float(np.percentile(v, q))

    return {
        "workload": "served_poisson_%d_jobs_1k_300k" % len(jobs), "jobs": n,
        "offered_rate_jobs_per_s": rate * dist.world,
        "sample": ("the whole 2,000-job stream" if len(jobs) == 2000 else
                   "first %d jobs of the 2,000-job stream" % len(jobs)) + " (seeds 100000+j, arrivals seed 7)",
        "engine": {"jobs_per_s": n / t_eng, "p50_latency_s": pct(lat_eng, 50), "p99_latency_s": pct(lat_eng, 99),
                   "max_jobs": args.max_jobs, "dct": ENGINE_DCT[args.engine_dct]},
        "plain_fp32": {"jobs_per_s": n / t_pl, "p50_latency_s": pct(lat_pl, 50), "p99_latency_s": pct(lat_pl, 99),
                       "dct": "fp32 fft"},
        "throughput_vs_plain": t_pl / t_eng,
        "p99_latency_vs_plain": pct(lat_pl, 99) / pct(lat_eng, 99),
        "results_vs_plain": _agree(r_eng, r_pl),
    }


# ---------------------------------------------------------------------------
# CPU form of the reference loop (the FP64 C restatement in oracle/): whole
# jobs, every checkpoint legalised, as place_electro runs them.  This part
# loads oracle/liboracle.so only: the netlist comes from the oracle's own
# copy of the generator and the workload table is read as data.
# ---------------------------------------------------------------------------
def _workload_table(name):
    with open(os.path.join(ROOT, "eisenjoch_b200", "workloads.json")) as f:
        w = json.load(f)[name]
    spec = dict(bins_x=0, bins_y=0, cluster_size=32, locality=0.6, macro_fraction=0.0, macro_min=2, macro_max=8)
    spec.update(w["spec"])
    return spec, w["cfg"]


_ORACLE_JOB = {}


def _oracle_problem(name):
    """The workload's netlist on the oracle (generated once per process)."""
    from types import SimpleNamespace

    from oracle.oracle import Cfg, Oracle, synth

    if name not in _ORACLE_JOB:
        spec, cfg = _workload_table(name)
        nl, chip = synth(SimpleNamespace(**spec))
        _ORACLE_JOB[name] = (Oracle(nl, chip), Cfg(**cfg))
    return _ORACLE_JOB[name]


def _oracle_job(name, field_mode):
    """One full placement job of workload `name` on the FP64 CPU form, in
    this process (1 thread).  Returns (seconds, summary)."""
    orc, cfg = _oracle_problem(name)
    t0 = time.perf_counter()
    st, r = orc.place(cfg, field_mode=field_mode)
    dt = time.perf_counter() - t0
    return dt, {"status": st, "iters": r["iters"], "converged": r["converged"], "hpwl": r["hpwl"]}


def _oracle_pool_jobs(name, field_mode, count, workers):
    """`count` full jobs on `workers` processes; returns (wall seconds of the
    batch, per-job summaries)."""
    import concurrent.futures as cf
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=ctx) as ex:
        # every worker generates the netlist before the clock starts
        list(ex.map(_prepare_worker, [(name, workers)] * workers))
        t0 = time.perf_counter()
        out = list(ex.map(_oracle_job, [name] * count, [field_mode] * count))
        dt = time.perf_counter() - t0
    return dt, [o for _, o in out]


def _prepare_worker(arg):
    name, _ = arg
    _oracle_problem(name)
    time.sleep(0.2)  # so that each worker takes one of the preparation tasks
    return os.getpid()


def cpu_baseline_one_job(name, field_mode):
    """cpu_baseline: one whole job of the workload on one host thread."""
    dt, r = _oracle_job(name, field_mode)
    sample = ("one full job of %s on the FP64 CPU form (oracle/), 1 thread: %d iterations, every checkpoint "
              "legalised, %.2f s" % (name, r["iters"], dt))
    return 1.0 / dt, sample, r


def reference_arm(args, dist):
    """The reference loop's CPU form on the host cores: each step is one
    whole job (initial placement, Nesterov iterations to overflow <= 0.10,
    every checkpoint legalised, final legalisation), K jobs spread over all
    host cores (one process per core, one job per process at a time);
    value = K / wall time of the K jobs.  W untimed jobs first."""
    if dist.rank != 0:
        return
    fm = 1 if args.field_mode == "potential_gradient" else 0
    spec, cfg = _workload_table(args.workload)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    t_start = time.perf_counter()
    if args.warmup > 0:
        _oracle_pool_jobs(args.workload, fm, args.warmup, min(cores, args.warmup))
    workers = min(cores, args.steps)
    dt, runs = _oracle_pool_jobs(args.workload, fm, args.steps, workers)
    value = args.steps / dt
    iters = sorted({r["iters"] for r in runs})
    sample = ("%d whole jobs of %s (FP64 CPU form of the reference loop, oracle/), %d processes x 1 thread on %d "
              "host cores; %s iterations per job, every checkpoint legalised; %.1f s wall" %
              (args.steps, args.workload, workers, cores, "/".join(map(str, iters)), dt))
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1000.0 * dt / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded generator, benchmark shapes)",
        "config": {"workload": args.workload, "cells": spec["num_cells"], "nets": spec["num_nets"],
                   "pads": spec["num_pads"], "sites": [spec["width"], spec["height"]],
                   "bins": [spec["bins_x"], spec["bins_y"]], "max_iters": cfg.get("max_iters", 500),
                   "legalize_interval": cfg.get("legalize_interval", 5),
                   "field_mode": args.field_mode, "parallelism": "%d processes" % workers},
        "job": {"iters": runs[0]["iters"], "converged": runs[0]["converged"], "hpwl": runs[0]["hpwl"]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.perf_counter() - t_start,
    }
    print(json.dumps(line), flush=True)


def replica_spec(spec, rank):
    """Rank r places its own netlist: the workload's generator with seed +
    7919 r (independent replicas, no data-path collective)."""
    import dataclasses

    return dataclasses.replace(spec, seed=spec.seed + 7919 * rank)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def ours(args, dist):
    import torch

    import eisenjoch_b200 as E

    dev = dist.local
    torch.cuda.set_device(dev)
    w = E.WORKLOADS[args.workload]
    nl, chip = E.synth_netlist(replica_spec(w["spec"], dist.rank))
    cfg = E.ElectroPlaceCfg(**w["cfg"])
    hbm, bf16, peak_src = peaks()

    dct_modes = {"fp32": 0, "bf16x3": 1, "fft": 2}
    opts = E.RunOptions(field_mode=1 if args.field_mode == "potential_gradient" else 0,
                        dct_mode=dct_modes[args.dct])
    ctx = E.PlacementContext(nl, chip, device=dev)
    # --- per-kernel device times (CUDA events on the library's stream) ---
    stage_ms = ctx.profile_stages(cfg, reps=args.profile_reps, opts=opts)
    if args.profile_only:
        if dist.rank == 0:
            print(json.dumps({"workload": args.workload, "dct": args.dct, "stage_ms": stage_ms}), flush=True)
        ctx.close()
        return
    # the other transform beside it: the FP32 GEMMs for the FFT and BF16x3
    # forms, BF16x3 for the FP32 GEMMs
    alt_opts = E.RunOptions(field_mode=opts.field_mode, dct_mode=1 if opts.dct_mode == 0 else 0)
    try:
        alt_stage_ms = ctx.profile_stages(cfg, reps=args.profile_reps, opts=alt_opts)
    except E.EplaceError as e:
        alt_stage_ms = {"unavailable": str(e)}
    for _ in range(args.warmup):
        ctx.run(cfg, opts)

    clocks = Clocks(dev)
    clocks.start()
    dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    lat, results = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = ctx.run(cfg, opts)
        lat.append(time.perf_counter() - t0)
        results.append(r)
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    total_s = e0.elapsed_time(e1) / 1000.0
    ck = clocks.stop()
    max_s = dist.max(total_s)
    jobs = dist.sum(args.steps)
    value = jobs / max_s

    # --- end to end through the C ABI with host buffers ---
    for _ in range(1):
        E.place_electro(nl, chip, cfg, opts, device=dev)
    dist.barrier()
    torch.cuda.synchronize()
    e0.record()
    e2e_res = []
    for _ in range(args.steps):
        e2e_res.append(E.place_electro(nl, chip, cfg, opts, device=dev))
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    e2e_s = dist.max(e0.elapsed_time(e1) / 1000.0)
    e2e_value = jobs / e2e_s
    ctx.close()

    # --- per-kernel roofline of the precision form (800k cells, 1024^2 bins,
    # BF16x3 transform): the configuration whose bytes exceed L2 ---
    prec = prec_report = None
    if not args.no_precision_form and dist.rank == 0:
        prec = precision_form_roofline(E, args, hbm, bf16, peak_src)
        prec_report = precision_report(E, dev)

    mixed_cfg = E.ElectroPlaceCfg(max_iters=500)
    batched = None if args.no_batched else batched_arm(args, dist, E, mixed_cfg)
    served = None if args.no_served else served_arm(args, dist, E, mixed_cfg, args.served_rate)
    served_2 = None
    if not args.no_served and args.served_rate_2 > 0:
        served_2 = served_arm(args, dist, E, mixed_cfg, args.served_rate_2)

    if dist.rank != 0:
        return

    r0 = results[-1]
    # --- roofline of the dominant kernel ---
    algo = algorithmic(nl, chip, args.dct)
    per_iter = {k: stage_ms[k] for k in stage_ms}
    dom = max(per_iter, key=lambda k: per_iter[k])
    kind, amount = algo[dom]
    dur_s = stage_ms[dom] / 1000.0
    if kind == "hbm":
        achieved = amount / dur_s / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm}
    else:
        achieved = amount / dur_s / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s", "frac": achieved / bf16}
    roof["traffic"] = ncu_traffic(dom, args.workload)
    roof["kernel"] = dom
    roof["peak_source"] = peak_src + " (MEASURED_PEAKS.json)" if peak_src == "measured" else "fallback"
    roof["algorithmic_per_launch"] = amount
    stages = {}
    for k, ms in stage_ms.items():
        kd, am = algo[k]
        if kd == "hbm":
            stages[k] = {"ms": ms, "GB/s": am / (ms / 1e3) / 1e9}
            if args.dct == "fft" and k == "density_final":
                stages[k]["note"] = "fused into the first FFT stage (the time is the empty graph node's)"
            if args.dct == "fft" and k == "dct_gemm4":
                stages[k]["note"] = "the FFT form has three stages (the time is the empty graph node's)"
        else:
            stages[k] = {"ms": ms, "TFLOP/s": am / (ms / 1e3) / 1e12}

    cpu = None
    if not args.no_cpu_baseline and dist.world == 1:
        v, sample, _ = cpu_baseline_one_job(args.workload, opts.field_mode)
        cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample}

    launches = sum(r.gpu_launches for r in results)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": dist.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": max_s * 1000.0 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "bf16x3->f32 (FP64 global reductions)" if args.dct == "bf16x3" else "f32 (FP64 global reductions)",
        "data": "synthetic (seeded generator, benchmark shapes); replica r uses seed + 7919 r",
        "config": {
            "workload": args.workload,
            "cells": nl.num_cells, "nets": nl.num_nets, "pins": nl.num_pins, "pads": nl.num_fixed,
            "sites": [chip.width, chip.height], "bins": [chip.bins_x, chip.bins_y],
            "max_iters": cfg.max_iters, "legalize_interval": cfg.legalize_interval,
            "parallelism": "replicas x%d" % dist.world,
            "l2": "per-iteration working set is L2-resident at this size; no flush between jobs "
                  "(each job runs hundreds of iterations)",
            "dct": {"fp32": "fp32 simt gemm", "bf16x3": "tcgen05 bf16 3-term split, fp32 accumulate",
                    "fft": "fp32 fft (one N-point FFT per line)"}[args.dct],
            "field_mode": args.field_mode + ("" if args.field_mode == "reference" else
                                             " (extension: the reference field does not spread cells; on this "
                                             "workload the reference FP64 loop reaches a non-finite gradient at iteration 50)"),
        },
        "job": {
            "iters": r0.iters, "converged": r0.converged, "overlap": r0.overlap, "hpwl": r0.hpwl,
            "best_iter": r0.best_iter, "time_to_overflow_s": statistics.median(lat),
            "gpu_loop_s": r0.gpu_seconds, "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)),
            "iter_us": 1e6 * r0.gpu_seconds / max(1, r0.iters),
        },
        "e2e": {
            "value": e2e_value, "unit": UNIT,
            "h2d_bytes_per_step": int(np.mean([r.h2d_bytes for r in e2e_res])),
            "d2h_bytes_per_step": int(np.mean([r.d2h_bytes for r in e2e_res])),
        },
        "roofline": roof,
        "stages": stages,
        "stages_other_dct_ms": alt_stage_ms,
        "cpu_baseline": cpu,
        "gpu_launches": int(launches),
        "clocks": ck,
        "precision_form_stages": prec,
        "precision_form": prec_report,
        "batched": batched,
        "served": served,
        "served_rate_2": served_2,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    dist = Dist(args)
    try:
        if args.impl == "reference":
            reference_arm(args, dist)
        else:
            ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()

"""Benchmark: ABMC-ICCG to relative residual 1e-8 on one B200.

Workload (one step = one full solve of one system):
  3D 7-point Laplacian, 128^3 grid (n = 2,097,152, nnz = 14,581,760),
  coefficients 1, 1, 0.01; ABMC with block size 16 (16 consecutive rows per
  block, greedy block coloring: 2 colors), b = A x*, x* ~ U(-1,1) from
  splitmix64(0); x0 = 0;
  IC(0) preconditioner; A and L stored in FP32, x / r / p / z and all inner
  products in FP64, FP64 residual replacement every 50 iterations; converged
  when the FP64 true relative residual is below 1e-8.

Prints ONE JSON line (rank 0).  `value` is the device time per solve
(CUDA events around the timed steps, max over ranks); `e2e` repeats the
measurement through the C ABI with host (pinned) buffers, copies included.
`--impl reference` times the reference's own OpenMP CPU code (compiled from
its sources into oracle/_ref) on the same problem.

Multi-GPU: one process per GPU (torchrun); each rank solves its own replica
of the system (independent solves, no data-path collective: weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SIDE = 128
BLOCK = 16
BLOCKING = "linear"   # 16 consecutive rows per block: 2 block colors on this grid
TOL = 1e-8
RR = 50
METRIC = "ICCG ms to resid 1e-8 (ABMC B=16, 3D 7-pt 128^3 aniso, FP32 storage / FP64 recurrences)"
WORKLOAD = "abmc_iccg_laplace3d_aniso_128"


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_problem():
    import iccg_b200.problems as pb
    t0 = time.perf_counter()
    P = pb.config_abmc_aniso(SIDE, BLOCK, BLOCKING, seed=0)
    return P, time.perf_counter() - t0


def bytes_model(P, storage_bytes: int):
    """Algorithmic bytes (compulsory traffic) of the kernels of one PCG iteration."""
    n = P.A_run.n
    nnz = P.A_run.nnz
    nnzS = (nnz - n) // 2                   # strict lower (= strict upper) entries of L
    sv = storage_bytes
    S_A = nnz * (sv + 4) + 4 * (n + 1)
    S_L = nnzS * (sv + 4) + 4 * (n + 1) + sv * n   # strict part + row pointers + diagonal
    return {
        "spmv": S_A + 16 * n,                 # A, p gathered (compulsory once), Ap written
        "fwd_sweep": S_L + 16 * n,            # r read, y written
        "bwd_sweep": S_L + 24 * n,            # y read, z written, r read for r.z
        "iteration": S_A + 2 * S_L + 16 * 8 * n,
    }


def _solve_case(P, device: int, with_plain: bool = True) -> dict:
    """One system: the mixed form (FP32 A and L, FP64 vectors, replacement
    every RR) and the FP64 fused and plain forms, each timed by CUDA events
    (median of 3 after a warm-up solve), with iterations, the true residual
    and the mixed solution's error against the FP64 one."""
    import iccg_b200 as ib
    ctx = ib.Context(device)
    ctx.upload(P.A_run)
    ctx.set_schedule(P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    out = {"n": P.A_run.n, "nnz": P.A_run.nnz, "colors": P.nc}
    xs = {}
    forms = [("mixed", ib.STORE_FP32, ib.MODE_FUSED), ("fp64_fused", ib.STORE_FP64, ib.MODE_FUSED)]
    if with_plain:
        forms.append(("fp64_plain", ib.STORE_FP64, ib.MODE_PLAIN))
    for name, st, mode in forms:
        ms = []
        for _ in range(4):
            x = np.zeros(P.A_run.n)
            r = ctx.solve(P.b_run, x, 10000, TOL, mode=mode, storage=st, rr_interval=RR)
            ms.append(r.solve_ms)
        xs[name] = x
        out[name] = {"ms": round(statistics.median(ms[1:]), 4), "iters": r.iters, "converged": r.converged,
                     "true_rel_resid": r.true_rel_resid}
    x64 = xs["fp64_fused"]
    out["mixed"]["err_vs_fp64_solution"] = float(np.linalg.norm(xs["mixed"] - x64) / np.linalg.norm(x64))
    out["speedup_mixed_vs_fp64_fused"] = round(out["fp64_fused"]["ms"] / out["mixed"]["ms"], 3)
    ctx.close()
    return out


def serving_case(device: int, requests: int = 48, max_points: float = 1e5, rate: float = 30.0,
                 builders: int = 16) -> dict:
    """A short serving stream for the headline line: `requests` kNN-Laplacian
    solves (N log-uniform in [1e3, max_points]) arriving as a Poisson
    process at `rate` per second, through the continuous-batching loop
    (batch.ServingLoop) under the 100 GB budget; solves/s and p50 / p99
    latency, arrival to result with host set-up included.  Two requests
    are also solved alone and through a batch session, to check the bits."""
    import iccg_b200 as ib
    import iccg_b200.batch as bt
    import iccg_b200.problems as pb
    rng = np.random.default_rng(11)
    sizes = [int(np.exp(rng.uniform(np.log(1e3), np.log(max_points)))) for _ in range(requests)]
    arr = np.random.default_rng(13)
    t, reqs = 0.0, []
    for i, npts in enumerate(sizes):
        t += arr.exponential(1.0 / rate)
        reqs.append(bt.Request(i, t, (lambda npts=npts, i=i: pb.config_knn(npts, seed=i)),
                               bt.estimate_device_bytes(npts, 18 * npts)))
    loop = bt.ServingLoop(budget_bytes=100 * 10**9, device=device, builders=builders, slots=256, graph_iters=4,
                          rr_interval=RR)
    st = bt.serve_sharded(reqs, loop, dist=None)
    same, plain = True, []
    B = ib.Batch(device)
    B.open(1, ib.STORE_FP32, rr_interval=RR, graph_iters=4)
    for i, npts in enumerate(sizes[:2]):
        P = pb.config_knn(npts, seed=i)
        c = bt.batch_context(device)
        bt.load_system(c, P, ib.STORE_FP32)
        x = np.zeros(P.A_run.n)
        r = c.solve(P.b_run, x, 10000, TOL, storage=ib.STORE_FP32, rr_interval=RR, graph_iters=4)
        k = B.add_system(c)
        B.submit(k, P.b_run, None, 10000, TOL)
        while True:
            stopped, _ = B.step()
            if stopped:
                break
        xb, rb = B.retire(stopped)
        B.remove_system(k)
        same = same and np.array_equal(xb[0], x) and rb[0].iters == r.iters
        xp = np.zeros(P.A_run.n)
        plain.append(c.solve(P.b_run, xp, 10000, TOL, storage=ib.STORE_FP64, mode=ib.MODE_PLAIN).solve_ms)
        c.close()
    B.close()
    return {"requests": requests, "points": {"min": min(sizes), "max": max(sizes), "distribution": "log-uniform"},
            "arrival_rate_per_s": rate, "solves_per_s": st.get("solves_per_s"), "p50_ms": st.get("p50_ms"),
            "p99_ms": st.get("p99_ms"), "failed": st.get("failed"), "mean_iters": st.get("mean_iters"),
            "peak_device_bytes": (st.get("peak_device_bytes_per_rank") or [None])[0],
            "plain_fp64_solve_ms_alone": [round(v, 3) for v in plain],
            "batch_session_same_bits_as_alone": bool(same)}


def sub_results(device: int) -> dict:
    """Short results of the other workloads, carried on the headline line:
    C1 the 2D 5-point 128^2 Poisson problem with greedy multicolor IC(0);
    C3 the 27-point variable-coefficient 96^3 problem, multicolor and ABMC
    B=8; the batched engine on 64 of the batched workload's systems x 4
    right-hand sides; a short serving stream (serving_case)."""
    import iccg_b200.problems as pb
    out = {}
    t0 = time.perf_counter()
    try:
        out["c1_poisson2d_128_mc"] = _solve_case(pb.config_small_mc(128, seed=0), device)
        for key, (v, B) in {"c3_diffusion27_96_mc": ("piccg", 16), "c3_diffusion27_96_abmc8": ("abmc", 8)}.items():
            out[key] = _solve_case(pb.config_diffusion27(96, v, block_size=B, seed=0), device, with_plain=False)
        out["batched_64x4"] = batched_case(64, 4, steps=2, warmup=1, device=device, compare_streams=False, sample=8)
        out["serving_48"] = serving_case(device)
    except Exception as e:   # the headline number stands; the failure is shown, not hidden
        out["error"] = repr(e)
    out["wall_s"] = round(time.perf_counter() - t0, 1)
    return out


def run_gpu(args):
    import torch
    import iccg_b200 as ib

    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local = _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    P, setup_s = build_problem()
    n = P.A_run.n
    ctx = ib.Context(local)
    # set-up phases, wall time each (every call ends with its stream synced)
    setup_ms = {"host_problem": setup_s * 1e3}
    t0 = time.perf_counter()
    ctx.upload(P.A_run)
    t1 = time.perf_counter()
    ctx.set_schedule(P.sched)
    t2 = time.perf_counter()
    ctx.build(ib.PRECOND_IC0, 0.0)
    t3 = time.perf_counter()
    setup_ms.update(upload=(t1 - t0) * 1e3, schedule=(t2 - t1) * 1e3, ic0_build=(t3 - t2) * 1e3)
    stream = torch.cuda.ExternalStream(ctx.stream)
    dev = torch.device("cuda", local)
    b_d = torch.from_numpy(P.b_run).to(dev)
    x_d = torch.zeros(n, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    def solve(storage, mode=ib.MODE_FUSED):
        with torch.cuda.stream(stream):
            x_d.zero_()
        return ctx.solve_dev(b_d.data_ptr(), x_d.data_ptr(), 10000, TOL, mode=mode, storage=storage, rr_interval=RR)

    # FP64 reference solution on the device (for the error report); the
    # first solve also builds the lane-interleaved system and its graphs
    t0 = time.perf_counter()
    r64 = solve(ib.STORE_FP64)
    torch.cuda.synchronize()
    setup_ms["first_solve_fp64_with_q_build"] = (time.perf_counter() - t0) * 1e3
    setup_ms["first_solve_fp64_device"] = r64.solve_ms
    x64 = x_d.cpu().numpy().copy()
    for _ in range(args.warmup):
        solve(ib.STORE_FP32)
    # timed region: barrier, CUDA events on the context's stream, barrier,
    # slowest rank's time (replicas: no collective on the data path)
    from iccg_b200.replicas import timed_replicas, max_over_ranks
    clocks = ClockSampler(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches0 = ctx.launches
    results = []

    def timed():
        clocks.start()
        with torch.cuda.stream(stream):
            e0.record(stream)
        for _ in range(args.steps):
            results.append(solve(ib.STORE_FP32))
        with torch.cuda.stream(stream):
            e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    tr = timed_replicas(timed, args.steps, dist=dist, device=dev, sync=torch.cuda.synchronize)
    launches = ctx.launches - launches0
    clk = clocks.stop()
    total_ms = tr.ms
    ms_per = total_ms / args.steps
    r32 = results[-1]
    x32 = x_d.cpu().numpy()
    err = float(np.linalg.norm(x32 - x64) / np.linalg.norm(x64))
    per_solve = [r.solve_ms for r in results]

    # plain FP64 path (one kernel per reference op, host-checked) and fused
    # FP64, outside the timed region: the median of 3 solves each
    def median_solve(storage, mode):
        rs = sorted((solve(storage, mode) for _ in range(3)), key=lambda r: r.solve_ms)
        return rs[1]

    plain = median_solve(ib.STORE_FP64, ib.MODE_PLAIN)
    fused64 = median_solve(ib.STORE_FP64, ib.MODE_FUSED)

    # per-kernel device time.  The solve's kernels run back to back inside
    # CUDA graphs (with programmatic dependent launch), so a kernel's time is
    # its share of the graph-replayed solve -- from the committed ncu launch
    # list of the same solve -- times the event-timed solve above.  One more
    # solve with every launch bracketed by CUDA events (no graphs) is
    # reported beside it; it runs about a fifth slower.
    ctx.profile(True)
    rp = solve(ib.STORE_FP32)
    brk = {}
    names = {0: "spmv", 1: "fwd_sweep", 2: "bwd_sweep", 3: "vector", 4: "residual"}
    for cls, nm in names.items():
        brk[nm] = ctx.profile_read(cls)
    ctx.profile(False)
    iters = r32.iters
    bm = bytes_model(P, 4)
    peak, peak_kind = _peaks()
    shares = _launch_shares()
    kernels = {}
    for nm in ("spmv", "fwd_sweep", "bwd_sweep", "vector", "residual"):
        b_ms, b_cnt = brk[nm]
        per = "launch" if nm == "spmv" else "sweep" if nm.endswith("sweep") else "solve"
        units = {"launch": iters + 1, "sweep": iters + 1, "solve": 1}[per]   # SpMV / sweeps: one per iteration + r0's
        if nm == "spmv":
            units = iters
        k = {"per": per, "bracketed_ms": round(b_ms / units, 5), "bracketed_launches": b_cnt}
        if shares is not None and nm in shares:
            k["share"] = round(shares[nm], 4)
            k["ms"] = round(shares[nm] * ms_per / units, 5)
        else:
            k["ms"] = k["bracketed_ms"]
        if nm in bm:
            k["bytes"] = bm[nm]
            gbs = bm[nm] / (k["ms"] * 1e-3) / 1e9 if k["ms"] > 0 else 0.0
            k["GB/s"] = round(gbs, 1)
            k["frac"] = round(gbs / peak, 4)
        kernels[nm] = k
    # the dominant kernel: largest device time per solve; per-launch figures
    # (a sweep is one launch per color)
    kernel_ms = {nm: kernels[nm]["ms"] * (iters if nm == "spmv" else iters + 1)
                 for nm in ("spmv", "fwd_sweep", "bwd_sweep")}
    dom_name = max(kernel_ms, key=kernel_ms.get)
    launches_per_unit = 1 if dom_name == "spmv" else max(1, P.nc)
    dom = dict(kernels[dom_name])
    dom["bytes"] = bm[dom_name] // launches_per_unit
    traffic = _traffic_from_profiles(dom_name)
    dom_label = {"spmv": "k_spmv_q: SpMV p -> Ap with p.Ap, p.p, Ap.Ap (FP32 values, FP64 vectors)",
                 "fwd_sweep": "forward substitution L y = r, one launch per color (k_sweep_chain for the color "
                              "with in-block entries only, k_sweep_st for the other; FP32 factor)",
                 "bwd_sweep": "backward substitution L^T z = y with r.z, one launch per color (k_sweep_chain for "
                              "the color with in-block entries only, k_sweep_st for the other; FP32 factor)"}[dom_name]

    # e2e: through the C ABI with host (pinned) buffers, H2D of b and x0 and D2H of x inside the timed region
    pin_b = torch.from_numpy(P.b_run).pin_memory()
    pin_x = torch.zeros(n, dtype=torch.float64).pin_memory()
    xb = pin_x.numpy()
    e2e = []
    for _ in range(max(1, min(args.steps, 5))):
        xb[:] = 0.0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.solve(pin_b.numpy(), xb, 10000, TOL, storage=ib.STORE_FP32, rr_interval=RR)
        e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = max_over_ranks(statistics.median(e2e), dist=dist, device=dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(P, samples=args.cpu_samples)
    subs = None
    if world == 1 and not args.no_sub_results:
        ctx.close()
        ctx = None
        subs = sub_results(local)

    line = {
        "metric": METRIC,
        "value": round(ms_per, 4),
        "unit": "ms",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_per, 4),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "storage": "fp32 A and L, fp64 vectors and reductions",
        "data": "synthetic",
        "config": headline_config(n, P.A_run.nnz, P.nb, P.nc),
        "parallelism": f"replicas x{world}",
        "solves_per_s": round(tr.units_per_s, 3),
        "iters": r32.iters,
        "true_rel_resid": r32.true_rel_resid,
        "residual_replacements": r32.n_replacements,
        "err_vs_fp64_solution": err,
        "per_solve_ms": {"p50": round(statistics.median(per_solve), 4), "max": round(max(per_solve), 4)},
        "fp64": {"fused_ms": round(fused64.solve_ms, 4), "fused_iters": fused64.iters,
                 "plain_ms": round(plain.solve_ms, 4), "plain_iters": plain.iters,
                 "true_rel_resid": r64.true_rel_resid},
        "speedup_vs_plain_fp64": round(plain.solve_ms / ms_per, 3),
        "speedup_vs_fused_fp64": round(fused64.solve_ms / ms_per, 3),
        "roofline": {"bound": "hbm", "kernel": dom_label, "achieved": dom["GB/s"],
                     "peak": peak, "unit": "GB/s", "frac": dom["frac"], "peak_source": peak_kind,
                     "traffic": traffic, "algorithmic_bytes_per_launch": dom["bytes"],
                     "share_of_solve": round(kernel_ms[dom_name] / max(ms_per, 1e-9), 3)},
        "kernels": kernels,
        "kernels_timing": ("ms = share of the solve in the committed ncu launch list (profiles/"
                           "launches_solve_abmc128.md) x the event-timed solve; bracketed_ms: one extra solve "
                           "with every launch bracketed by CUDA events, no graphs") if shares else
                          "each launch bracketed by CUDA events in one extra solve (no graphs)",
        "iteration_bytes": bm["iteration"],
        "iteration_GBps": round(bm["iteration"] * iters / (rp.solve_ms * 1e-3) / 1e9, 1) if rp.solve_ms else None,
        "gpu_launches": int(launches),
        "e2e": {"value": round(e2e_ms, 4), "unit": "ms", "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 8 * n},
        "setup_ms": {k: round(v, 2) for k, v in setup_ms.items()},
        "clocks": clk,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if subs is not None:
        line["sub_results"] = subs
    if ctx is not None:
        ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def _kernel_class(name: str):
    """The solve part a kernel of the launch list belongs to (None: set-up)."""
    import re
    if name.startswith("iccg::k_spmv_q"):
        return "spmv"
    m = re.match(r"iccg::k_sweep_(?:st|chain|q2|q)<\w+, (\d)", name)
    if m:
        return "fwd_sweep" if m.group(1) == "1" else "bwd_sweep"
    if name.startswith("iccg::k_persist"):
        return "persistent"
    if name.startswith(("iccg::k_update", "iccg::k_xpay", "iccg::k_copy", "iccg::k_resume", "iccg::k_apply_xp",
                        "iccg::k_clear_xp")):
        return "vector"
    if name.startswith("iccg::k_residual_q"):
        return "residual"
    return None


def _launch_shares(name: str = "launches_solve_abmc128.md"):
    """Each solve part's share of the solve's device time, from the committed
    ncu launch list (kernel, launches, total ms, share rows)."""
    import re
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    tot = {}
    for kname, _, ms, _ in re.findall(r"^\| `([^`]+)` \| (\d+) \| ([\d.]+) \| ([\d.]+)%", p.read_text(), re.M):
        cls = _kernel_class(kname)
        if cls is not None:
            tot[cls] = tot.get(cls, 0.0) + float(ms)
    s = sum(tot.values())
    return {k: v / s for k, v in tot.items()} if s > 0 else None


_PROFILE_OF = {"spmv": "ncu_spmv_abmc128.txt", "bwd_sweep": "ncu_sweep_st_abmc128.txt"}


def _traffic_from_profiles(kernel: str):
    """DRAM bytes per launch of `kernel` from its committed ncu summary, if any."""
    name = _PROFILE_OF.get(kernel)
    p = ROOT / "profiles" / name if name else None
    if p is None or not p.exists():
        return None
    for ln in p.read_text().splitlines():
        if ln.startswith("traffic_bytes_per_launch:"):
            try:
                return float(ln.split(":", 1)[1])
            except ValueError:
                return None
    return None


def cpu_baseline(P, samples=3):
    """The reference's OpenMP CG (compiled from its sources) on the same
    problem, all host cores; or the oracle port on one core if the compiled
    reference is absent."""
    from oracle import bindings as ob
    n = P.A.n
    if ob.ref() is not None:
        cores = os.cpu_count() or 1
        ob.ref().ref_set_threads(cores)
        R = ob.RefProblem(4, n, P.A.rowptr, P.A.colind, P.A.val, P.block_of_old, P.nb, P.block_color, P.nc)
        times, iters = [], 0
        for _ in range(samples):
            x, it, rel, cv, us = R.cg(P.b_run, np.zeros(n), 10000, TOL)
            times.append(us / 1e3)
            iters = it
        return {"value": round(statistics.median(times), 3), "unit": "ms", "cores": cores, "kind": "reference",
                "sample": f"{samples} full ABMC-ICCG solves of the same 128^3 system (median), {iters} iterations, "
                          f"conjugate_gradient only (cg_crs.cpp:507-510)"}
    rp, ci, v = P.A_run.rowptr, P.A_run.colind, P.A_run.val
    ic0 = ob.OracleIC0(n, rp, ci, v, 0.0)
    t0 = time.perf_counter()
    x, it, rel, cv, _ = ob.cg(n, rp, ci, v, P.b_run, np.zeros(n), 2, 10000, TOL, ic0, P.sched)
    ms = (time.perf_counter() - t0) * 1e3
    return {"value": round(ms, 3), "unit": "ms", "cores": 1, "kind": "port",
            "sample": f"1 full solve by the C restatement ({it} iterations)"}


def headline_config(n: int, nnz: int, nb: int, nc: int) -> dict:
    """The headline workload, the same in both arms' lines."""
    return {"workload": WORKLOAD, "n": n, "nnz": nnz, "grid": f"{SIDE}^3", "coeffs": [1, 1, 0.01],
            "block_size": BLOCK, "blocking": BLOCKING, "nb": nb, "colors": nc, "tol": TOL, "rr_interval": RR,
            "x0": "zeros", "rhs": "b = A x*, x* ~ U(-1,1) splitmix64(0)",
            "l2": "inputs larger than L2: ~0.5 GB streamed per iteration vs 126 MB L2"}


def _splitmix_uniform(n: int, seed: int) -> np.ndarray:
    """x_i ~ U(-1,1): the i-th splitmix64 output of `seed`, top 53 bits."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (np.arange(1, n + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53 * 2.0 - 1.0


def reference_inputs(workdir: Path):
    """The headline problem for the reference arm, made without this
    package's library and read back through the reference's own readers
    (read_matrix_market_crs, crs_io.cpp:73-159; ReadBlockFile_1Based /
    ReadBlockColorFile_1Based, block.cpp:15-89), as its driver reads them.

    The 3D 7-point stencil (x fastest; entries -0.01 (z-), -1 (y-), -1 (x-),
    2 (1 + 1 + 0.01), -1 (x+), -1 (y+), -0.01 (z+)) is written as a
    symmetric MatrixMarket file; blocks are 16 consecutive rows; the greedy
    block coloring in block order of this bipartite block grid is the parity
    of (block x + y + z), two colors.  b = A x* with x* the splitmix64(0)
    U(-1,1) sequence, summed in row order."""
    from oracle import bindings as ob
    N = SIDE
    n = N ** 3
    idx = np.arange(n, dtype=np.int64)
    x, y, z = idx % N, (idx // N) % N, idx // (N * N)
    diag = 2.0 * (1.0 + 1.0 + 0.01)
    # lower triangle, row by row: (z-), (y-), (x-), diagonal
    parts = [(z > 0, -N * N, -0.01), (y > 0, -N, -1.0), (x > 0, -1, -1.0), (np.ones(n, bool), 0, diag)]
    rows, cols, vals = [], [], []
    for m, off, v in parts:
        r = idx[m]
        rows.append(r)
        cols.append(r + off)
        vals.append(np.full(r.size, v))
    order = np.lexsort((np.concatenate(cols), np.concatenate(rows)))
    I = np.concatenate(rows)[order] + 1
    J = np.concatenate(cols)[order] + 1
    V = np.concatenate(vals)[order]
    u, inv = np.unique(V, return_inverse=True)
    vs = np.array([repr(float(t)) for t in u])
    lines = np.char.add(np.char.add(np.char.add(np.char.add(I.astype(str), " "), J.astype(str)), " "), vs[inv])
    mtx = workdir / "laplace3d_aniso_128.mtx"
    with open(mtx, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n")
        f.write(f"{n} {n} {I.size}\n")
        f.write("\n".join(lines.tolist()))
        f.write("\n")
    nb = n // BLOCK
    blk = workdir / "laplace3d_aniso_128.blk"
    with open(blk, "w") as f:
        f.write(f"{nb}\n")
        f.write("\n".join(f"{i + 1} {i // BLOCK + 1}" for i in range(n)))
        f.write("\n")
    b_idx = np.arange(nb)
    bx, by, bz = b_idx % (N // BLOCK), (b_idx // (N // BLOCK)) % N, b_idx // ((N // BLOCK) * N)
    bcolor = (bx + by + bz) % 2
    bcol = workdir / "laplace3d_aniso_128.bcol"
    with open(bcol, "w") as f:
        f.write("2\n")
        f.write("\n".join(f"{b + 1} {c + 1}" for b, c in enumerate(bcolor.tolist())))
        f.write("\n")
    # read back with the reference's readers
    n_, rowptr, colind, val = ob.ref_read_mm(str(mtx))
    block_of_old, nb_ = ob.ref_read_assignment(1, str(blk), n_)
    block_color, nc = ob.ref_read_assignment(2, str(bcol), nb_)
    R = ob.RefProblem(4, n_, rowptr, colind, val, block_of_old, nb_, block_color, nc)
    # b = A x* in the original order (row order sums), then into the run order
    xs = _splitmix_uniform(n_, 0)
    b = np.zeros(n_)
    cnt = np.diff(rowptr)
    for j in range(int(cnt.max())):
        has = cnt > j
        pos = rowptr[:-1][has] + j
        b[has] = b[has] + val[pos] * xs[colind[pos]]
    b_run = np.empty_like(b)
    b_run[R.perm()] = b
    return R, b_run, headline_config(n_, int(rowptr[-1]), nb_, nc)


def run_reference(args):
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    if rank != 0:
        return
    from oracle import bindings as ob
    if ob.ref() is None:
        print(json.dumps({"impl": "reference", "unavailable": "compiled reference (oracle/_ref) not present"}))
        return
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        R, b_run, config = reference_inputs(Path(td))
    n = config["n"]
    cores = os.cpu_count() or 1
    ob.ref().ref_set_threads(cores)
    for _ in range(args.warmup):
        R.cg(b_run, np.zeros(n), 10000, TOL)
    times, iters, rel = [], 0, 0.0
    for _ in range(args.steps):
        x, it, rel, cv, us = R.cg(b_run, np.zeros(n), 10000, TOL)
        times.append(us / 1e3)
        iters = it
    ms = statistics.mean(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(ms, 3), "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config, "parallelism": f"OpenMP x{cores} host threads",
        "inputs": "made with numpy, written as .mtx/.blk/.bcol and read by the reference's own readers",
        "iters": iters, "rel_resid": rel,
        "cpu_baseline": {"value": round(ms, 3), "unit": "ms", "cores": cores, "kind": "reference",
                         "sample": f"{args.steps} full solves (mean), conjugate_gradient only"},
        "e2e": {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="iccg_b200", choices=["iccg_b200", "reference"])
    ap.add_argument("--cpu-samples", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sub-results", action="store_true",
                    help="headline only: leave out the C1 / C3 / batched sub-results")
    ap.add_argument("--kernel-only", choices=["spmv", "apply", "solve"], default=None,
                    help="set up the workload, then launch only this operation --reps times "
                         "(FP32 storage) and print its mean device time; for profilers")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--kernel-storage", choices=["fp32", "fp64"], default="fp32",
                    help="--kernel-only: storage of A and L (fp32: the headline's mixed form)")
    ap.add_argument("--persist", type=int, choices=[0, 1], default=0,
                    help="--kernel-only: 1 runs each IC(0) apply as one persistent launch; 0 (the default, "
                         "as the headline solve) one launch per level")
    ap.add_argument("--workload", choices=["abmc128", "batched", "serving", "diffusion27", "poisson2d"],
                    default="abmc128",
                    help="abmc128: the headline solve (default); batched: many uneven systems with 4 "
                         "right-hand sides each, solved concurrently; serving: Poisson-arriving kNN "
                         "Laplacian solves under a device-memory budget; diffusion27: multicolor vs "
                         "ABMC B=8/16/32 on the 27-point variable-coefficient 96^3 problem; poisson2d: "
                         "plain FP64 multicolor ICCG on the 2D 5-point 128^2 Poisson problem")
    ap.add_argument("--side", type=int, default=96, help="diffusion27: grid side")
    ap.add_argument("--variant", choices=["mc", "abmc8", "abmc16", "abmc32"], default="mc",
                    help="diffusion27 with --kernel-only: the ordering of the system")
    ap.add_argument("--systems", type=int, default=512, help="batched: number of systems")
    ap.add_argument("--no-batch-tune", action="store_true",
                    help="batched: greedy multicolor for every system instead of the tuned orderings")
    ap.add_argument("--threads", type=int, default=16, help="batched / serving: concurrent solves")
    ap.add_argument("--requests", type=int, default=400, help="serving: requests per arrival rate")
    ap.add_argument("--max-points", type=int, default=1000000, help="serving: largest kNN system")
    args = ap.parse_args()
    if args.workload == "batched":
        run_batched(args)
    elif args.workload == "serving":
        run_serving(args)
    elif args.kernel_only:
        run_kernel_only(args)
    elif args.workload == "diffusion27":
        run_diffusion27(args)
    elif args.workload == "poisson2d":
        run_poisson2d(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


def _batched_matrices(count: int, seed: int = 4):
    """The batched workload's matrices: 50/50 a 2D 5-point Poisson problem
    with side U{32..256} and a 3D 7-point Laplacian with side U{16..48}."""
    import iccg_b200.problems as pb
    rng = np.random.default_rng(seed)
    mats = []
    for _ in range(count):
        if rng.random() < 0.5:
            mats.append(pb.poisson2d(int(rng.integers(32, 257))))
        else:
            mats.append(pb.laplace3d_aniso(int(rng.integers(16, 49)), 1.0))
    return mats


def _batched_problems(count: int, seed: int = 4, tune: bool = False, device: int = 0):
    """The batched workload's systems, greedy multicolor each; with `tune`
    the ordering of each class of systems (autotune.tune_batch: entries per
    row and power of two of the size) is the fastest of multicolor and ABMC
    with 8, 16 and 32-row blocks, timed on the class's largest system.
    Returns the problems and the tuner's table (None untuned)."""
    import iccg_b200.problems as pb
    mats = _batched_matrices(count, seed)
    if not tune:
        return [pb.make(A, "piccg", seed=i) for i, A in enumerate(mats)], None
    import iccg_b200.autotune as at
    probs, table = at.tune_batch(mats, seeds=list(range(count)), tol=TOL, device=device)
    return probs, [{"class": list(r["class"]), "systems": r["systems"], "tuned_on_rows": r["tuned_on_rows"],
                    "choice": r["choice"], "ms": {t["candidate"]: t["ms"] for t in r["trials"]}} for r in table]


def batched_case(count: int, nrhs: int = 4, steps: int = 3, warmup: int = 1, device: int = 0,
                 compare_streams: bool = True, sample: int = 32, tune: bool = True):
    """All count x nrhs solves of the batched workload through the batched
    engine (ib.Batch: one launch per CG step for every solve), FP32 A and L,
    FP64 vectors and reductions, tol 1e-8.  Reports solves/s from the device
    time (CUDA events) and end to end (host arrays in and out, wall clock),
    per-solve latency percentiles (batch start to the solve's stop, device
    clock), the algorithmic GB/s of the iterations, and the same solves one
    at a time (fused mixed path per system, and plain FP64) on a sample.
    `tune`: orderings per class of systems by the tuner (its time is
    reported as setup_s.tune)."""
    import iccg_b200 as ib
    t0 = time.perf_counter()
    probs, table = _batched_problems(count, tune=tune, device=device)
    tune_s = time.perf_counter() - t0
    import iccg_b200.problems as pb
    rhs = [[pb.with_rhs(P, seed=1000 * i + k).b_run.copy() for k in range(nrhs)] for i, P in enumerate(probs)]
    host_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    import iccg_b200.batch as bt
    ctxs = []
    for P in probs:
        c = bt.batch_context(device)
        c.upload(P.A_run)
        c.set_schedule(P.sched)
        c.build(ib.PRECOND_IC0, 0.0)
        ctxs.append(c)
    B = ib.Batch(device)
    for c in ctxs:
        B.add_system(c)
    upload_s = time.perf_counter() - t0
    systems = [i for i in range(count) for _ in range(nrhs)]
    bs = [rhs[i][k] for i in range(count) for k in range(nrhs)]
    t0 = time.perf_counter()
    xs = [np.zeros(len(b)) for b in bs]
    res = B.solve(systems, bs, xs, 10000, TOL, storage=ib.STORE_FP32, rr_interval=RR)
    first_s = time.perf_counter() - t0
    for _ in range(max(0, warmup - 1)):
        xs = [np.zeros(len(b)) for b in bs]
        B.solve(systems, bs, xs, 10000, TOL, storage=ib.STORE_FP32, rr_interval=RR)
    dev_ms, wall_ms, lat, l0 = [], [], [], B.launches
    for _ in range(steps):
        xs = [np.zeros(len(b)) for b in bs]
        t0 = time.perf_counter()
        res = B.solve(systems, bs, xs, 10000, TOL, storage=ib.STORE_FP32, rr_interval=RR)
        wall_ms.append((time.perf_counter() - t0) * 1e3)
        dev_ms.append(B.device_ms)
        lat.extend(r.solve_ms for r in res)
    launches = (B.launches - l0) // max(1, steps)
    ok = all(r.converged and r.true_rel_resid <= TOL for r in res)
    nsolve = len(bs)
    dms = statistics.median(dev_ms)
    wms = statistics.median(wall_ms)
    it_bytes = sum(bytes_model(probs[k], 4)["iteration"] * r.iters for k, r in zip(systems, res))
    out = {"systems": count, "rhs_per_system": nrhs, "solves": nsolve, "all_converged_1e-8": ok,
           "rows": {"min": min(P.A.n for P in probs), "max": max(P.A.n for P in probs),
                    "mean": round(statistics.mean(P.A.n for P in probs))},
           "solves_per_s": round(nsolve / (dms * 1e-3), 2),
           "e2e_solves_per_s": round(nsolve / (wms * 1e-3), 2),
           "batch_ms": {"device": round(dms, 3), "e2e": round(wms, 3)},
           "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3),
                          "p99": round(float(np.percentile(lat, 99)), 3)},
           "mean_iters": round(statistics.mean(r.iters for r in res), 1),
           "max_iters": max(r.iters for r in res),
           "iteration_GBps": round(it_bytes / (dms * 1e-3) / 1e9, 1),
           "launches_per_batch": int(launches),
           "setup_s": {"host": round(host_s, 2), "upload_and_ic0": round(upload_s, 2),
                       "first_batch_with_layouts": round(first_s, 2)},
           "steps": steps,
           "orderings": "tuned per class" if tune else "greedy multicolor"}
    if tune:
        out["setup_s"]["tune"] = round(tune_s, 2)
        out["tuning"] = table
    # the same solves one at a time: the per-system fused mixed path (its
    # own CUDA graphs) and the plain FP64 path, on a sample of the solves
    pick = list(range(0, nsolve, max(1, nsolve // sample)))
    one_mixed, one_plain = [], []
    for s in pick:
        c = ctxs[systems[s]]
        x = np.zeros(len(bs[s]))
        c.solve(bs[s], x, 10000, TOL, storage=ib.STORE_FP32, rr_interval=RR)
        x[:] = 0.0
        r = c.solve(bs[s], x, 10000, TOL, storage=ib.STORE_FP32, rr_interval=RR)
        one_mixed.append(r.solve_ms)
        x[:] = 0.0
        r = c.solve(bs[s], x, 10000, TOL, storage=ib.STORE_FP64, mode=ib.MODE_PLAIN)
        one_plain.append(r.solve_ms)
    mixed_per_s = 1000.0 / statistics.mean(one_mixed)
    plain_per_s = 1000.0 / statistics.mean(one_plain)
    out["one_at_a_time_solves_per_s"] = {"fused_mixed": round(mixed_per_s, 2), "plain_fp64": round(plain_per_s, 2),
                                         "sample": len(pick)}
    out["speedup_vs_one_at_a_time_fused_mixed"] = round(out["solves_per_s"] / mixed_per_s, 2)
    out["speedup_vs_one_at_a_time_plain_fp64"] = round(out["solves_per_s"] / plain_per_s, 2)
    B.close()
    if compare_streams:
        # the earlier form: one context and stream per system, 16 host threads
        import iccg_b200.batch as bt
        for c in ctxs:
            c.close()
        ctxs = []
        rs = [bt.ResidentSystem(P, device=device, storage=ib.STORE_FP32) for P in probs]
        bt.solve_batch(rs, [[r[0]] for r in rhs], threads=16)
        t0 = time.perf_counter()
        recs = bt.solve_batch(rs, rhs, threads=16)
        wall = time.perf_counter() - t0
        out["streams_16_threads_solves_per_s"] = round(len(recs) / wall, 2)
        for r in rs:
            r.close()
    for c in ctxs:
        c.close()
    return out


def run_batched(args):
    """Many independent SPD systems of uneven size, 4 right-hand sides each
    (--systems, default 512: 2048 solves), through the batched engine: every
    CG step of all solves is one kernel launch over a device work list, with
    per-solve CG scalars and reductions.  The comparisons are the same solves
    one at a time (the per-system fused path and the plain FP64 path) and the
    earlier many-streams form (one context and stream per system, 16 host
    threads)."""
    import torch
    torch.cuda.set_device(0)
    out = batched_case(args.systems, 4, steps=max(1, args.steps), warmup=max(1, args.warmup),
                       tune=not args.no_batch_tune)
    line = {"workload": "batched", **out,
            "storage": "fp32 A and L, fp64 vectors",
            "preconditioner": "IC(0), " + ("greedy multicolor" if args.no_batch_tune else
                                           "multicolor or ABMC per class of systems (tuned)"),
            "data": "synthetic",
            "timing": "device: CUDA events around each batch on the batch's stream (median over steps); "
                      "e2e: wall clock of Batch.solve with host arrays in and out"}
    print(json.dumps(line), flush=True)


def run_serving(args):
    """Serving: kNN-Laplacian solve requests arriving as a Poisson process.

    Each request is a symmetrised 8-nearest-neighbour graph Laplacian plus
    1e-2 I, on N points with N log-uniform in [1e3, --max-points]. It gets a
    seeded right-hand side and ABMC ICCG to 1e-8 with FP32 storage.  The
    continuous-batching loop (iccg_b200.batch.ServingLoop) admits requests by
    free device memory under a 100 GB budget, builds their systems on
    --threads builder threads and steps every running solve together in one
    batch session, retiring solves as they stop.  Each arrival rate reports
    p50 / p99 latency (arrival to result, host set-up included) and solves/s.
    The comparisons are the earlier thread-pool loop (one context and stream
    per request) at the top rate and the same requests one at a time on the
    plain FP64 path.

    Under torchrun (one process per GPU) every rank serves its share of the
    stream on its own GPU (iccg_b200.batch.serve_sharded), the arrival rates
    scale with the number of GPUs, and rank 0 prints the summary over all
    requests.
    """
    import torch
    import iccg_b200 as ib
    import iccg_b200.batch as bt
    import iccg_b200.problems as pb
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local = _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900), device_id=torch.device("cuda", local))
    rng = np.random.default_rng(5)
    lo, hi = np.log(1e3), np.log(float(args.max_points))
    sizes = [int(np.exp(rng.uniform(lo, hi))) for _ in range(args.requests * world)]
    budget = 100 * 10**9

    def make_requests(rate):
        t, reqs = 0.0, []
        arr = np.random.default_rng(int(rate * 1000) + 7)
        for i, npts in enumerate(sizes):
            t += arr.exponential(1.0 / rate)
            reqs.append(bt.Request(i, t, (lambda npts=npts, i=i: pb.config_knn(npts, seed=i)),
                                   bt.estimate_device_bytes(npts, 18 * npts)))
        return reqs

    # one request at a time, end to end (host set-up, upload, IC(0), mixed
    # solve), and the plain FP64 solve alone, on a sample
    sample = sizes[:: max(1, len(sizes) // 16)]
    alone_ms, plain_ms, bits_same = [], [], True
    B = ib.Batch(local)
    B.open(1, ib.STORE_FP32, rr_interval=RR, graph_iters=4)
    for i, npts in enumerate(sample):
        t0 = time.perf_counter()
        P = pb.config_knn(npts, seed=10_000 + i)
        c = ib.Context(local)
        bt.load_system(c, P, ib.STORE_FP32)
        x = np.zeros(P.A_run.n)
        r = c.solve(P.b_run, x, 10000, TOL, storage=ib.STORE_FP32, rr_interval=RR, graph_iters=4)
        alone_ms.append((time.perf_counter() - t0) * 1e3)
        # the same solve through a batch session: the same bits
        k = B.add_system(c)
        B.submit(k, P.b_run, None, 10000, TOL)
        while True:
            stopped, _ = B.step()
            if stopped:
                break
        xb, rb = B.retire(stopped)
        B.remove_system(k)
        bits_same = bits_same and np.array_equal(xb[0], x) and rb[0].iters == r.iters
        xp = np.zeros(P.A_run.n)
        rp = c.solve(P.b_run, xp, 10000, TOL, storage=ib.STORE_FP64, mode=ib.MODE_PLAIN)
        plain_ms.append(rp.solve_ms)
        c.close()
    B.close()
    sat = world * args.threads * 1000.0 / statistics.mean(alone_ms)
    if dist is not None:
        box = [sat]
        dist.broadcast_object_list(box, src=0)   # every rank uses rank 0's arrival rates
        sat = box[0]
    out = []
    for f in (0.25, 0.5, 1.0):
        loop = bt.ServingLoop(budget_bytes=budget, device=local, builders=args.threads, slots=1024,
                              graph_iters=4, rr_interval=RR)
        st = bt.serve_sharded(make_requests(f * sat), loop, dist=dist)
        st["arrival_rate_per_s"] = round(f * sat, 2)
        out.append(st)
    # the top rate on the thread-pool loop (one context and stream per request)
    loop = bt.ThreadedServingLoop(budget_bytes=budget, workers=args.threads, device=local)
    threaded = bt.serve_sharded(make_requests(sat), loop, dist=dist)
    threaded["arrival_rate_per_s"] = round(sat, 2)
    line = {"workload": "serving", "n_gpus": world, "requests_per_rate": len(sizes),
            "points": {"min": min(sizes), "max": max(sizes), "distribution": "log-uniform",
                       "max_points_arg": args.max_points},
            "builders_per_gpu": args.threads, "budget_bytes_per_gpu": budget,
            "admission": "free device memory (cudaMemGetInfo + idle pooled contexts - 2 GiB reserve) "
                         "and the 100 GB budget",
            "rates": out, "thread_pool_loop_at_top_rate": threaded,
            "one_at_a_time_ms": {"mixed_end_to_end_mean": round(statistics.mean(alone_ms), 3),
                                 "plain_fp64_solve_mean": round(statistics.mean(plain_ms), 3),
                                 "sample": len(sample)},
            "plain_fp64_one_at_a_time_solves_per_s": round(1000.0 / statistics.mean(plain_ms), 2),
            "batch_session_same_bits_as_alone": bool(bits_same),
            "storage": "fp32 A and L, fp64 vectors", "preconditioner": "IC(0), ABMC B=16",
            "data": "synthetic",
            "latency": "arrival to result, host set-up (kNN graph, blocking, PtAP, upload, IC(0)) included"}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_diffusion27(args):
    """Multicolor vs ABMC (B = 8, 16, 32) on a 27-point diffusion problem.

    The operator is the 27-point variable-coefficient diffusion on a
    --side^3 grid (96^3: n = 884,736, nnz = 23,393,656). Its face
    coefficients are harmonic means of exp(sigma g), where g is a smoothed
    Gaussian field; sigma is set for a 1e4 contrast. b = A x*, and
    x* ~ U(-1,1) from splitmix64(0).
    - IC(0) is factored in FP64 on the device. A non-positive pivot restarts
      it with a larger shift, and the shift used is reported.
    - Each variant is solved in FP64 and in mixed precision: FP32 A and L,
      FP64 recurrences, residual replacement every 50 iterations.
    - Reported per variant: colors, iterations and device ms per solve
      (CUDA events, mean over --steps after --warmup), plus the iteration's
      algorithmic bandwidth.
    - The reference's OpenMP CG runs once, on the ABMC B=16 system.
    """
    import torch
    import iccg_b200 as ib
    import iccg_b200.problems as pb
    side = args.side
    variants = [("mc", "piccg", 0), ("abmc8", "abmc", 8), ("abmc16", "abmc", 16), ("abmc32", "abmc", 32)]
    peak, peak_kind = _peaks()
    dev = torch.device("cuda", 0)
    out = []
    cpu = None
    for label, variant, B in variants:
        t0 = time.perf_counter()
        P = pb.config_diffusion27(side, variant, block_size=max(B, 1), seed=0)
        host_s = time.perf_counter() - t0
        n = P.A_run.n
        ctx = ib.Context(0)
        t0 = time.perf_counter()
        ctx.upload(P.A_run)
        ctx.set_schedule(P.sched)
        ctx.build(ib.PRECOND_IC0, 0.0, auto_shift=True)
        factor_s = time.perf_counter() - t0
        b_d = torch.from_numpy(P.b_run).to(dev)
        x_d = torch.zeros(n, dtype=torch.float64, device=dev)
        stream = torch.cuda.ExternalStream(ctx.stream)
        torch.cuda.synchronize()
        row = {"variant": label, "colors": P.nc, "blocks": P.nb if variant == "abmc" else None,
               "ic0_shift": ctx.shift, "setup_s": {"host": round(host_s, 2), "upload_and_ic0": round(factor_s, 2)}}
        # substitution kernel per color (counts by kind) for each storage and direction
        row["sweep_kernels"] = {}
        for st_name, storage in (("fp64", ib.STORE_FP64), ("mixed", ib.STORE_FP32)):
            for d in ("fwd", "bwd"):
                kinds = {}
                for k, _ in ctx.sweep_plan(storage, d == "fwd"):
                    kinds[k] = kinds.get(k, 0) + 1
                row["sweep_kernels"][f"{st_name}_{d}"] = kinds
        x64 = None
        for st_name, storage in (("fp64", ib.STORE_FP64), ("mixed", ib.STORE_FP32)):
            res = []
            for i in range(args.warmup + args.steps):
                with torch.cuda.stream(stream):
                    x_d.zero_()
                r = ctx.solve_dev(b_d.data_ptr(), x_d.data_ptr(), 10000, TOL, storage=storage, rr_interval=RR)
                if i >= args.warmup:
                    res.append(r)
            ms = statistics.mean(r.solve_ms for r in res)
            last = res[-1]
            bm = bytes_model(P, 8 if storage == ib.STORE_FP64 else 4)
            gbs = bm["iteration"] * last.iters / (ms * 1e-3) / 1e9
            row[st_name] = {"ms": round(ms, 3), "iters": last.iters, "converged": last.converged,
                            "true_rel_resid": last.true_rel_resid, "iteration_GBps": round(gbs, 1),
                            "frac": round(gbs / peak, 4)}
            xs = x_d.cpu().numpy().copy()
            if storage == ib.STORE_FP64:
                x64 = xs
            else:
                row[st_name]["err_vs_fp64_solution"] = float(np.linalg.norm(xs - x64) / np.linalg.norm(x64))
        if label == "abmc16" and not args.no_cpu_baseline:
            from oracle import bindings as ob
            if ob.ref() is not None:
                cores = os.cpu_count() or 1
                ob.ref().ref_set_threads(cores)
                R = ob.RefProblem(4, P.A.n, P.A.rowptr, P.A.colind, P.A.val, P.block_of_old, P.nb,
                                  P.block_color, P.nc)
                _, it, _, cv, us = R.cg(P.b_run, np.zeros(P.A.n), 10000, TOL)
                cpu = {"value": round(us / 1e3, 3), "unit": "ms", "cores": cores, "kind": "reference",
                       "iters": it, "converged": bool(cv), "sample": "1 full ABMC B=16 solve, conjugate_gradient only"}
        out.append(row)
        del b_d, x_d
        ctx.close()
        torch.cuda.synchronize()
    # the tuner's choice: the fastest ordering (mixed form) from the timings
    # above, then its kernel options by coordinate search on that system
    import iccg_b200.autotune as at
    best = min(out, key=lambda r: r["mixed"]["ms"])
    variant, B = {"mc": ("piccg", 16), "abmc8": ("abmc", 8), "abmc16": ("abmc", 16),
                  "abmc32": ("abmc", 32)}[best["variant"]]
    P = pb.config_diffusion27(side, variant, block_size=B, seed=0)
    ctx = ib.Context(0)
    ctx.upload(P.A_run)
    ctx.set_schedule(P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0, auto_shift=True)
    kt = at.tune_kernels(ctx, P.b_run, storage=ib.STORE_FP32, tol=TOL, reps=max(1, args.steps))
    ctx.close()
    tuned = {"ordering": best["variant"], "untuned_mixed_ms": best["mixed"]["ms"],
             "kernel_options": {k: v for k, v in kt.choice.items() if k != "ms"},
             "tuned_mixed_ms": round(kt.choice["ms"], 3), "trials": kt.table()}
    line = {"workload": "diffusion27", "metric": "ICCG ms to resid 1e-8 per variant", "unit": "ms",
            "higher_is_better": False, "steps": args.steps, "warmup": args.warmup,
            "config": {"grid": f"{side}^3", "stencil": "27-point", "n": side ** 3, "contrast": 1e4,
                       "coefficients": "harmonic means of exp(sigma g), g a 3-cell box-smoothed Gaussian field",
                       "tol": TOL, "rr_interval": RR, "x0": "zeros",
                       "rhs": "b = A x*, x* ~ U(-1,1) splitmix64(0)", "blocking": "bfs"},
            "peak_GBps": peak, "peak_source": peak_kind, "variants": out, "tuned": tuned,
            "dtype": "f64", "data": "synthetic"}
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def run_poisson2d(args):
    """The small multicolor case: 2D 5-point Poisson, 128 x 128 interior grid
    with Dirichlet boundaries (n = 16,384, nnz = 81,408), greedy multicolor
    IC(0), b = A x*, x* ~ U(-1,1) from splitmix64(0), x0 = 0, tolerance 1e-8.
    Everything (A, L, vectors: about 4.4 MB per iteration) stays in L2, so a
    solve is bound by launch and reduction latency, not by HBM; it is
    reported in ms.  Device ms per solve (CUDA events, mean over --steps after
    --warmup) for the FP64 paths (fused, and plain: one kernel per reference
    operation) and the mixed form, the same solve end to end through the C
    ABI with host buffers, and the reference's OpenMP CG on the host cores.
    """
    import iccg_b200 as ib
    import iccg_b200.problems as pb
    P = pb.config_small_mc(128, seed=0)
    n = P.A_run.n
    ctx = ib.Context(0)
    ctx.upload(P.A_run)
    ctx.set_schedule(P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    out = {}
    x64 = None
    for name, storage, mode in (("fp64_fused", ib.STORE_FP64, ib.MODE_FUSED),
                                ("fp64_plain", ib.STORE_FP64, ib.MODE_PLAIN),
                                ("mixed_fused", ib.STORE_FP32, ib.MODE_FUSED)):
        res, wall = [], []
        for i in range(args.warmup + args.steps):
            x = np.zeros(n)
            t0 = time.perf_counter()
            r = ctx.solve(P.b_run, x, 10000, TOL, mode=mode, storage=storage, rr_interval=RR)
            if i >= args.warmup:
                res.append(r)
                wall.append((time.perf_counter() - t0) * 1e3)
        out[name] = {"ms": round(statistics.mean(r.solve_ms for r in res), 4), "iters": res[-1].iters,
                     "true_rel_resid": res[-1].true_rel_resid,
                     "e2e_ms": round(statistics.mean(wall), 4)}
        if x64 is None:
            x64 = x.copy()
        else:
            out[name]["err_vs_fp64_solution"] = float(np.linalg.norm(x - x64) / np.linalg.norm(x64))
    ctx.close()
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import bindings as ob
        if ob.ref() is not None:
            cores = os.cpu_count() or 1
            ob.ref().ref_set_threads(cores)
            R = ob.RefProblem(3, n, P.A.rowptr, P.A.colind, P.A.val, P.color, P.nc)
            times, it = [], 0
            for _ in range(max(3, args.steps)):
                _, it, _, _, us = R.cg(P.b_run, np.zeros(n), 10000, TOL)
                times.append(us / 1e3)
            cpu = {"value": round(statistics.median(times), 4), "unit": "ms", "cores": cores, "kind": "reference",
                   "iters": it, "sample": f"{max(3, args.steps)} full solves (median), conjugate_gradient only"}
    line = {"workload": "poisson2d", "metric": "ICCG ms to resid 1e-8", "unit": "ms", "higher_is_better": False,
            "steps": args.steps, "warmup": args.warmup,
            "config": {"grid": "128^2", "stencil": "5-point", "n": n, "nnz": P.A_run.nnz, "colors": P.nc,
                       "ordering": "greedy multicolor", "tol": TOL, "x0": "zeros",
                       "rhs": "b = A x*, x* ~ U(-1,1) splitmix64(0)",
                       "l2": "L2-resident (about 4.4 MB per iteration): latency-bound, reported in ms"},
            "paths": out, "dtype": "f64", "data": "synthetic"}
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def run_kernel_only(args):
    """One operation of the hot path on the benchmark system (or, with
    --workload diffusion27, the 27-point system of --side and --variant),
    repeated."""
    import torch
    import iccg_b200 as ib
    if args.workload == "diffusion27":
        import iccg_b200.problems as pb
        variant, B = {"mc": ("piccg", 16), "abmc8": ("abmc", 8), "abmc16": ("abmc", 16),
                      "abmc32": ("abmc", 32)}[args.variant]
        P = pb.config_diffusion27(args.side, variant, block_size=B, seed=0)
    else:
        P, _ = build_problem()
    n = P.A_run.n
    ctx = ib.Context(0)
    ctx.upload(P.A_run)
    ctx.set_schedule(P.sched)
    ctx.build(ib.PRECOND_IC0, 0.0)
    ctx.set_option(ib.OPT_PERSIST, args.persist)
    dev = torch.device("cuda", 0)
    a = torch.from_numpy(ib.gen_uniform(n, 5)).to(dev)
    b = torch.zeros(n, dtype=torch.float64, device=dev)
    L = ib.lib()
    torch.cuda.synchronize()
    ms = []
    if args.kernel_only == "solve":
        # the headline solve: b = A x*, x0 = 0, mixed form
        rhs = torch.from_numpy(P.b_run).to(dev)
        storage = ib.STORE_FP32 if args.kernel_storage == "fp32" else ib.STORE_FP64
        for _ in range(args.reps):
            b.zero_()
            torch.cuda.synchronize()
            res = ctx.solve_dev(rhs.data_ptr(), b.data_ptr(), 10000, TOL, storage=storage, rr_interval=RR)
            ms.append(res.solve_ms)
        print(json.dumps({"kernel_only": "solve", "reps": args.reps, "solve_ms": ms, "iters": res.iters}))
        ctx.close()
        return
    fn = L.iccg_spmv_dev if args.kernel_only == "spmv" else L.iccg_precond_apply_dev
    for _ in range(args.reps):
        t0 = time.perf_counter()
        rc = fn(ctx.h, ib.C.c_void_p(a.data_ptr()), ib.C.c_void_p(b.data_ptr()), ib.STORE_FP32)
        ms.append((time.perf_counter() - t0) * 1e3)
        assert rc == 0, L.iccg_ctx_last_error(ctx.h)
    print(json.dumps({"kernel_only": args.kernel_only, "reps": args.reps, "host_ms": ms,
                      "sweep_plan_fp32_fwd": ctx.sweep_plan(ib.STORE_FP32, True)[:4]}))
    ctx.close()


if __name__ == "__main__":
    main()

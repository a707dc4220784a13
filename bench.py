"""Benchmark of the ERI engine: unique ERIs per second on B200.

Workload: the 24-atom split-valence molecule (8 heavy atoms with s6 s3 p3 s1 p1 shells,
16 H with s3 s1; exponents log-uniform in [0.1, 5e3], seed 1; 104 cartesian functions,
14,908,530 unique integrals, 3,454,506 shell quartets, 124.8 M primitive quartets).

A step is one plan execute: primitive-pair build, Schwarz bounds and every shell quartet,
writing the packed iindex vector into HBM.  ``value`` is the mixed-precision rate (FP32 VRR
for quartets whose Schwarz bound is below ``fp32_cutoff``) whose max abs error against the
FP64 path is reported beside it; ``fp64`` is the plain FP64 rate.  The packed output (119 MB)
fits in L2, so a 256 MB buffer is written between timed steps (outside the timed events).
``e2e`` is the same metric through the public call with host buffers (basis upload, device
path, 119 MB device-to-host copy into pinned memory).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import __graft_entry__  # noqa: E402

mi = __graft_entry__.load_package()

METRIC = "ERIs/sec on 1 B200 (mixed vs plain FP64, max err <=1e-9); serve p50/p99 ms"
UNIT = "ERI/s"
WORKLOAD = "split_valence_24 (8 heavy s6s3p3s1p1 + 16 H s3s1, seed 1, 104 cart. functions)"
CPU_SAMPLE_SECONDS = 10.0


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of this process's GPU while the timed region
    runs.  NVML is polled every millisecond from a thread, so even a timed region of a few
    milliseconds gets samples; the GPU is found by its UUID, which stays right when
    CUDA_VISIBLE_DEVICES renumbers the devices.  Without NVML, nvidia-smi is sampled every 200
    ms instead.  Reads only; no GPU setting is changed."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.nvml = None
        self.thread = None
        self.stop = False
        self.samples = []  # (sm MHz, max sm MHz, reason bits)

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def __enter__(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)

            def poll():
                while not self.stop:
                    self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), smax,
                                         nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
                    time.sleep(0.001)

            self.nvml = nv
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop = True
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.nvml is not None:
            sm = [x[0] for x in self.samples]
            reasons = {n for n, attr in self.REASONS for x in self.samples
                       if x[2] & getattr(self.nvml, attr, 0)}
            return {"sm_mhz": statistics.median(sm) if sm else None,
                    "sm_max_mhz": max(x[1] for x in self.samples) if sm else None,
                    "samples": len(sm), "source": "nvml, 1 ms", "reasons": sorted(reasons)}
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "source": "nvidia-smi, 200 ms", "reasons": sorted(reasons)}


def cpu_reference_rate(shells, threads: int, min_seconds: float):
    """The oracle's HGP driver (restatement of the reference's all_twoe_ints_chrr) over the
    whole workload on `threads` host threads, repeated until min_seconds have passed:
    (ERI/s, seconds, passes)."""
    from oracle import oracle as orc
    out = np.zeros(shells.npacked)
    t0 = time.perf_counter()
    n = passes = 0
    while True:
        n += orc.eri_packed_hgp_sample(shells, threads, 1, out)
        passes += 1
        dt = time.perf_counter() - t0
        if dt >= min_seconds or passes >= 1000:
            return n / dt, dt, passes


def run_reference(args):
    rank, world, _ = _dist()
    if rank != 0:
        return 0
    sh = mi.config1()
    threads = os.cpu_count() or 1
    cpu_reference_rate(sh, threads, 0.0)  # builds the oracle, warms caches
    for _ in range(max(args.warmup, 0)):
        cpu_reference_rate(sh, threads, 0.0)
    t0 = time.perf_counter()
    passes = 0
    for _ in range(args.steps):
        _, _, p = cpu_reference_rate(sh, threads, 0.0)
        passes += p
    wall = time.perf_counter() - t0
    value = passes * sh.npacked / wall
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "algorithm": "HGP (restated all_twoe_ints_chrr, C, OpenMP)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"one full pass over the workload per step ({sh.npacked} integrals)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def flush_l2(buf):
    buf.add_(1.0)


def run_ours(args):
    import torch
    import torch.distributed as dist
    from molints_b200 import engine as E
    from molints_b200 import flops as F

    rank, world, local = _dist()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    eng = E.Engine(local)
    eng.set_stream(stream.cuda_stream)
    sh = mi.config1()
    npacked = sh.npacked
    per_class, tot = F.workload(sh)

    out = torch.empty(npacked, dtype=torch.float64, device=dev)
    flush = torch.zeros(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    from molints_b200 import autotune
    fp32_cut, tune_table = autotune.tune_fp32_cutoff(eng, sh)
    # per class pair: HGP or Rys, and whether MIXED plans use the FP32 variant, timed on a
    # sample of the batch and serving molecules (l <= 3) at the tuned cutoff
    t_tune = time.perf_counter()
    class_table, class_timings = autotune.tune_class_methods(
        eng, [mi.config3_molecule(m) for m in range(1, 16, 2)] + [mi.config4_request(r) for r in range(4)],
        fp32_cutoff=fp32_cut)
    t_tune = time.perf_counter() - t_tune
    eng.set_class_methods(class_table)
    eng.set_stream(stream.cuda_stream)
    plan64 = eng.plan(sh, precision=E.FP64)
    planmx = eng.plan(sh, precision=E.MIXED, fp32_cutoff=fp32_cut)

    # accuracy of the mixed path against the FP64 path on the same device
    plan64.execute(out.data_ptr())
    ref = out.clone()
    planmx.execute(out.data_ptr())
    max_err = (out - ref).abs().max().item()
    mx_stats = planmx.stats()
    del ref

    def timed(plan, k):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(k)]
        for a, b in ev:
            flush_l2(flush)
            a.record(stream)
            plan.execute(out.data_ptr())
            b.record(stream)
        torch.cuda.synchronize(dev)
        return sum(a.elapsed_time(b) for a, b in ev)

    for plan in (plan64, planmx):
        timed(plan, max(args.warmup, 3))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        ms64 = timed(plan64, args.steps)
        msmx = timed(planmx, args.steps)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
        t = torch.tensor([ms64, msmx], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms64, msmx = t.tolist()
    clocks = clk.summary()
    value64 = world * args.steps * npacked / (ms64 * 1e-3)
    valuemx = world * args.steps * npacked / (msmx * 1e-3)

    # per-launch times of one FP64 execute -> dominant kernel and its roofline
    plan64.set_profiling(True)
    flush_l2(flush)
    plan64.execute(out.data_ptr())
    launches = plan64.launch_times()
    plan64.set_profiling(False)
    eri_l = [(n, ms) for n, ms in launches if n.startswith("eri_")]
    top_name, top_ms = max(eri_l, key=lambda x: x[1])
    top_flop = per_class[top_name[4:]]["flop"]
    peak_fp64 = measure_fp64_peak(dev)
    traffic = None
    tfile = ROOT / "profiles" / "dram_traffic_split_valence_24.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get("bytes_per_launch", {}).get(top_name)
    roofline = {
        "bound": "fp64", "kernel": top_name, "achieved": top_flop / (top_ms * 1e-3) / 1e12,
        "peak": peak_fp64, "unit": "TFLOP/s",
        "frac": top_flop / (top_ms * 1e-3) / 1e12 / peak_fp64,
        "traffic": traffic,
        "peak_source": "measured in this run: torch float64 8192^3 matmul (cuBLAS DGEMM), "
                       "MEASURED_PEAKS.json has no FP64 figure",
        "whole_step_tflops": tot["flop"] / (ms64 / args.steps * 1e-3) / 1e12,
        "launch_share": {n: ms for n, ms in launches},
    }

    # end to end through the public call: host basis in, pinned host vector out
    host_out = torch.empty(npacked, dtype=torch.float64, pin_memory=True).numpy()
    eng_e2e = E.Engine(local)
    eng_e2e.eri_packed(sh, precision=E.MIXED, fp32_cutoff=fp32_cut, out=host_out)
    e2e_t = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        eng_e2e.eri_packed(sh, precision=E.MIXED, fp32_cutoff=fp32_cut, out=host_out)
        e2e_t.append(time.perf_counter() - t0)
    h2d = int(sh.xyz.nbytes + sh.L.nbytes + sh.nprim.nbytes + sh.prim_off.nbytes +
              sh.expn.nbytes + sh.coef.nbytes)
    e2e = {"value": world * npacked * len(e2e_t) / sum(e2e_t), "unit": UNIT,
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": npacked * 8,
           "timing": "host wall clock around molints_eri_packed (synchronous call)"}

    batch = serving = tuned = jk = None
    parts = set(args.parts.split(","))
    if "jk" in parts:
        jk = measure_jk(eng, stream, dev, sh, plan64, flush)
    if parts & {"batch", "serve"}:
        AT = autotune
        # FP32 cutoff for l <= 3 molecules under the tuned methods (FP32 Rys tables and FP32
        # HGP VRR): the smallest of the cutoffs tuned on three serving-shaped molecules
        tunes = [AT.tune_fp32_cutoff(eng, mi.config4_request(r)) for r in (6, 1, 7)]
        fp32_cut_l3 = min(c for c, _ in tunes)
        tune_l3 = [t for _, t in tunes]
        eng.set_stream(stream.cuda_stream)
        tuned = {"seconds": t_tune,
                 "rys_classes": sorted(t for t in class_timings
                                       if class_table[AT._class_index(t)] & 3 == E.METHOD_RYS),
                 "fp32_classes": sorted(t for t in class_timings
                                        if not class_table[AT._class_index(t)] & E.CLASS_NO_FP32),
            "fp32_cutoff_l3": fp32_cut_l3, "fp32_cutoff_l3_tuning": tune_l3}
        if "batch" in parts:
            batch = measure_batch(eng, stream, dev, fp32_cut_l3, rank, world)
        if "serve" in parts:
            serving = measure_serving(local, fp32_cut_l3, args.serve_window, rank, class_table=class_table)

    cpu = None
    if rank == 0 and world == 1 and "cpu" in parts:
        r, dt, passes = cpu_reference_rate(sh, os.cpu_count() or 1, CPU_SAMPLE_SECONDS)
        cpu = {"value": r, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"{passes} full passes over the workload in {dt:.1f} s (oracle HGP, OpenMP)"}
        r1, dt1, passes1 = cpu_reference_rate(sh, 1, 3.0)
        cpu["one_core"] = {"value": r1, "unit": UNIT, "cores": 1,
                           "sample": f"{passes1} full pass(es) in {dt1:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": valuemx, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": msmx / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (FP32 VRR below the Schwarz cutoff)", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_eri_per_step": npacked,
                       "shell_quartets": tot["quartets"], "prim_quartets": tot["prim_quartets"],
                       "fp32_cutoff": fp32_cut, "fp32_quartets": mx_stats["n_fp32_quartets"],
                       "fp32_cutoff_tuning": tune_table,
                       "prim_pairs": mx_stats["n_prim_pairs"],
                       "prim_pairs_kept": mx_stats["n_prim_pairs_kept"],
                       "prim_quartets_computed": mx_stats["n_prim_quartets"],
                       "prim_cutoff": E.PRIM_CUTOFF,
                       "l2": "256 MB buffer written between timed steps",
                       "parallelism": f"replicas x{world}"},
            "max_abs_err_mixed_vs_fp64": max_err,
            "fp64": {"value": value64, "ms_per_step": ms64 / args.steps},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "batch_config3": batch,
            "serving_config4": serving,
            "jk_config1": jk,
            "class_method_tuning": tuned,
            "gpu_launches": args.steps * 2 * plan64.stats()["n_kernel_launches"],
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    plan64.close()
    planmx.close()
    eng_e2e.close()
    eng.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def measure_batch(eng, stream, dev, fp32_cut, rank, world, cap=1.5e9):
    """The 256-molecule batch (4-40 atoms, l <= 2, 4.9e10 integrals): molecules sharded over
    ranks round-robin by size, grouped into batch plans of at most `cap` doubles of output
    each (HBM holds one group's output at a time), every shell quartet of a group in one work
    queue per class pair.  Device-timed executes of all groups, FP64 and MIXED; plan creation
    (host tables, device bound pass) is timed separately."""
    import torch
    from molints_b200 import engine as E
    mols = mi.config3(256)
    order = sorted(range(len(mols)), key=lambda i: -mols[i].npacked)
    mine = order[rank::world]
    groups, cur, tot = [], [], 0
    for i in mine:
        if cur and tot + mols[i].npacked > cap:
            groups.append(cur)
            cur, tot = [], 0
        cur.append(i)
        tot += mols[i].npacked
    if cur:
        groups.append(cur)
    n_eri = sum(mols[i].npacked for i in mine)
    out = torch.empty(int(max(sum(mols[i].npacked for i in g) for g in groups)), dtype=torch.float64,
                      device=dev)
    eng.set_stream(stream.cuda_stream)
    res = {"workload": "256 molecules, seeds 3000+m, l<=2, K in {1,3,6,7}", "n_eri_this_rank": n_eri,
           "groups": len(groups), "output_cap_doubles": cap}
    for name, prec, cut in (("fp64", E.FP64, 0.0), ("mixed", E.MIXED, fp32_cut)):
        t_plan = t_exec = 0.0
        for g in groups:
            t0 = time.perf_counter()
            plan = eng.plan_batch([mols[i] for i in g], precision=prec, fp32_cutoff=cut)
            t_plan += time.perf_counter() - t0
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            plan.execute(out.data_ptr())
            b.record(stream)
            torch.cuda.synchronize(dev)
            t_exec += a.elapsed_time(b) * 1e-3
            plan.close()
        tot_eri, t_max = float(n_eri), t_exec
        if world > 1:
            import torch.distributed as dist
            v = torch.tensor([float(n_eri), t_exec], dtype=torch.float64, device=dev)
            n_t = v[:1].clone()
            dist.all_reduce(n_t, op=dist.ReduceOp.SUM)
            t_t = v[1:].clone()
            dist.all_reduce(t_t, op=dist.ReduceOp.MAX)
            tot_eri, t_max = n_t.item(), t_t.item()
        res[name] = {"value": tot_eri / t_max, "unit": UNIT, "exec_s_max_over_ranks": t_max,
                     "plan_s": t_plan}
    res["fp32_cutoff"] = fp32_cut
    # accuracy of MIXED against FP64 on a sample of the batch's molecules
    errs = []
    for i in mine[len(mine) // 2:len(mine) // 2 + 2] + mine[-2:]:
        a = eng.eri_packed(mols[i])
        b = eng.eri_packed(mols[i], precision=E.MIXED, fp32_cutoff=fp32_cut)
        errs.append(float(np.max(np.abs(a - b))))
    res["max_abs_err_mixed_vs_fp64_sample"] = max(errs)
    return res


def measure_serving(device, fp32_cut, window_s, rank, rate=200.0, nslots=8,
                    budget=150 * 10**9, class_table=None):
    """The serving stream: Poisson arrivals (mean `rate` per s over `window_s` s) of
    synthetic molecules with 20-285 cartesian functions, l <= 3 (f shells on heavy atoms
    half the time), submitted to the engine's server as they arrive.  The server admits them
    against a 150 GB HBM ledger (result vectors kept resident until released plus the pair
    tables of running plans) into `nslots` concurrent slots.  The client releases each result
    as soon as it is ready.  Latency = completion - submission (host steady clock inside the
    library); throughput = integrals / (last completion - first arrival).  FP64 and MIXED."""
    from molints_b200 import engine as E
    arrivals = mi.config4_arrivals(rate=rate, window_s=window_s)
    mols = [mi.config4_request(r) for r in range(len(arrivals))]
    out = {"workload": f"Poisson {rate:g}/s for {window_s:g} s, {len(mols)} molecules "
                       f"({min(m.nbf for m in mols)}-{max(m.nbf for m in mols)} functions, l<=3)",
           "slots": nslots, "hbm_budget_bytes": budget,
           "n_eri": int(sum(m.npacked for m in mols))}
    srv = E.Engine(device)
    try:
        if class_table:
            srv.set_class_methods(class_table)
        srv.serve_start(nslots=nslots, hbm_budget_bytes=budget)
        # warm-up: kernel attributes and the result pool, grown by the largest requests
        big = sorted(mols, key=lambda m: -m.npacked)[:4 * nslots]
        for r in [srv.submit(sh) for sh in big]:
            r.poll(-1)
            r.release()
        for name, prec, cut in (("fp64", E.FP64, 0.0), ("mixed", E.MIXED, fp32_cut)):
            pending, lat = [], []
            t0 = time.perf_counter()
            first = last = None
            k = 0
            while k < len(mols) or pending:
                now = time.perf_counter() - t0
                while k < len(mols) and arrivals[k] <= now:
                    pending.append(srv.submit(mols[k], precision=prec, fp32_cutoff=cut))
                    k += 1
                still = []
                for r in pending:
                    if r.poll(0):
                        inf = r.info()
                        lat.append(inf["t_done"] - inf["t_submit"])
                        first = inf["t_submit"] if first is None else min(first, inf["t_submit"])
                        last = inf["t_done"] if last is None else max(last, inf["t_done"])
                        r.release()
                    else:
                        still.append(r)
                pending = still
                if k < len(mols):
                    time.sleep(max(0.0, min(0.002, arrivals[k] - (time.perf_counter() - t0))))
                else:
                    time.sleep(0.001)
            lat = np.array(lat) * 1e3
            out[name] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                         "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
                         "throughput_eri_per_s": out["n_eri"] / (last - first),
                         "requests_per_s": len(mols) / (last - first), "span_s": last - first}
        # accuracy of the mixed path on a sample of the stream
        errs = []
        for sh in mols[:6]:
            a = srv.submit(sh)
            b = srv.submit(sh, precision=E.MIXED, fp32_cutoff=fp32_cut)
            a.poll(-1)
            b.poll(-1)
            errs.append(float(np.max(np.abs(a.result() - b.result()))))
            a.release()
            b.release()
        out["max_abs_err_mixed_vs_fp64_sample"] = max(errs)
        out["fp32_cutoff"] = fp32_cut
    finally:
        srv.close()
    return out


def measure_jk(eng, stream, dev, sh, plan, flush, k=5):
    """Coulomb and exchange matrices of the headline workload for a random symmetric
    density, digested in the integral kernels (molints_plan_jk: no packed vector written):
    device time per build and the rate in integrals digested per second."""
    import torch
    n = sh.nbf
    g = torch.Generator(device="cpu").manual_seed(0)
    A = torch.randn(n, n, generator=g, dtype=torch.float64)
    D = ((A + A.T) / n).to(dev)
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    plan.jk(D.data_ptr(), J.data_ptr(), K.data_ptr())
    torch.cuda.synchronize(dev)
    ts = []
    for _ in range(k):
        flush_l2(flush)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        plan.jk(D.data_ptr(), J.data_ptr(), K.data_ptr())
        b.record(stream)
        torch.cuda.synchronize(dev)
        ts.append(a.elapsed_time(b))
    ms = float(np.median(ts))
    return {"ms_per_build": ms, "eri_digested_per_s": sh.npacked / (ms * 1e-3),
            "note": "J and K (n x n) from one execute with the digestion sink; FP64 atomics"}


def measure_fp64_peak(dev) -> float:
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize(dev)
        best = max(best, 2 * 8192 ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    return best


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--serve-window", type=float, default=5.0,
                    help="seconds of Poisson arrivals in the serving measurement")
    ap.add_argument("--parts", default="batch,serve,cpu,jk",
                    help="extra measurements beside the headline workload (profiling runs "
                         "pass an empty string)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

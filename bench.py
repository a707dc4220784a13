"""Benchmark of the ERI engine: unique ERIs per second on one B200.

Headline workload: the 256-molecule batch (seeds 3000+m, m < 256; 4-40 atoms, a third heavy;
recipes alternating the split-valence s/p shells and the polarised s/p/d shells, K in
{1,3,6,7}; 15-330 cartesian functions; 49,135,675,191 unique integrals).  The molecules are
grouped into batch plans of at most 1.5e9 output doubles each (one group's packed vectors fit
in HBM at a time; the whole batch's 393 GB do not).  A step is one pass over all 256
molecules: every group's plan executed (one CUDA graph per plan) into a device output larger
than L2.

  value      MIXED: FP32 variants below the tuned fp32_cutoff where they measured faster, and
             Schwarz screening at screen_cutoff 5e-10 (each screened integral is below 5e-10
             by the Schwarz inequality); max abs error against the oracle is reported beside it
  fp64       the plain FP64 path on the same plans' molecules (no screening)
  e2e        the same metric through the public batch API from host arrays: plan creation from
             the host basis, execute, and every packed vector copied to pinned host memory
             (through a pinned ring, overlapped with the next group's compute)
  roofline   the dominant class kernel of the FP64 pass (per-launch CUDA events of a
             serialised profiling pass), against the FP64 peak measured in the same run

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --case config1|batch|fmol|req [--repeat R]   (one workload's plans, for ncu)
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
NMOL = 256
WORKLOAD = ("batch256: 256 synthetic molecules (seeds 3000+m, 4-40 atoms, l<=2, K in {1,3,6,7}, "
            "15-330 cart. functions, 4.91e10 unique integrals)")
GROUP_CAP = 1.5e9          # output doubles per batch plan
# MIXED: quartets whose Schwarz bound Qabs_P Qabs_Q is below this are written as 0, so each
# screened integral is off by less than 5e-10; with the FP32 cutoff tuned to an error of at most
# 2.5e-10, the MIXED error stays below the 1e-9 target
SCREEN_CUTOFF = 5e-10
# The CPU sample: the batch molecules among its first eight with fewer than 150 functions and
# more than 40 (m = 1, 2, 4: 130, 82 and 67 functions, both recipes, 44.6 M integrals)
CPU_SAMPLE = (1, 2, 4)
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


def cpu_reference_rate(mols, threads: int, min_seconds: float):
    """The oracle's HGP driver (the C restatement of the reference's all_twoe_ints_chrr) over
    the molecules in `mols`, whole passes on `threads` host threads, repeated until
    min_seconds have passed: (ERI/s, seconds, passes)."""
    from oracle import oracle as orc
    outs = [np.zeros(sh.npacked) for sh in mols]
    t0 = time.perf_counter()
    n = passes = 0
    while True:
        for sh, out in zip(mols, outs):
            n += orc.eri_packed_hgp_sample(sh, threads, 1, out)
        passes += 1
        dt = time.perf_counter() - t0
        if dt >= min_seconds or passes >= 1000:
            return n / dt, dt, passes


def cpu_sample():
    return [mi.config3_molecule(m) for m in CPU_SAMPLE]


def run_reference(args):
    """The reference arm: the oracle port of all_twoe_ints_chrr on the host cores, on a bounded
    sample of the headline workload (batch molecules m = 1, 2, 4), one pass per step."""
    rank, world, _ = _dist()
    if rank != 0:
        return 0
    mols = cpu_sample()
    threads = os.cpu_count() or 1
    cpu_reference_rate(mols[:1], threads, 0.0)  # builds the oracle, warms caches
    for _ in range(max(args.warmup, 0)):
        cpu_reference_rate(mols, threads, 0.0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_reference_rate(mols, threads, 0.0)
    wall = time.perf_counter() - t0
    n = sum(sh.npacked for sh in mols)
    value = args.steps * n / wall
    sample = (f"batch molecules m = {', '.join(map(str, CPU_SAMPLE))} "
              f"({', '.join(str(sh.nbf) for sh in mols)} functions, {n} integrals) per step")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_block(args, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample + "; oracle HGP restatement, OpenMP"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config_block(args, world):
    """The workload description shared by both arms."""
    return {"workload": WORKLOAD, "molecules": NMOL, "group_cap_doubles": GROUP_CAP,
            "screen_cutoff_mixed": SCREEN_CUTOFF,
            "l2": "every group's output (>= 126 MB L2) is written anew each step",
            "parallelism": f"molecules sharded over {world} rank(s)"}


def make_groups(mols, idx, cap=GROUP_CAP):
    """Molecules (indices idx, largest first) packed into groups of at most `cap` output
    doubles (a molecule larger than cap is a group of its own)."""
    order = sorted(idx, key=lambda i: -mols[i].npacked)
    groups, cur, tot = [], [], 0
    for i in order:
        if cur and tot + mols[i].npacked > cap:
            groups.append(cur)
            cur, tot = [], 0
        cur.append(i)
        tot += mols[i].npacked
    if cur:
        groups.append(cur)
    return groups


def flush_l2(buf):
    buf.add_(1.0)


def timed_steps(plans, out, stream, k):
    """k steps (every plan executed into `out`), CUDA events around each step on the launching
    stream; total ms."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(k)]
    for a, b in ev:
        a.record(stream)
        for p in plans:
            p.execute(out.data_ptr())
        b.record(stream)
    torch.cuda.synchronize(stream.device)
    return sum(a.elapsed_time(b) for a, b in ev)


def run_ours(args):
    import torch
    import torch.distributed as dist
    from molints_b200 import autotune as AT
    from molints_b200 import engine as E

    rank, world, local = _dist()
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    eng = E.Engine(local)
    eng.set_stream(stream.cuda_stream)
    parts = set(filter(None, args.parts.split(",")))

    # ---- tuning: the FP32 cutoff (every FP32 variant in use, error <= 2.5e-10 against FP64)
    # on two batch molecules (one per recipe), then each class pair's method and FP32 choice
    t_tune = time.perf_counter()
    tunes = [AT.tune_fp32_cutoff(eng, mi.config3_molecule(m), boys=E.BOYS_EXACT) for m in (2, 1)]
    fp32_cut = min(c for c, _ in tunes)
    class_table, class_timings = AT.tune_class_methods(
        eng, [mi.config3_molecule(m) for m in range(1, 16, 2)] + [mi.config4_request(r) for r in range(4)],
        fp32_cutoff=fp32_cut)
    eng.set_class_methods(class_table)
    # then the work-queue schedule (lane split, chunk lengths) with that table
    schedule, sched_trials = AT.tune_schedule(eng, [mi.config3_molecule(m) for m in range(1, 16, 2)])
    eng.set_schedule(schedule)
    eng.set_stream(stream.cuda_stream)
    t_tune = time.perf_counter() - t_tune
    tuned = {"seconds": t_tune, "fp32_cutoff": fp32_cut, "fp32_cutoff_tuning": [t for _, t in tunes],
             "rys_classes": sorted(t for t in class_timings
                                   if class_table[AT._class_index(t)] & 3 == E.METHOD_RYS),
             "fp32_classes": sorted(t for t in class_timings
                                    if not class_table[AT._class_index(t)] & E.CLASS_NO_FP32),
             "timings_ms": class_timings, "schedule": schedule,
             "schedule_trials": [[{k: v for k, v in sc.items()}, round(ms, 3)] for sc, ms in sched_trials]}

    # ---- the headline: the 256-molecule batch, molecules sharded over ranks by size
    mols = mi.config3(NMOL)
    order = sorted(range(NMOL), key=lambda i: -mols[i].npacked)
    mine = order[rank::world]
    groups = make_groups(mols, mine)
    n_eri = sum(mols[i].npacked for i in mine)
    t0 = time.perf_counter()
    plans64 = [eng.plan_batch([mols[i] for i in g], boys=E.BOYS_EXACT) for g in groups]
    t_plan64 = time.perf_counter() - t0
    t0 = time.perf_counter()
    plansmx = [eng.plan_batch([mols[i] for i in g], boys=E.BOYS_EXACT, precision=E.MIXED,
                              fp32_cutoff=fp32_cut, screen_cutoff=SCREEN_CUTOFF) for g in groups]
    t_planmx = time.perf_counter() - t0
    for p in plans64 + plansmx:
        p.set_graph(True)
    out = torch.empty(max(p.npacked for p in plans64), dtype=torch.float64, device=dev)
    for plans in (plans64, plansmx):
        timed_steps(plans, out, stream, max(args.warmup, 3))
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        ms64 = timed_steps(plans64, out, stream, args.steps)
        msmx = timed_steps(plansmx, out, stream, args.steps)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
        t = torch.tensor([ms64, msmx, float(n_eri)], dtype=torch.float64, device=dev)
        tm = t[:2].clone()
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        tn = t[2:].clone()
        dist.all_reduce(tn, op=dist.ReduceOp.SUM)
        ms64, msmx = tm.tolist()
        n_all = tn.item()
    else:
        n_all = float(n_eri)
    clocks = clk.summary()
    value64 = args.steps * n_all / (ms64 * 1e-3)
    valuemx = args.steps * n_all / (msmx * 1e-3)
    stmx = [p.stats() for p in plansmx]
    st64 = [p.stats() for p in plans64]
    launches = sum(s["n_kernel_launches"] for s in st64) + sum(s["n_kernel_launches"] for s in stmx)
    plan_ph = plan_phases(np.sum(np.array([s["plan_ms"] for s in st64]), axis=0))
    mixed_stats = {k: int(sum(s[k] for s in stmx)) for k in
                   ("n_shell_quartets", "n_fp32_quartets", "n_screened", "n_fp32_launches")}

    roofline = measure_roofline(plans64, groups, mols, out, stream, dev)
    tmx, _, _ = profile_pass(plansmx, out)
    roofline["mixed_kernel_ms_per_step"] = {n: round(t, 3) for n, t in sorted(tmx.items(), key=lambda x: -x[1])}
    e2e = measure_e2e(eng, dev, stream, mols, groups, fp32_cut, min(args.steps, args.e2e_steps))
    plain = measure_plain_fp64(eng, dev, mols, mine) if "plain" in parts else None
    for p in plans64 + plansmx:
        p.close()
    del out
    torch.cuda.empty_cache()

    errors = measure_errors(eng, fp32_cut) if "errors" in parts and rank == 0 else None
    cfg1 = measure_config1(eng, dev, stream, fp32_cut, args) if "config1" in parts else None
    jk = measure_jk(eng, stream, dev, mi.config1()) if "jk" in parts else None
    serving = None
    if "serve" in parts:
        serving = measure_serving(local, fp32_cut, args.serve_window, rank, class_table=class_table,
                                  schedule=schedule)
    cpu = None
    if rank == 0 and world == 1 and "cpu" in parts:
        smp = cpu_sample()
        r, dt, passes = cpu_reference_rate(smp, os.cpu_count() or 1, CPU_SAMPLE_SECONDS)
        cpu = {"value": r, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"{passes} passes over batch molecules m = {CPU_SAMPLE} "
                         f"({sum(s.npacked for s in smp)} integrals) in {dt:.1f} s "
                         f"(oracle HGP restatement, OpenMP)"}
        r1, dt1, passes1 = cpu_reference_rate(smp[-1:], 1, 3.0)
        cpu["one_core"] = {"value": r1, "unit": UNIT, "cores": 1,
                           "sample": f"{passes1} pass(es) over batch molecule m = {CPU_SAMPLE[-1]} in {dt1:.1f} s"}

    if rank == 0:
        cfg = config_block(args, world)
        cfg.update({"n_eri_per_step": int(n_all), "groups": len(groups), "fp32_cutoff": fp32_cut,
                    "boys": "exact", "mixed_quartets": mixed_stats,
                    "plan_create_s": {"fp64": t_plan64, "mixed": t_planmx},
                    "plan_create_phases_ms_fp64": plan_ph,
                    "cuda_graph": "one graph per batch plan"})
        line = {
            "metric": METRIC, "value": valuemx, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": msmx / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": f"f64 (FP32 VRR below the tuned cutoff where faster; Schwarz screening {SCREEN_CUTOFF:g})",
            "data": "synthetic", "config": cfg,
            "fp64": {"value": value64, "ms_per_step": ms64 / args.steps,
                     "mixed_over_fp64": valuemx / value64},
            "plain_fp64_per_molecule": plain,
            # rank 0's own molecules at N > 1: the ratio is stated for one GPU only
            "mixed_over_plain_fp64_per_molecule": (valuemx / plain["value"]
                                                   if plain is not None and world == 1 else None),
            "max_abs_err_vs_oracle": errors,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "config1": cfg1, "serving_config4": serving, "jk_config1": jk,
            "class_method_tuning": tuned,
            "gpu_launches": args.steps * launches, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def profile_pass(plans, out):
    """One serialised profiling execute of each plan: per kernel its summed device time (ms,
    per-launch CUDA events on the launching stream) and launches, and per class pair the FLOP
    of the primitive quartets its kernels evaluate."""
    from molints_b200 import flops as F
    times, nlaunch, executed = {}, {}, {}
    lv = {"s": 0, "p": 1, "d": 2, "f": 3}
    for p in plans:
        p.set_profiling(True)
        p.execute(out.data_ptr())
        for name, ms in p.launch_times():
            times[name] = times.get(name, 0.0) + ms
            nlaunch[name] = nlaunch.get(name, 0) + 1
        p.set_profiling(False)
        for tag, (nq, kq) in p.class_work().items():
            la, lb, lc, ld = (lv[c] for c in tag)
            executed[tag] = executed.get(tag, 0.0) + kq * F.per_prim_flops(la, lb, lc, ld) + \
                nq * F.hrr_flops(la, lb, lc, ld)
    return times, nlaunch, executed


def measure_roofline(plans, groups, mols, out, stream, dev):
    """One serialised profiling pass of the FP64 plans (per-launch CUDA events on the launching
    stream), per kernel its device time over the whole batch.  The dominant kernel gets the
    roofline: the gather pass of the two-phase output is HBM-bound (16 algorithmic bytes per
    packed integral: one scratch read, one output write; peak = MEASURED_PEAKS.json hbm_gbs),
    a class kernel FP64-bound (flops.py algorithmic FLOP over all primitive quartets; peak =
    FP64 DGEMM measured here).  The top class kernel is reported beside it, also against the
    FLOP of the primitive quartets it evaluates (after primitive-pair screening).  DRAM
    traffic comes from an ncu capture recorded in profiles/ when one exists for the kernel."""
    from molints_b200 import flops as F
    per_tag = {}
    for g in groups:
        for i in g:
            w, _ = F.workload(mols[i])
            for tag, d in w.items():
                per_tag[tag] = per_tag.get(tag, 0.0) + d["flop"]
    times, nlaunch, executed = profile_pass(plans, out)
    total_ms = sum(times.values())
    peak64 = measure_fp64_peak(dev)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    hbm_src = "MEASURED_PEAKS.json hbm_gbs (copy)" if "hbm_gbs" in peaks else "fallback 6.65 TB/s"
    traffic_db = {}
    tfile = ROOT / "profiles" / "dram_traffic_batch256.json"
    if tfile.exists():
        traffic_db = json.loads(tfile.read_text()).get("bytes_per_integral", {})
    n_eri = sum(p.npacked for p in plans)

    def class_entry(name):
        flop = per_tag.get(name[4:], 0.0)
        ach = flop / (times[name] * 1e-3) / 1e12
        ex = executed.get(name[4:], 0.0) / (times[name] * 1e-3) / 1e12
        return {"bound": "fp64", "kernel": name, "achieved": ach, "peak": peak64, "unit": "TFLOP/s",
                "frac": ach / peak64, "executed_tflops": ex, "executed_frac": ex / peak64,
                "launches": nlaunch[name], "kernel_ms_per_step": times[name],
                "kernel_flop_per_step": flop, "executed_flop_per_step": executed.get(name[4:], 0.0),
                "traffic": None,
                "peak_source": "measured in this run: torch float64 8192^3 matmul (cuBLAS DGEMM); "
                               "MEASURED_PEAKS.json has no FP64 figure"}
    cls = [n for n in times if n.startswith(("eri_", "rys_"))]
    top_cls = max(cls, key=times.get)
    top = max(times, key=times.get)
    if top == "gather_packed":
        ach = 16.0 * n_eri / (times[top] * 1e-3) / 1e9
        t = traffic_db.get(top)
        roof = {"bound": "hbm", "kernel": top, "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "launches": nlaunch[top], "kernel_ms_per_step": times[top],
                "algorithmic_bytes_per_step": 16.0 * n_eri,
                "traffic": None if t is None else t * n_eri / nlaunch[top], "peak_source": hbm_src}
    else:
        roof = class_entry(top)
    roof["top_class_kernel"] = class_entry(top_cls)
    roof["whole_step_tflops"] = sum(per_tag.values()) / (total_ms * 1e-3) / 1e12
    roof["serialised_ms"] = total_ms
    roof["share"] = {n: round(t / total_ms, 4) for n, t in sorted(times.items(), key=lambda x: -x[1])}
    return roof


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


def measure_e2e(eng, dev, stream, mols, groups, fp32_cut, steps, ring_doubles=32 * 2**20, ncopy=2):
    """The headline metric end to end through the public batch API: per group, the plan is
    created from the host basis arrays (normalisation, pair tables, device bound pass, work
    queues, uploads), executed, and its packed vectors are copied to pinned host memory through
    a ring of four 256 MB pinned buffers on `ncopy` copy streams taking the chunks in turn
    (overlapped with the next group's compute; two device outputs alternate).  Host wall clock
    around whole passes."""
    import torch
    from molints_b200 import engine as E
    if steps <= 0:
        return None
    cap = max(sum(mols[i].npacked for i in g) for g in groups)
    outs = [torch.empty(cap, dtype=torch.float64, device=dev) for _ in range(2)]
    ring = [torch.empty(ring_doubles, dtype=torch.float64, pin_memory=True) for _ in range(4)]
    copies = [torch.cuda.Stream(dev) for _ in range(ncopy)]
    done = [[torch.cuda.Event() for _ in range(ncopy)] for _ in range(2)]
    computed = torch.cuda.Event()
    h2d = 0
    for g in groups:
        for i in g:
            sh = mols[i]
            h2d += int(sh.xyz.nbytes + sh.L.nbytes + sh.nprim.nbytes + sh.prim_off.nbytes +
                       sh.expn.nbytes + sh.coef.nbytes)
    walls = []
    for _ in range(steps):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        chunk = 0
        for gi, g in enumerate(groups):
            buf = outs[gi % 2]
            for ev in done[gi % 2]:
                stream.wait_event(ev)  # the copies of group gi-2 have read this buffer
            plan = eng.plan_batch([mols[i] for i in g], boys=E.BOYS_EXACT, precision=E.MIXED,
                                  fp32_cutoff=fp32_cut, screen_cutoff=SCREEN_CUTOFF)
            plan.execute(buf.data_ptr())
            computed.record(stream)
            for cs in copies:
                cs.wait_event(computed)
            for off in range(0, plan.npacked, ring_doubles):
                n = min(ring_doubles, plan.npacked - off)
                with torch.cuda.stream(copies[chunk % ncopy]):
                    ring[chunk % 4][:n].copy_(buf[off:off + n], non_blocking=True)
                chunk += 1
            for k, cs in enumerate(copies):
                done[gi % 2][k].record(cs)
            plan.close()
        torch.cuda.synchronize(dev)
        walls.append(time.perf_counter() - t0)
    n = sum(mols[i].npacked for g in groups for i in g)
    return {"value": n * len(walls) / sum(walls), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": 8 * n, "steps": len(walls), "seconds_per_step": walls,
            "d2h_gbs": 8 * n / (sum(walls) / len(walls)) / 1e9,
            "timing": "host wall clock: plan creation from host arrays, execute, D2H of every "
                      "packed vector into pinned host memory (MIXED, same options as value)"}


def measure_plain_fp64(eng, dev, mols, mine):
    """The plain FP64 GPU path: the drop-in call molints_eri_packed, one molecule at a time,
    output on the device (plan creation from the host basis included), host wall clock."""
    import torch
    out = torch.empty(max(mols[i].npacked for i in mine), dtype=torch.float64, device=dev)
    eng.eri_packed_device(mols[mine[-1]], out.data_ptr())  # warm-up
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for i in mine:
        eng.eri_packed_device(mols[i], out.data_ptr())
    torch.cuda.synchronize(dev)
    dt = time.perf_counter() - t0
    n = sum(mols[i].npacked for i in mine)
    return {"value": n / dt, "unit": UNIT, "seconds": dt,
            "note": "molints_eri_packed per molecule (FP64, default options), device output, "
                    "plan creation included (host wall clock)"}


def measure_errors(eng, fp32_cut):
    """Max abs error against the oracle (the long-double restatement of the reference HGP in
    the engine's pair orientation, exact Boys function) for every config, FP64 and MIXED with
    the bench's options: configs 0-2 whole, batch molecules m = 6, 4, 2, serving requests
    31 (f shells) and 9."""
    from molints_b200 import engine as E
    from oracle import oracle as orc
    cases = [("config0", mi.config0()), ("config1", mi.config1()), ("config2", mi.config2()),
             ("config3_m6", mi.config3_molecule(6)), ("config3_m4", mi.config3_molecule(4)),
             ("config3_m2", mi.config3_molecule(2)), ("config4_r31", mi.config4_request(31)),
             ("config4_r9", mi.config4_request(9))]
    res = {}
    t0 = time.perf_counter()
    for name, sh in cases:
        with orc.exact_boys(), orc.stable_orientation():
            ld = orc.eri_packed_hgp_ld(sh, nthreads=0)
        a = eng.eri_packed(sh, boys=E.BOYS_EXACT)
        b = eng.eri_packed(sh, boys=E.BOYS_EXACT, precision=E.MIXED, fp32_cutoff=fp32_cut,
                           screen_cutoff=SCREEN_CUTOFF)
        res[name] = {"fp64": float(np.max(np.abs(a - ld))), "mixed": float(np.max(np.abs(b - ld))),
                     "nbf": sh.nbf}
    res["oracle"] = "long-double HGP restatement, engine orientation, exact Boys"
    res["seconds"] = time.perf_counter() - t0
    return res


def measure_config1(eng, dev, stream, fp32_cut, args):
    """The 24-atom split-valence molecule (104 functions, 14.9 M integrals): device-resident
    plan executes (a 256 MB buffer written between steps: the output fits in L2), FP64 and
    MIXED, and end to end through molints_eri_packed into pinned host memory."""
    import torch
    from molints_b200 import engine as E
    sh = mi.config1()
    out = torch.empty(sh.npacked, dtype=torch.float64, device=dev)
    flush = torch.zeros(256 * 2**20 // 4, dtype=torch.float32, device=dev)
    res = {"workload": "split_valence_24 (seed 1, 104 functions)", "n_eri": sh.npacked}
    for name, prec in (("fp64", E.FP64), ("mixed", E.MIXED)):
        plan = eng.plan(sh, precision=prec, fp32_cutoff=fp32_cut if prec else 0.0,
                        screen_cutoff=SCREEN_CUTOFF if prec else 0.0)
        ts = []
        for k in range(args.warmup + args.steps):
            flush_l2(flush)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            plan.execute(out.data_ptr())
            b.record(stream)
            torch.cuda.synchronize(dev)
            if k >= args.warmup:
                ts.append(a.elapsed_time(b))
        plan.close()
        res[name] = {"value": sh.npacked / (np.mean(ts) * 1e-3), "ms": float(np.mean(ts))}
    host = torch.empty(sh.npacked, dtype=torch.float64, pin_memory=True).numpy()
    e = E.Engine(dev.index)
    e.eri_packed(sh, out=host)
    ts, phases = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e.eri_packed(sh, out=host)
        ts.append(time.perf_counter() - t0)
    for _ in range(args.steps):  # the phases, from calls outside the timed ones
        _, st = e.eri_packed(sh, out=host, with_stats=True)
        phases.append(st["plan_ms"] + [st["device_ms"]])
    e.close()
    ph = np.mean(np.array(phases), axis=0)
    res["e2e_fp64"] = {"value": sh.npacked / np.mean(ts), "ms": 1e3 * float(np.mean(ts)),
                       "timing": "host wall clock around molints_eri_packed (host output)",
                       "plan_ms": plan_phases(ph), "execute_ms": ph[4]}
    return res


def plan_phases(ph):
    """molints_stats.plan_ms by name."""
    return {"host_tables": ph[0], "device_build": ph[1], "queue_emit": ph[2], "finish": ph[3]}


def measure_serving(device, fp32_cut, window_s, rank, rate=200.0, nslots=8,
                    budget=150 * 10**9, class_table=None, schedule=None):
    """The serving stream: Poisson arrivals (mean `rate` per s over `window_s` s) of
    synthetic molecules with 20-285 cartesian functions, l <= 3 (f shells on heavy atoms
    half the time), submitted to the engine's server as they arrive.  The server admits them
    against a 150 GB HBM ledger (result vectors kept resident until released plus the pair
    tables of running plans) into `nslots` concurrent slots.  The client releases each result
    as soon as it is ready.  Latency = completion - submission (host steady clock inside the
    library), split into queue wait (admission - submission) and service (completion -
    admission), also by request-size decile; throughput = integrals / (last completion - first
    arrival).  FP64 and MIXED."""
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
        if schedule:
            srv.set_schedule(schedule)
        srv.serve_start(nslots=nslots, hbm_budget_bytes=budget)
        # warm-up: kernel attributes and the result pool, grown by the largest requests
        big = sorted(mols, key=lambda m: -m.npacked)[:4 * nslots]
        for r in [srv.submit(sh) for sh in big]:
            r.poll(-1)
            r.release()
        for name, prec, cut in (("fp64", E.FP64, 0.0), ("mixed", E.MIXED, fp32_cut)):
            pending, rec = [], []
            t0 = time.perf_counter()
            k = 0
            while k < len(mols) or pending:
                now = time.perf_counter() - t0
                while k < len(mols) and arrivals[k] <= now:
                    scut = SCREEN_CUTOFF if prec == E.MIXED else 0.0
                    pending.append((k, srv.submit(mols[k], precision=prec, fp32_cutoff=cut,
                                                  screen_cutoff=scut)))
                    k += 1
                still = []
                for i, r in pending:
                    if r.poll(0):
                        inf = r.info()
                        rec.append((mols[i].npacked, inf["t_submit"], inf["t_admit"], inf["t_done"]))
                        r.release()
                    else:
                        still.append((i, r))
                pending = still
                if k < len(mols):
                    time.sleep(max(0.0, min(0.002, arrivals[k] - (time.perf_counter() - t0))))
                else:
                    time.sleep(0.001)
            a = np.array(rec)
            lat, wait, serv = (a[:, 3] - a[:, 1]) * 1e3, (a[:, 2] - a[:, 1]) * 1e3, (a[:, 3] - a[:, 2]) * 1e3
            span = a[:, 3].max() - a[:, 1].min()
            dec = np.argsort(np.argsort(a[:, 0])) * 10 // len(a)
            out[name] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                         "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
                         "queue_wait_p50_ms": float(np.percentile(wait, 50)),
                         "queue_wait_p99_ms": float(np.percentile(wait, 99)),
                         "service_p50_ms": float(np.percentile(serv, 50)),
                         "service_p99_ms": float(np.percentile(serv, 99)),
                         "by_size_decile": [{"decile": d, "p50_ms": float(np.percentile(lat[dec == d], 50)),
                                             "p99_ms": float(np.percentile(lat[dec == d], 99)),
                                             "wait_p50_ms": float(np.percentile(wait[dec == d], 50)),
                                             "service_p50_ms": float(np.percentile(serv[dec == d], 50))}
                                            for d in range(10) if (dec == d).any()],
                         "throughput_eri_per_s": out["n_eri"] / span,
                         "requests_per_s": len(mols) / span, "span_s": float(span)}
        # accuracy of the mixed path on a sample of the stream
        errs = []
        for sh in mols[:6]:
            a = srv.submit(sh)
            b = srv.submit(sh, precision=E.MIXED, fp32_cutoff=fp32_cut, screen_cutoff=SCREEN_CUTOFF)
            a.poll(-1)
            b.poll(-1)
            errs.append(float(np.max(np.abs(a.result() - b.result()))))
            a.release()
            b.release()
        out["max_abs_err_mixed_vs_fp64_sample"] = max(errs)
        out["fp32_cutoff"] = fp32_cut
        out["screen_cutoff_mixed"] = SCREEN_CUTOFF
    finally:
        srv.close()
    return out


def measure_jk(eng, stream, dev, sh, k=5):
    """Coulomb and exchange matrices of the 24-atom molecule for a random symmetric density,
    digested in the integral kernels (molints_plan_jk: no packed vector written): device time
    per build and the rate in integrals digested per second."""
    import torch
    plan = eng.plan(sh)
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
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        plan.jk(D.data_ptr(), J.data_ptr(), K.data_ptr())
        b.record(stream)
        torch.cuda.synchronize(dev)
        ts.append(a.elapsed_time(b))
    plan.close()
    ms = float(np.median(ts))
    return {"ms_per_build": ms, "eri_digested_per_s": sh.npacked / (ms * 1e-3),
            "note": "J and K (n x n) from one execute with the digestion sink; FP64 atomics"}


def run_case(args):
    """One workload's plan executed --repeat times on cuda:0, the device time of each execute
    printed: the command the ncu captures in profiles/ run.  Cases: config0, config1, config2
    (the benchmark molecules), batch (a batch plan over the molecules --mols of the
    256-molecule batch), fmol (polarised heavy atoms with an f shell, and hydrogens: --nheavy,
    --nh, --seed), req (request --seed of the serving stream)."""
    import torch
    from molints_b200 import engine as E
    if args.case == "fmol":
        mols = [mi.basis.synthetic_molecule(args.seed, args.nheavy, args.nh, mi.basis.POLARISED_C,
                                            mi.basis.POLARISED_H, 0.1, 1e4, "fmol", heavy_extra=[(3, 1)])]
    elif args.case == "req":
        mols = [mi.config4_request(args.seed)]
    elif args.case == "batch":
        mols = [mi.config3_molecule(int(m)) for m in args.mols.split(",")]
    else:
        mols = [getattr(mi, args.case)()]
    method = {"auto": E.METHOD_AUTO, "hgp": E.METHOD_HGP, "rys": E.METHOD_RYS}[args.method]
    eng = E.Engine(0)
    stream = torch.cuda.current_stream()
    eng.set_stream(stream.cuda_stream)
    mixed = args.mixed > 0 or args.screen > 0
    plan = eng.plan_batch(mols, method=method, precision=E.MIXED if mixed else E.FP64,
                          fp32_cutoff=args.mixed, screen_cutoff=args.screen, boys=E.BOYS_EXACT)
    out = torch.empty(max(plan.npacked, 1), dtype=torch.float64, device="cuda")
    for k in range(args.repeat):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        plan.execute(out.data_ptr())
        e.record(stream)
        torch.cuda.synchronize()
        print(f"{args.case} nbf={[m.nbf for m in mols]} execute {k}: {s.elapsed_time(e):.3f} ms", flush=True)
    plan.close()
    eng.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=2,
                    help="passes of the end-to-end measurement (each copies every packed vector "
                         "to host memory)")
    ap.add_argument("--serve-window", type=float, default=30.0,
                    help="seconds of Poisson arrivals in the serving measurement")
    ap.add_argument("--parts", default="errors,plain,config1,serve,cpu,jk",
                    help="measurements beside the headline (profiling runs pass an empty string)")
    ap.add_argument("--case", default=None,
                    choices=["config0", "config1", "config2", "batch", "fmol", "req"],
                    help="run one workload's plan (for ncu) instead of the benchmark")
    ap.add_argument("--mols", default="0,1,2")
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--nheavy", type=int, default=8)
    ap.add_argument("--nh", type=int, default=16)
    ap.add_argument("--method", default="auto", choices=["auto", "hgp", "rys"])
    ap.add_argument("--mixed", type=float, default=0.0, help="FP32 cutoff of --case (0: plain FP64)")
    ap.add_argument("--screen", type=float, default=0.0, help="quartet screening cutoff of --case (0: none)")
    ap.add_argument("--repeat", type=int, default=3)
    args = ap.parse_args()
    if args.case:
        return run_case(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

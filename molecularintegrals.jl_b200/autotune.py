"""Autotuning: the mixed-precision cutoff, the per-class method table and the work-queue
schedule.

``tune_fp32_cutoff`` runs the FP64 path once and the MIXED path over a ladder of cutoffs on
the device, and returns the largest cutoff whose max abs error against FP64 stays below
``target * safety``.  The cutoff compares against R_ab * R_cd, the bound of the VRR output
block (see molints_options.fp32_cutoff), so the error is close to eps_fp32 * R_ab R_cd and a
single basis calibrates the ladder well; ``safety`` keeps a margin for other bases.
"""
from __future__ import annotations

import numpy as np

# Cutoffs tried, up to 1e-2: the FP32 error is about eps_fp32 R_ab R_cd (eps_fp32 = 6e-8), so
# larger cutoffs cannot keep a 1e-9 target in general even where one molecule happens to.
LADDER = tuple(10.0 ** k for k in range(-6, -1))


def tune_fp32_cutoff(engine, shells, target: float = 1e-9, safety: float = 0.25,
                     ladder=LADDER, boys=None, method=None):
    import torch
    from . import engine as E
    boys = E.BOYS_REFERENCE if boys is None else boys
    method = E.METHOD_AUTO if method is None else method
    dev = torch.device("cuda", engine.device)
    ref = torch.empty(shells.npacked, dtype=torch.float64, device=dev)
    out = torch.empty_like(ref)
    stream = torch.cuda.current_stream(dev)
    engine.set_stream(stream.cuda_stream)
    # the error is measured with every class pair's FP32 variant in use (the table's
    # "FP32 no faster" flags cleared); the context's table is restored afterwards
    saved = engine.class_methods()
    engine.set_class_methods({k: v & ~E.CLASS_NO_FP32 for k, v in saved.items()})
    try:
        p64 = engine.plan(shells, precision=E.FP64, boys=boys, method=method)
        p64.execute(ref.data_ptr())
        p64.close()
        table = []
        best = 0.0
        for c in sorted(ladder):
            pm = engine.plan(shells, precision=E.MIXED, boys=boys, fp32_cutoff=c, method=method)
            pm.execute(out.data_ptr())
            st = pm.stats()
            pm.close()
            err = (out - ref).abs().max().item() if shells.npacked else 0.0
            frac = st["n_fp32_quartets"] / max(st["n_shell_quartets"], 1)
            table.append({"cutoff": c, "max_abs_err": err, "fp32_quartet_fraction": frac,
                          "fp32_launches": st["n_fp32_launches"]})
            if err <= target * safety:
                best = c
            else:
                break
        return best, table
    finally:
        engine.set_class_methods(saved)
        engine.set_stream(None)


def _class_index(tag: str):
    """'ddps' -> (bra pair-class index, ket pair-class index) in the engine's order."""
    from . import engine as E
    lv = {"s": 0, "p": 1, "d": 2, "f": 3}
    bra = (lv[tag[0]], lv[tag[1]])
    ket = (lv[tag[2]], lv[tag[3]])
    return E.PAIR_CLASSES.index(bra), E.PAIR_CLASSES.index(ket)


def tune_class_methods(engine, molecules, repeats: int = 3, margin: float = 0.95,
                       fp32_cutoff: float | None = None):
    """Per class pair, HGP or Rys, whichever kernel is faster on `molecules` (one batch plan
    per method; each launch timed alone with CUDA events in profiling mode, best of
    `repeats`).  Rys is taken only where it is faster by `margin`.  With `fp32_cutoff`, the
    MIXED kernels of the chosen method are timed too, and classes whose FP32 variant is not
    faster get the MOLINTS_CLASS_NO_FP32 flag (MIXED plans then run their FP64 kernel).
    Returns (table, timings): table[(x, y)] for engine.set_class_methods; timings maps the class
    tag to (HGP ms, Rys ms[, mixed ms of the chosen method]).  Classes with an f shell and no
    HGP kernel have only Rys and are listed only for the FP32 decision."""
    import torch
    from . import engine as E
    mols = list(molecules)
    dev = torch.device("cuda", engine.device)
    n = sum(m.npacked for m in mols)
    out = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    engine.set_stream(stream.cuda_stream)
    best = {}
    runs = [(E.METHOD_HGP, E.FP64), (E.METHOD_RYS, E.FP64)]
    if fp32_cutoff:
        runs += [(E.METHOD_HGP, E.MIXED), (E.METHOD_RYS, E.MIXED)]
    # every FP32 variant runs while its time is measured; the table is restored afterwards
    saved = engine.class_methods()
    engine.set_class_methods({k: v & ~E.CLASS_NO_FP32 for k, v in saved.items()})
    try:
        for meth, prec in runs:
            plan = engine.plan_batch(mols, method=meth, boys=E.BOYS_EXACT, precision=prec,
                                     fp32_cutoff=fp32_cutoff or 0.0)
            plan.set_profiling(True)
            for _ in range(repeats):
                plan.execute(out.data_ptr())
                for name, ms in plan.launch_times():
                    if name.startswith("eri_") or name.startswith("rys_"):
                        key = (name[4:], name[:3], prec)
                        best[key] = min(best.get(key, float("inf")), ms)
            plan.close()
    finally:
        engine.set_class_methods(saved)
        engine.set_stream(None)
    table, timings = {}, {}
    for tag in sorted({k[0] for k in best}):
        h = best.get((tag, "eri", E.FP64))
        r = best.get((tag, "rys", E.FP64))
        if h is not None and r is not None:
            meth = E.METHOD_RYS if r < margin * h else E.METHOD_HGP
        elif h is not None:
            meth = E.METHOD_HGP
        else:
            meth = E.METHOD_RYS
        entry = meth
        t = (h, r)
        if fp32_cutoff:
            fam = "eri" if meth == E.METHOD_HGP else "rys"
            m64, mmx = best.get((tag, fam, E.FP64)), best.get((tag, fam, E.MIXED))
            if m64 is not None and mmx is not None:
                t = (h, r, mmx)
                if not mmx < margin * m64:
                    entry |= E.CLASS_NO_FP32
        timings[tag] = t
        table[_class_index(tag)] = entry
    return table, timings


# Values tried per schedule knob (molints_schedule), in the order the knobs are tuned.
# hgp_widen is left out: on the batch it moves the time by under 1 %, within the noise the
# tuner picks from, while wider chunks cost small molecules (the 24-atom split-valence molecule:
# 0.43 -> 0.57 ms at 4)
SCHEDULE_GRID = (
    ("lane_cost", (40.0, 80.0, 160.0, 320.0, 640.0, 1280.0)),
    ("rys_chunks", (1024, 4096, 16384)),
    ("rys_max_width", (4, 8, 16)),
    ("gather_blocks", (3, 4, 5, 6, 8)),
)


def tune_schedule(engine, molecules, repeats: int = 3, margin: float = 0.99, precision=None,
                  grid=SCHEDULE_GRID):
    """The work-queue schedule (engine.set_schedule) that runs a batch plan over `molecules`
    fastest: one pass of coordinate descent over `grid` from the context's current schedule,
    each knob set to the value with the shortest execute (CUDA events around the whole
    execute, median of `repeats` after one warm-up) while the others keep their best values so
    far; a value replaces the current one only when faster by `margin`.  The context's
    schedule is restored.  Returns (best, trials) with trials = [(schedule, ms), ...]."""
    import torch
    from . import engine as E
    mols = list(molecules)
    dev = torch.device("cuda", engine.device)
    out = torch.empty(max(sum(m.npacked for m in mols), 1), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    prec = E.FP64 if precision is None else precision
    saved = engine.schedule()
    trials = []

    def run(sched):
        engine.set_schedule(sched)
        plan = engine.plan_batch(mols, boys=E.BOYS_EXACT, precision=prec)
        try:
            plan.execute(out.data_ptr())
            ts = []
            for _ in range(repeats):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                plan.execute(out.data_ptr())
                b.record(stream)
                b.synchronize()
                ts.append(a.elapsed_time(b))
        finally:
            plan.close()
        ms = float(np.median(ts))
        trials.append((dict(sched), ms))
        return ms

    engine.set_stream(stream.cuda_stream)
    try:
        best = dict(saved)
        best_ms = run(best)
        for key, values in grid:
            for v in values:
                if v == best[key]:
                    continue
                cand = dict(best, **{key: v})
                ms = run(cand)
                if ms < margin * best_ms:
                    best, best_ms = cand, ms
    finally:
        engine.set_schedule(saved)
        engine.set_stream(None)
    return best, trials


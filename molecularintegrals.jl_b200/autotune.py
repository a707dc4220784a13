"""Autotuning of the mixed-precision cutoff.

``tune_fp32_cutoff`` runs the FP64 path once and the MIXED path over a ladder of cutoffs on
the device, and returns the largest cutoff whose max abs error against FP64 stays below
``target * safety``.  The cutoff compares against R_ab * R_cd, the bound of the VRR output
block (see molints_options.fp32_cutoff), so the error is close to eps_fp32 * R_ab R_cd and a
single basis calibrates the ladder well; ``safety`` keeps a margin for other bases.
"""
from __future__ import annotations

import numpy as np

LADDER = tuple(10.0 ** k for k in range(-6, 5))


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
            table.append({"cutoff": c, "max_abs_err": err, "fp32_quartet_fraction": frac})
            if err <= target * safety:
                best = c
            else:
                break
        return best, table
    finally:
        engine.set_stream(None)


def _class_index(tag: str):
    """'ddps' -> (bra pair-class index, ket pair-class index) in the engine's order."""
    from . import engine as E
    lv = {"s": 0, "p": 1, "d": 2, "f": 3}
    bra = (lv[tag[0]], lv[tag[1]])
    ket = (lv[tag[2]], lv[tag[3]])
    return E.PAIR_CLASSES.index(bra), E.PAIR_CLASSES.index(ket)


def tune_class_methods(engine, molecules, repeats: int = 3, margin: float = 0.95):
    """Per class pair, HGP or Rys, whichever kernel is faster on `molecules` (one batch plan
    per method; each launch timed alone with CUDA events in profiling mode, best of
    `repeats`).  Rys is taken only where it is faster by `margin`.  Returns (table, timings):
    table[(x, y)] = METHOD_HGP or METHOD_RYS for engine.set_class_methods; timings maps the
    class tag to (HGP ms, Rys ms).  Classes with an f shell have only Rys and are not listed."""
    import torch
    from . import engine as E
    mols = list(molecules)
    dev = torch.device("cuda", engine.device)
    n = sum(m.npacked for m in mols)
    out = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    engine.set_stream(stream.cuda_stream)
    best = {}
    try:
        for meth, prefix in ((E.METHOD_HGP, "eri_"), (E.METHOD_RYS, "rys_")):
            plan = engine.plan_batch(mols, method=meth, boys=E.BOYS_EXACT)
            plan.set_profiling(True)
            for _ in range(repeats):
                plan.execute(out.data_ptr())
                for name, ms in plan.launch_times():
                    if name.startswith(prefix):
                        key = (name[4:], meth)
                        best[key] = min(best.get(key, float("inf")), ms)
            plan.close()
    finally:
        engine.set_stream(None)
    table, timings = {}, {}
    for (tag, meth), ms in best.items():
        if meth != E.METHOD_HGP or (tag, E.METHOD_RYS) not in best:
            continue
        rys = best[(tag, E.METHOD_RYS)]
        timings[tag] = (ms, rys)
        table[_class_index(tag)] = E.METHOD_RYS if rys < margin * ms else E.METHOD_HGP
    return table, timings

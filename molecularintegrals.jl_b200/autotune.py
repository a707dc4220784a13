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
                     ladder=LADDER, boys=None):
    import torch
    from . import engine as E
    boys = E.BOYS_REFERENCE if boys is None else boys
    dev = torch.device("cuda", engine.device)
    ref = torch.empty(shells.npacked, dtype=torch.float64, device=dev)
    out = torch.empty_like(ref)
    stream = torch.cuda.current_stream(dev)
    engine.set_stream(stream.cuda_stream)
    try:
        p64 = engine.plan(shells, precision=E.FP64, boys=boys)
        p64.execute(ref.data_ptr())
        p64.close()
        table = []
        best = 0.0
        for c in sorted(ladder):
            pm = engine.plan(shells, precision=E.MIXED, boys=boys, fp32_cutoff=c)
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

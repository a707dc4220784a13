"""Run one workload's plan a few times on cuda:0 and print the device time per execute: the
command profiles and quick timings run (e.g. under ncu with -k on one class kernel).

    python molecularintegrals.jl_b200/run_case.py --case fmol --nheavy 8 --nh 16 --repeat 3

Cases: config0, config1, config2 (the benchmark molecules), fmol (a serving-shaped molecule:
polarised heavy atoms carrying an f shell, and hydrogens, seed --seed), req (serving request
--seed of the serving stream).
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="config1", choices=["config0", "config1", "config2", "fmol", "req"])
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--nheavy", type=int, default=8)
    ap.add_argument("--nh", type=int, default=16)
    ap.add_argument("--method", default="auto", choices=["auto", "hgp", "rys"])
    ap.add_argument("--mixed", type=float, default=0.0, help="FP32 cutoff (0: plain FP64)")
    ap.add_argument("--repeat", type=int, default=3)
    a = ap.parse_args()
    sys.path.insert(0, str(ROOT))
    import __graft_entry__
    mi = __graft_entry__.load_package()
    import torch
    from molints_b200 import engine as E
    if a.case == "fmol":
        sh = mi.basis.synthetic_molecule(a.seed, a.nheavy, a.nh, mi.basis.POLARISED_C, mi.basis.POLARISED_H,
                                         0.1, 1e4, "fmol", heavy_extra=[(3, 1)])
    elif a.case == "req":
        sh = mi.config4_request(a.seed)
    else:
        sh = getattr(mi, a.case)()
    method = {"auto": E.METHOD_AUTO, "hgp": E.METHOD_HGP, "rys": E.METHOD_RYS}[a.method]
    eng = E.Engine(0)
    stream = torch.cuda.current_stream()
    eng.set_stream(stream.cuda_stream)
    plan = eng.plan(sh, method=method, precision=E.MIXED if a.mixed > 0 else E.FP64, fp32_cutoff=a.mixed)
    out = torch.empty(max(sh.npacked, 1), dtype=torch.float64, device="cuda")
    for k in range(a.repeat):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        plan.execute(out.data_ptr())
        e.record(stream)
        torch.cuda.synchronize()
        print(f"{a.case} nbf={sh.nbf} execute {k}: {s.elapsed_time(e):.3f} ms", flush=True)
    plan.close()
    eng.close()


if __name__ == "__main__":
    main()

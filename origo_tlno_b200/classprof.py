"""Per-class statistics and timings of the direct J/K build.

Plans a synthetic workload and, for every quartet class combination (or the
selected ones), prints one JSON line: surviving contracted and primitive
quartets, the flop model, the kernel (compile-time or warp-per-quartet) and
the CUDA-event time of one class launch in FP64, FP32 and without J/K
digestion.  With --once it only launches the selected classes one time each
(a target for a profiler run).

    python -m origo_tlno_b200.classprof cfg4 --classes "10|00" --once
    python -m origo_tlno_b200.classprof water60 --reps 3 --fp32
    python -m origo_tlno_b200.classprof water200 --onee
"""
from __future__ import annotations

import argparse
import json
import time

from . import engine as E
from . import molecules as M


def workload(name: str):
    """Molecule and Schwarz threshold of a named synthetic workload."""
    if name.startswith("water"):
        return M.water_cluster(int(name[5:]), seed=5), 1e-11
    mol = getattr(M, name)()
    return mol, (1e-11 if name == "cfg4" else 1e-12)


def tag(c) -> str:
    return f"{c['la']}{c['lb']}|{c['lc']}{c['ld']}"


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("workload", help="cfg0..cfg4 or waterN")
    ap.add_argument("--classes", default="", help='comma-separated class tags such as "10|00,11|10"')
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--fp32", action="store_true", help="also time the FP32 kernel of each class (with --once: launch only the FP32 kernel)")
    ap.add_argument("--eri-only", action="store_true", help="also time the class without J/K digestion")
    ap.add_argument("--once", action="store_true", help="launch each selected class once, no timing loop")
    ap.add_argument("--plan-only", action="store_true")
    ap.add_argument("--onee", action="store_true", help="only build S, T, V once (the one-electron kernel)")
    ap.add_argument("--jk-mixed", action="store_true",
                    help="only run one mixed-precision J/K build of the workload's standard density")
    ap.add_argument("--force-generic", default="",
                    help='comma-separated class tags run by the generic kernel even when compiled, such as "21|11"')
    ap.add_argument("--generic-warps", type=int, default=0,
                    help="0: block-per-quartet generic kernel; 1..8: warp-per-quartet kernel with that many warps")
    a = ap.parse_args(argv)

    mol, tau = workload(a.workload)
    t0 = time.time()
    ctx = E.Context(mol)
    for t in (t.strip() for t in a.force_generic.split(",")):
        if t:
            la, lb, lc, ld = int(t[0]), int(t[1]), int(t[3]), int(t[4])
            X, Y = la * (la + 1) // 2 + lb, lc * (lc + 1) // 2 + ld
            ctx.set_combo_generic(X * 15 + Y, True)
    ctx.plan(E.ScreeningOptions(integral_threshold=tau))
    if a.generic_warps:
        ctx.set_tuning(generic_warps=a.generic_warps)
    prof = ctx.profile()
    prof["plan_s"] = time.time() - t0
    prof["workload"] = a.workload
    print(json.dumps(prof), flush=True)
    if a.onee or a.jk_mixed:
        t0 = time.time()
        if a.onee:
            ctx.onee()
            if not a.once:
                import torch
                from . import _native as N
                bufs = [torch.empty(mol.n_sph, mol.n_sph, dtype=torch.float64, device="cuda") for _ in range(3)]
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                st = torch.cuda.ExternalStream(ctx.stream())
                ms = []
                for _ in range(a.reps + 1):
                    ev[0].record(st)
                    N.check(N.lib().tlno_gpu_onee(ctx.h, bufs[0].data_ptr(), bufs[1].data_ptr(), bufs[2].data_ptr(),
                                                  1, N.DEVICE_PTRS))
                    ev[1].record(st)
                    torch.cuda.synchronize()
                    ms.append(ev[0].elapsed_time(ev[1]))
                print(json.dumps({"onee_gpu_ms": min(ms[1:]), "M": mol.n_sph, "nuclei": int(len(mol.charges))}),
                      flush=True)
        else:
            # water clusters: 5 occupied orbitals per water, as cfg4
            dens = (M.density_for(a.workload, mol) if a.workload in M.N_OCC
                    else M.random_density(mol.n_sph, mol.n_sph * 5 // 24, seed=105))
            ctx.jk(dens, mixed=True)
        print(json.dumps({"onee" if a.onee else "jk_mixed": "done", "host_s": time.time() - t0}), flush=True)
        ctx.close()
        return 0
    want = {t.strip() for t in a.classes.split(",") if t.strip()}
    for i, c in enumerate(ctx.combos()):
        if want and tag(c) not in want:
            continue
        row = {"index": i, "class": tag(c), "kernel": "compile-time" if c["fast"] else "warp-per-quartet",
               "tiles": c["n_tiles"], "quartets": c["quartets"], "prim_quartets": c["prim_quartets"],
               "flops_model": c["flops"]}
        if not a.plan_only:
            reps = 0 if a.once else a.reps
            if a.once and a.fp32:  # launch the FP32 kernel only
                row["ms_fp32"] = ctx.time_combo(i, fp32=True, reps=0)
                print(json.dumps(row), flush=True)
                continue
            ms = ctx.time_combo(i, reps=reps)
            row["ms_fp64"] = ms
            if not a.once:
                row["tflops_model"] = c["flops"] / (ms * 1e-3) / 1e12
                if a.eri_only:
                    row["ms_fp64_eri_only"] = ctx.time_combo(i, reps=a.reps, want_j=False, want_k=False)
                if a.fp32:
                    row["ms_fp32"] = ctx.time_combo(i, fp32=True, reps=a.reps)
        print(json.dumps(row), flush=True)
    ctx.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

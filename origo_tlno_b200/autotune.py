"""Autotuner of the mixed-precision split threshold.

The mixed path evaluates a quartet in FP32 when Q_ab Q_cd max|D| falls
below the split threshold and accumulates every J/K element in FP64.  A
larger threshold sends more quartets to FP32 (faster) and moves J/K further
from the FP64 build.  `tune_mixed_threshold` builds J/K once in FP64 and once
per candidate threshold (largest first) on a density that lives on the
device, and keeps the largest threshold whose errors stay within the given
tolerances:

    |dE| = |tr(D (dJ - dK/2))| <= tol_energy,
    max|dJ| <= tol_jk and max|dK| <= tol_jk.

Every build runs through the library's stream with CUDA-event timing; the
density, J and K buffers are torch CUDA tensors (device plumbing only).
"""
from __future__ import annotations

from typing import Iterable, Optional

# Largest first; the search stops at the first candidate inside the
# tolerances, so a molecule whose FP32 error budget is generous pays one trial.
DEFAULT_CANDIDATES = (1e-1, 3e-2, 1e-2, 3e-3, 1e-3, 3e-4, 1e-4, 3e-5, 1e-5, 1e-6, 1e-7, 1e-8, 1e-9)


def _build(ctx, D, J, K, mixed: bool) -> float:
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream(), device=D.device)
    torch.cuda.synchronize(D.device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), mixed=mixed)
    e1.record(stream)
    torch.cuda.synchronize(D.device)
    return e0.elapsed_time(e1)


def tune_mixed_threshold(ctx, D, candidates: Iterable[float] = DEFAULT_CANDIDATES, tol_energy: float = 1e-7,
                         tol_jk: float = 1e-8, reference: Optional[tuple] = None) -> dict:
    """Chooses the split threshold for `ctx` (a planned engine.Context) on the
    device density `D` (M x M float64 CUDA tensor).  `reference` may hold an
    FP64 (J, K) already built from D.  Sets the chosen threshold on the
    context and returns {"threshold", "trials": [...], "fp64_ms"}."""
    import torch
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    fp64_ms = None
    if reference is None:
        fp64_ms = _build(ctx, D, J, K, mixed=False)
        J0, K0 = J.clone(), K.clone()
    else:
        J0, K0 = reference
    trials = []
    chosen = None
    for thr in sorted(set(float(c) for c in candidates), reverse=True):
        ctx.set_mixed_threshold(thr)
        ms = _build(ctx, D, J, K, mixed=True)
        dJ = (J - J0).abs().max().item()
        dK = (K - K0).abs().max().item()
        dE = abs(torch.sum(D * ((J - J0) - 0.5 * (K - K0))).item())
        ok = dE <= tol_energy and dJ <= tol_jk and dK <= tol_jk
        trials.append({"threshold": thr, "ms": ms, "abs_dE": dE, "max_abs_dJ": dJ, "max_abs_dK": dK, "ok": ok})
        if ok:
            chosen = thr
            break
    if chosen is None:
        chosen = min(float(c) for c in candidates)
    ctx.set_mixed_threshold(chosen)
    return {"threshold": chosen, "trials": trials, "fp64_ms": fp64_ms,
            "tolerances": {"abs_dE": tol_energy, "max_abs_dJK": tol_jk}}


# 0.0 keeps a class in FP64 (one launch, no FP32 pass): the starting point
# of every class, left only where an FP32 split saves time.
CLASS_CANDIDATES = (0.0, 1e-1, 1e-2, 1e-3, 1e-4, 1e-5, 1e-6)


def _class_jk(ctx, i, D, J, K, mixed):
    import ctypes as C
    from . import _native as N
    ms = C.c_double()
    N.check(N.lib().tlno_gpu_class_jk(ctx.h, i, D.data_ptr(), J.data_ptr(), K.data_ptr(),
                                      N.MIXED if mixed else 0, C.byref(ms)))
    return ms.value


def _set_class(ctx, i, scale, chunk):
    from . import _native as N
    N.check(N.lib().tlno_gpu_set_class_tuning(ctx.h, i, scale, chunk))


def allocate_budget(rows, tol_energy: float, tol_jk: float):
    """Greedy allocation of the accuracy budget over classes.

    `rows`: per class {"trials": [{"ms", "max_abs_dJ", "max_abs_dK",
    "abs_dE"}, ...] ordered by increasing split threshold, "pick": index}.
    Every class starts at its pick (the first trial: the class in FP64);
    the step with the largest time saved per unit of budget used is taken
    while the summed per-class errors stay within the tolerances.  Sets each
    row's "pick" and returns the summed (max|dJ|, max|dK|, |dE|)."""
    def used(r, k):
        tr = r["trials"][k]
        return tr["max_abs_dJ"], tr["max_abs_dK"], tr["abs_dE"]
    sJ = sum(used(r, r["pick"])[0] for r in rows)
    sK = sum(used(r, r["pick"])[1] for r in rows)
    sE = sum(used(r, r["pick"])[2] for r in rows)
    while True:
        best = None
        for r in rows:
            k = r["pick"]
            for k2 in range(k + 1, len(r["trials"])):
                a, b = used(r, k), used(r, k2)
                nJ, nK, nE = sJ - a[0] + b[0], sK - a[1] + b[1], sE - a[2] + b[2]
                if nJ > tol_jk or nK > tol_jk or nE > tol_energy:
                    break
                gain = r["trials"][k]["ms"] - r["trials"][k2]["ms"]
                cost = max((b[0] - a[0]) / tol_jk, (b[1] - a[1]) / tol_jk, (b[2] - a[2]) / tol_energy, 1e-12)
                score = gain / cost
                if gain > 0 and (best is None or score > best[0]):
                    best = (score, r, k2, nJ, nK, nE)
        if best is None:
            break
        _, r, k2, sJ, sK, sE = best
        r["pick"] = k2
    return sJ, sK, sE


def tune_classes(ctx, D, tol_energy: float = 1e-7, tol_jk: float = 1e-8,
                 candidates: Iterable[float] = CLASS_CANDIDATES, chunks: Iterable[int] = ()) -> dict:
    """Per-class autotuner of the mixed path on the device density `D`.

    Split threshold per class: every class c is built alone at every
    candidate threshold t, in FP64 and mixed (tlno_gpu_class_jk), giving its
    error e_c(t) = (max|dJ_c|, max|dK_c|, |dE_c|) and its kernel time.  J, K
    and E are sums over classes, so sum_c e_c bounds the build's error; a
    greedy allocation starts every class at the smallest candidate (0: the
    class stays FP64, one launch) and keeps
    raising the threshold of the class with the largest time saved per unit
    of budget used while the summed errors stay within the tolerances.  The
    thresholds become per-class multipliers of a unit global threshold.

    Tile chunk per class (optional, `chunks`): the compile-time kernel's tiles
    per fetch of its dynamic schedule, the one with the smallest FP64 + FP32
    launch time.

    Returns {"classes": [...], "predicted": {...}}."""
    import torch
    cands = sorted(set(float(c) for c in candidates))
    combos = ctx.combos()
    live = [i for i, c in enumerate(combos) if c["n_tiles"] > 0]
    J64, K64 = torch.empty_like(D), torch.empty_like(D)
    J, K = torch.empty_like(D), torch.empty_like(D)
    ctx.set_mixed_threshold(1.0)
    rows = []
    for i in live:
        chunk = 0
        if chunks and combos[i]["fast"]:
            best = None
            for ch in chunks:
                _set_class(ctx, i, 1.0, ch)
                t = ctx.time_combo(i, fp32=False, reps=1) + ctx.time_combo(i, fp32=True, reps=1)
                if best is None or t < best[0]:
                    best = (t, ch)
            chunk = best[1]
        _set_class(ctx, i, cands[0], chunk)
        t64 = _class_jk(ctx, i, D, J64, K64, mixed=False)
        trials = []
        for t in cands:
            _set_class(ctx, i, t, chunk)
            ms = _class_jk(ctx, i, D, J, K, mixed=True)
            dJ = (J - J64).abs().max().item()
            dK = (K - K64).abs().max().item()
            dE = abs(torch.sum(D * ((J - J64) - 0.5 * (K - K64))).item())
            trials.append({"threshold": t, "ms": ms, "max_abs_dJ": dJ, "max_abs_dK": dK, "abs_dE": dE})
        rows.append({"index": i, "class": f"{combos[i]['la']}{combos[i]['lb']}|{combos[i]['lc']}{combos[i]['ld']}",
                     "chunk": chunk, "fp64_ms": t64, "trials": trials, "pick": 0})
    sJ, sK, sE = allocate_budget(rows, tol_energy, tol_jk)
    total = 0.0
    for r in rows:
        tr = r["trials"][r["pick"]]
        _set_class(ctx, r["index"], tr["threshold"], r["chunk"])
        r["threshold"] = tr["threshold"]
        total += tr["ms"]
    return {"classes": [{k: v for k, v in r.items() if k != "trials" and k != "pick"} for r in rows],
            "candidates": cands,
            "predicted": {"sum_max_abs_dJ": sJ, "sum_max_abs_dK": sK, "sum_abs_dE": sE, "class_ms": total},
            "tolerances": {"abs_dE": tol_energy, "max_abs_dJK": tol_jk}}

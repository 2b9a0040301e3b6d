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

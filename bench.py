#!/usr/bin/env python
"""Benchmark of the B200 integral engine: Schwarz-screened direct J/K builds.

One step = one complete J/K build (Coulomb J and exchange K, D in HBM ->
J, K in HBM) of the selected synthetic workload, through the library's
CUDA-graph replay of the whole build.  Default workload: cfg4, the
400-water SCF-like sequence (M = 9600, Schwarz 1e-11), where step k uses
D_k with D_{k+1} = D_k + 1e-3 C_k C_k^T.

Printed JSON (one line, rank 0):
  metric/value   ERI quartets/s of the mixed-precision build (surviving
                 unique contracted shell quartets / build time), all GPUs;
  jk_builds_per_s, fp64 {...}: builds/s and the plain-FP64 figures;
  accuracy       |dE| (E = tr(D (J - K/2))), max|dJ|, max|dK| of the mixed
                 build against the FP64 build on the last density;
  roofline       dominant ERI kernel of the mixed step (the FP32 launch of
                 the class that takes longest): algorithmic flops (flop
                 model in origo_tlno_b200/csrc/plan.cpp) per launch /
                 CUDA-event launch time, against the measured FP32 FMA peak;
                 the FP64 launch of the same class beside it against the
                 measured FP64 FMA peak;
  e2e            the same build through the host-buffer C-ABI call
                 (H2D of D, D2H of J and K inside the timed region);
  cpu_baseline   the reference engine (oracle/_ref, compiled from its
                 sources) timed on a bounded sample on one core, on both
                 of its x86 build routes (AVX2 and AVX-512); the faster is
                 the value, both are recorded.
`--impl reference` times the reference's CPU J+K on a bounded sample of the
workload instead and prints the same metric.  Multi-GPU: every rank runs
an independent replica (the J/K build of one molecule is not sharded), so
value = sum over ranks and scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from origo_tlno_b200 import molecules as MOL  # noqa: E402

METRIC = "ERI quartets/s"
UNIT = "quartets/s"
# Accuracy budget of the mixed path against the FP64 build: |dE| <= 1e-6 Eh,
# max|dJ|, max|dK| <= 1e-7; the split-threshold autotuner keeps a 3x margin.
TOL_ENERGY = 1e-6
TOL_JK = 1e-7


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _workload(name):
    if name == "cfg4":
        mol = MOL.cfg4()
        return mol, 1e-11, 2000, "cfg4: 400-water cluster, def2-SVP-like basis, M=9600, Schwarz 1e-11"
    if name == "cfg1":
        mol = MOL.cfg1()
        return mol, 1e-12, 45, "cfg1: 24 atoms, M=246, Schwarz 1e-12"
    if name == "cfg2":
        mol = MOL.cfg2()
        return mol, 1e-12, 130, "cfg2: 60 atoms up to f, M=1480, Schwarz 1e-12"
    if name.startswith("water"):
        n = int(name[5:])
        mol = MOL.water_cluster(n, seed=5)
        return mol, 1e-11, max(1, 5 * n), f"{name}: {n}-water cluster, def2-SVP-like basis, Schwarz 1e-11"
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._p = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                        "--format=csv,noheader,nounits", "-lms", "200"],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self._p = None
        return self

    def _read(self):
        for line in self._p.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self._p:
            self._p.terminate()
            try:
                self._p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._p.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for n, v in zip(names, r[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(self.rows[0][2]) if self.rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def _cpu_count():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _reference_sample(name, seconds_target=15.0):
    """Times the reference CPU J+K on a bounded sample of the workload.
    Returns (quartets/s, sample description, kind)."""
    sys.path.insert(0, ROOT)
    from origo_tlno_b200 import engine as E
    from oracle import ref
    if name in ("cfg4",) or name.startswith("water"):
        sample_mol = MOL.water_cluster(40, seed=5)
        tau = 1e-11
        desc = "40-water sub-cluster of the cfg4 recipe (M=960), Schwarz 1e-11, one J+K build"
    elif name == "cfg2":
        sample_mol = MOL.cfg2_fragment()
        tau = 1e-12
        desc = "three-atom fragment of cfg2 with its f shells (M=74) as the bounded sample, one J+K build"
    else:
        sample_mol, tau, _, _ = _workload(name)
        desc = f"{name} whole molecule, one J+K build"
    D = MOL.random_density(sample_mol.n_sph, max(1, sample_mol.n_sph // 5), seed=77)
    rb = ref.RefBasis(sample_mol)
    t = rb.time_jk(D, schwarz=tau, reps=1)
    secs = float(t[0])
    return secs, desc, sample_mol, tau


ROUTES = {"avx2": "AVX2 (-march=x86-64-v3), the reference's legacy tuned route",
          "avx512": "AVX-512 (-march=x86-64-v4), the reference's native W8 route"}


def _route_sample(name, route):
    """One bounded reference sample on a reference build route: in this
    process when it runs that route, else in a child process (one route per
    process).  Returns (seconds, description, molecule, Schwarz threshold)."""
    from oracle import ref
    if route == ref.ROUTE:
        return _reference_sample(name)
    env = dict(os.environ, TLNO_REF_ROUTE=route)
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-sample", "--config", name],
                       env=env, capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        raise RuntimeError(f"{route} sample failed: {r.stderr.strip()[-300:]}")
    out = json.loads(r.stdout.strip().splitlines()[-1])
    secs, desc, mol, tau = out["secs"], out["desc"], None, None
    return secs, desc, mol, tau


def _routes_baseline(name):
    """The reference J+K sample on both of its x86 build routes; the faster
    route is the baseline, both are recorded."""
    from oracle import ref
    res = {}
    mol = tau = desc = None
    for route in ("avx2", "avx512"):
        lib_ok = os.path.exists(os.path.join(ROOT, "oracle", "_ref",
                                             "libtlno_ref.so" if route == "avx2" else "libtlno_ref_avx512.so"))
        if not lib_ok:
            res[route] = {"unavailable": "not built"}
            continue
        try:
            secs, d, m, t = _route_sample(name, route)
            res[route] = {"seconds": secs}
            desc = desc or d
            if m is not None:
                mol, tau = m, t
        except Exception as e:
            res[route] = {"unavailable": str(e)[:200]}
    if mol is None:
        _, _, mol, tau = _reference_sample(name) if ref.available() else (None, None, None, None)
    timed = {r: v["seconds"] for r, v in res.items() if "seconds" in v}
    if not timed:
        raise RuntimeError(f"no reference route could be timed: {res}")
    best = min(timed, key=timed.get)
    return timed[best], best, res, desc, mol, tau


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtlno_ref.so not built"}))
        return 0
    # quartet counts of the sample come from the same screening rule; they are
    # computed with the GPU plan when a device exists, else by the restated
    # count below.
    times = []
    desc = None
    q = None
    routes = None
    for i in range(args.warmup + args.steps):
        secs, best, routes, desc, mol, tau = _routes_baseline(args.config)
        if q is None:
            q = _count_quartets(mol, tau)
        if i >= args.warmup:
            times.append(secs)
    t = float(np.median(times))
    v = q / t
    out = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": args.config, "sample": desc},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference", "sample": desc,
                            "route": ROUTES[best], "routes_last_step_s": routes, "host": _host_cpu()},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def _count_quartets(mol, tau):
    """Unique contracted shell quartets with Q_ab Q_cd >= tau, from the
    reference's own Schwarz bounds (oracle/_ref)."""
    from oracle import ref
    rb = ref.RefBasis(mol)
    Q = rb.schwarz()
    Q = np.sort(Q)[::-1]
    # pairs (p >= q) with Q_p Q_q >= tau
    total = 0
    n = len(Q)
    for i in range(n):
        lo, hi = 0, i + 1
        # count j <= i with Q[j] * Q[i] >= tau (Q sorted descending, j < i has larger Q)
        while lo < hi:
            mid = (lo + hi) // 2
            if Q[i] * Q[mid] >= tau:
                lo = mid + 1
            else:
                hi = mid
        total += lo
    return total


def _profiled_traffic(workload, tag):
    """DRAM bytes per launch of class `tag` on `workload` from the committed
    ncu summary (profiles/dram_traffic.json): the FP32 kernel's entry
    ("(10|00) fp32") when there is one, else the FP64 kernel's.  Returns
    (bytes or None, which entry)."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(path) as f:
            table = json.load(f)
    except (OSError, ValueError):
        return None, None
    for key in (tag + " fp32", tag):
        v = table.get(workload, {}).get(key)
        if v is not None:
            return float(v), key
    return None, None


def _host_cpu():
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "logical_cores": os.cpu_count(), "cores_usable": _cpu_count()}


def _incremental_leg(ctx, Ds, tau, J64, K64):
    """The density sequence through the incremental state: time per update
    (host wall clock around each update call, which ends with the device work
    done) and the final G against the full FP64 build of the last density."""
    import torch
    from origo_tlno_b200 import engine as E
    interval = len(Ds)  # one exact build, then dP builds only
    st = E.Incremental(ctx, E.ScreeningOptions(integral_threshold=tau), exact_rebuild_interval=interval,
                       delta_density_threshold=tau)
    times, statuses = [], []
    for D in Ds:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        statuses.append(st.update_device(D.data_ptr()))
        times.append(time.perf_counter() - t0)
    G = torch.tensor(st.g(), device=Ds[-1].device)
    G64 = J64 - 0.5 * K64
    info = st.info()
    st.close()
    inc = [t for t, s in zip(times, statuses) if s == "incremental_update"]
    exa = [t for t, s in zip(times, statuses) if s == "exact_rebuild"]
    return {"updates": len(Ds), "exact_rebuilds": info["exact_rebuilds"],
            "incremental_updates": info["incremental_updates"],
            "ms_per_incremental_update": 1e3 * float(np.mean(inc)) if inc else None,
            "ms_per_exact_rebuild": 1e3 * float(np.mean(exa)) if exa else None,
            "ms_total": 1e3 * float(np.sum(times)),
            "delta_density_threshold": tau, "exact_rebuild_interval": interval,
            "final_max_abs_dG_vs_full_fp64": float((G - G64).abs().max().item()),
            "final_abs_dE_vs_full_fp64": abs(float(torch.sum(Ds[-1] * (G - G64)).item()))}


def _checksum_leg(ctx, quartets):
    """ERI-only throughput: the checksum stream over the plan (no J/K)."""
    ctx.eri_checksum()  # warm-up
    cs, ms = ctx.eri_checksum()
    return {"checksum": cs, "ms": ms, "value": quartets / (ms * 1e-3), "unit": UNIT,
            "note": "sum of the canonical unique spherical ERIs of the plan (build_eri_packed_for_G_rys)"}


def _onee_leg(ctx, mol, with_cpu):
    """One-electron S, T, V: GPU time of the workload (device buffers,
    CUDA events) and the reference on a bounded sample with every core."""
    import torch
    from origo_tlno_b200 import _native as N
    dev = torch.device("cuda", ctx.device)
    M = ctx.M
    bufs = [torch.empty(M, M, dtype=torch.float64, device=dev) for _ in range(3)]
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    run = lambda: N.check(N.lib().tlno_gpu_onee(ctx.h, bufs[0].data_ptr(), bufs[1].data_ptr(), bufs[2].data_ptr(),
                                                1, N.DEVICE_PTRS))
    run()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            run()
        e1.record(stream)
    torch.cuda.synchronize()
    out = {"gpu_ms": e0.elapsed_time(e1) / 3, "M": M, "nuclei": int(len(mol.charges))}
    if with_cpu:
        try:
            from oracle import ref
            sample = MOL.water_cluster(40, seed=5)
            rb = ref.RefBasis(sample)
            ref.set_threads(_cpu_count())
            t0 = time.perf_counter()
            rb.onee(screening=True)
            out["cpu_baseline"] = {"ms": 1e3 * (time.perf_counter() - t0), "cores": _cpu_count(),
                                   "kind": "reference", "sample": "40-water sub-cluster (M=960), S+T+V"}
            gctx = E_context(sample)
            gctx.onee()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            gctx.onee()
            out["gpu_ms_same_sample_host_call"] = 1e3 * (time.perf_counter() - t0)
            gctx.close()
        except Exception as e:  # the reference oracle may be absent
            out["cpu_baseline"] = {"unavailable": str(e)}
    return out


def E_context(mol):
    from origo_tlno_b200 import engine as E
    return E.Context(mol)


def run_batch(args):
    """cfg3: 256 molecules (3-30 atoms, cfg1 basis recipe) in one batch --
    one launch per quartet class over all molecules, the whole build one CUDA
    graph.  Step = one batched J/K build (FP64 and mixed); the same molecules
    built one context at a time (one graph each) are timed beside it."""
    import torch
    from origo_tlno_b200 import engine as E

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mols = MOL.cfg3(256)
    opts = E.ScreeningOptions(integral_threshold=1e-12, mixed_threshold=args.mixed_threshold)
    ctxs = [E.Context(m, device=local) for m in mols]
    batch = E.Batch(ctxs, opts)
    if args.streams > 1:
        batch.set_tuning(streams=args.streams)
    prof = batch.profile()
    Ds = [torch.tensor(MOL.random_density(m.n_sph, max(1, m.n_sph // 5), seed=100 + i)) for i, m in enumerate(mols)]
    D = torch.cat([d.ravel() for d in Ds]).to(dev)
    J = torch.empty_like(D)
    K = torch.empty_like(D)

    # the stacked matrices fit in L2: a 256 MB write between timed builds
    # evicts them
    flush = torch.empty(32 << 20, dtype=torch.float64, device=dev)

    def timed(launch, stream_handle, n):
        stream = torch.cuda.ExternalStream(stream_handle, device=dev)
        ev = []
        with torch.cuda.stream(stream):
            for _ in range(n):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                launch()
                e1.record(stream)
                ev.append((e0, e1))
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in ev]

    nd = args.warmup + args.steps
    out = {}
    sampler = ClockSampler(local)
    for mixed in (False, True):
        batch.graph_capture(D.data_ptr(), J.data_ptr(), K.data_ptr(), mixed=mixed)
        if not mixed:
            with sampler:
                ms = timed(batch.graph_launch, batch.stream(), nd)[args.warmup:]
        else:
            ms = timed(batch.graph_launch, batch.stream(), nd)[args.warmup:]
        out[mixed] = (float(np.sum(ms)) / 1e3, J.clone(), K.clone())
    t64, J64, K64 = out[False]
    tmx, Jmx, Kmx = out[True]
    # end to end through the host-buffer batch call (H2D of the stacked
    # densities, D2H of J and K), FP64
    Dh = [d.numpy() for d in Ds]
    e2e_t = []
    for _ in range(3):
        t0 = time.time()
        Jh, Kh = batch.jk(Dh, mixed=False)
        e2e_t.append(time.time() - t0)
    e2e_s = float(np.median(e2e_t[1:]))
    # reference CPU engine on a bounded sample: the first molecules of the
    # batch, one J+K build each, one core
    cpu = None
    if not args.no_cpu_baseline:
        try:
            from oracle import ref
            secs = 0.0
            qs = 0
            n = 0
            for i, m in enumerate(mols):
                if secs > 10.0:
                    break
                rb = ref.RefBasis(m)
                secs += float(rb.time_jk(Ds[i].numpy(), schwarz=1e-12, reps=1)[0])
                qs += _count_quartets(m, 1e-12)
                n += 1
            cpu = {"value": qs / secs, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"the first {n} molecules of the batch, one J+K build each ({qs} quartets, {secs:.2f} s)",
                   "host": _host_cpu(), "route": ROUTES[ref.ROUTE]}
        except Exception as e:  # the reference oracle may be absent
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"unavailable: {e}"}
    # one context (and one graph) per molecule, back to back
    seq = 0.0
    for i, c in enumerate(ctxs):
        c.plan(opts)
        Di = Ds[i].to(dev)
        Ji = torch.empty_like(Di)
        Ki = torch.empty_like(Di)
        c.graph_capture(Di.data_ptr(), Ji.data_ptr(), Ki.data_ptr(), mixed=False)
        seq += min(timed(c.graph_launch, c.stream(), 2)) / 1e3
    q = prof["quartets"]
    # The batch has no per-class split tuning: at the safe fixed split the
    # mixed build is not faster here, so the headline is the FP64 batch and
    # the mixed one is reported beside it.
    res = {"metric": METRIC, "value": q * args.steps / t64, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * t64 / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic",
           "config": {"workload": "cfg3", "description": "256 molecules of 3-30 atoms in one batch, Schwarz 1e-12",
                      "l2": "L2 flushed between timed builds (256 MB write)",
                      "molecules": len(mols), "functions_total": prof["M"], "quartets_per_build": q,
                      "streams": args.streams},
           "mixed": {"value": q * args.steps / tmx, "unit": UNIT, "ms_per_step": 1e3 * tmx / args.steps,
                     "mixed_threshold": args.mixed_threshold,
                     "accuracy": {"max_abs_dJ": float((Jmx - J64).abs().max()),
                                  "max_abs_dK": float((Kmx - K64).abs().max())}},
           "one_context_per_molecule_fp64_ms": 1e3 * seq,
           "batched_speedup_vs_one_context_per_molecule": seq / (t64 / args.steps),
           "e2e": {"value": q / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(sum(d.nbytes for d in Dh)),
                   "d2h_bytes_per_step": int(sum(a.nbytes for a in Jh) + sum(a.nbytes for a in Kh))},
           # per build: one launch per class combination over all molecules
           # and the two symmetrisations
           "gpu_launches": (prof["n_class_launches"] + 2) * args.steps,
           "roofline": None,
           "clocks": sampler.summary(),
           "cpu_baseline": cpu}
    if rank == 0:
        print(json.dumps(res))
    return 0


def run_native(args):
    import torch
    from origo_tlno_b200 import engine as E

    ws, rank, local = _dist()
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mol, tau, n_occ, wdesc = _workload(args.config)
    M = mol.n_sph
    ctx = E.Context(mol, device=local).plan(E.ScreeningOptions(integral_threshold=tau,
                                                               mixed_threshold=args.mixed_threshold))
    if args.streams > 1:
        ctx.set_tuning(streams=args.streams)
    prof = ctx.profile()
    quartets = prof["quartets"]

    # SCF-like density sequence on the device: D_{k+1} = D_k + 1e-3 C_k C_k^T.
    nd = args.warmup + args.steps
    g = torch.Generator(device="cpu").manual_seed(1000)
    C0 = (torch.randn(M, n_occ, generator=g, dtype=torch.float64) / np.sqrt(M)).to(dev)
    Ds = [C0 @ C0.T]
    for k in range(1, nd):
        Ck = (torch.randn(M, n_occ, generator=g, dtype=torch.float64) / np.sqrt(M)).to(dev)
        Ds.append(Ds[-1] + 1e-3 * (Ck @ Ck.T))
    for D in Ds:
        D.copy_(0.5 * (D + D.T))
    d_in = torch.empty(M, M, dtype=torch.float64, device=dev)
    J = torch.empty(M, M, dtype=torch.float64, device=dev)
    K = torch.empty(M, M, dtype=torch.float64, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)

    # inputs smaller than L2 (126 MB): a 256 MB write between timed builds
    # evicts them, so every build starts from HBM
    flush = torch.empty(32 << 20, dtype=torch.float64, device=dev) if M * M * 8 * 3 <= 126e6 else None

    def timed_sequence(mixed):
        ctx.graph_capture(d_in.data_ptr(), J.data_ptr(), K.data_ptr(), mixed=mixed)
        torch.cuda.synchronize()
        ev = []
        # NVTX range: lets a profiler select the launches of this sequence
        torch.cuda.nvtx.range_push("jk_mixed" if mixed else "jk_fp64")
        with torch.cuda.stream(stream):
            for k in range(nd):
                d_in.copy_(Ds[k])
                if flush is not None:
                    flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ctx.graph_launch()
                e1.record(stream)
                ev.append((e0, e1))
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        ms = [a.elapsed_time(b) for a, b in ev[args.warmup:]]
        return ms

    # FP64 sequence first (also the accuracy reference for the last density)
    ms64 = timed_sequence(False)
    J64, K64 = J.clone(), K.clone()
    # split threshold of the mixed path, per class: autotuned on the last
    # density, the summed per-class errors 3x inside the accuracy targets
    tune = None
    if not args.no_autotune:
        from origo_tlno_b200.autotune import tune_classes
        t0 = time.time()
        tune = tune_classes(ctx, Ds[-1], tol_energy=TOL_ENERGY / 3, tol_jk=TOL_JK / 3)
        tune["tuning_s"] = time.time() - t0
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    with sampler:
        t_wall0 = time.time()
        msmx = timed_sequence(True)
        t_wall = time.time() - t_wall0
    Dl = Ds[-1]
    dE = float(torch.sum(Dl * ((J - 0.5 * K) - (J64 - 0.5 * K64))).item())
    dJ = float((J - J64).abs().max().item())
    dK = float((K - K64).abs().max().item())
    t64 = float(np.sum(ms64)) / 1e3
    tmx = float(np.sum(msmx)) / 1e3
    if ws > 1:
        import torch.distributed as dist
        tt = torch.tensor([t64, tmx], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t64, tmx = float(tt[0]), float(tt[1])
    steps = args.steps
    value = ws * quartets * steps / tmx
    value64 = ws * quartets * steps / t64

    # end to end: host D (pinned) -> C-ABI host call -> host J, K
    Dh = Ds[-1].cpu().numpy()
    e2e_times = []
    for r in range(max(2, min(3, args.steps))):
        t0 = time.time()
        # the density contract is checked on every call, as the reference does
        out = ctx.jk(Dh, want=("J", "K"), mixed=True, validate=True)
        e2e_times.append(time.time() - t0)
    e2e_t = float(np.median(e2e_times[1:] if len(e2e_times) > 1 else e2e_times))
    e2e = {"value": ws * quartets / e2e_t, "unit": UNIT, "h2d_bytes_per_step": int(Dh.nbytes),
           "d2h_bytes_per_step": int(out["J"].nbytes + out["K"].nbytes)}

    # Roofline of the dominant kernel of the timed (mixed) step: at the
    # autotuned split most quartets run in the FP32 kernels, so the class
    # whose FP32 launch over all its quartets takes longest is the dominant
    # one; its FP64 launch is reported beside it.
    combos = ctx.combos()
    timings = []
    for i, cb in enumerate(combos):
        if cb["n_tiles"] == 0:
            continue
        t = ctx.time_combo(i, fp32=True, reps=1)
        timings.append((t, i, cb))
    timings.sort(key=lambda x: -x[0])
    tdom, idom, cdom = timings[0]
    tdom64 = ctx.time_combo(idom, fp32=False, reps=1)
    peak = E.fma_peak_tflops(True, device=local)
    peak64 = E.fma_peak_tflops(False, device=local)
    achieved = cdom["flops"] / (tdom * 1e-3) / 1e12
    achieved64 = cdom["flops"] / (tdom64 * 1e-3) / 1e12
    dom_tag = f"({cdom['la']}{cdom['lb']}|{cdom['lc']}{cdom['ld']})"
    traffic, traffic_key = _profiled_traffic(args.config, dom_tag)
    # kernels per build: one per class combination and precision pass, the
    # max|D| reduction (mixed) and the two final symmetrisations
    n_cls = sum(1 for cb in combos if cb["n_tiles"] > 0)
    launches = 2 * n_cls + 3

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            secs, best, routes, desc, smol, stau = _routes_baseline(args.config)
            q = _count_quartets(smol, stau)
            cpu = {"value": q / secs, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": desc + f" ({q} quartets, {secs:.2f} s)", "host": _host_cpu(),
                   "route": ROUTES[best] + " (the faster of its two x86 routes); its G/K endpoints refuse more "
                            "than one OpenMP thread",
                   "routes_s": routes}
        except Exception as e:  # the reference oracle may be absent
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"unavailable: {e}"}

    # incremental dP builds over the same density sequence (the reference's
    # EriDirectJKIncrementalState form): one exact build, then every changed
    # density as dP under the density screen at the Schwarz threshold
    incremental = None
    if not args.no_extra:
        incremental = _incremental_leg(ctx, Ds, tau, J64, K64)
        # ERI checksum stream (the reference's twoe_timing endpoint) on the plan
        checksum_leg = _checksum_leg(ctx, quartets)
        onee_leg = _onee_leg(ctx, mol, rank == 0 and not args.no_cpu_baseline)
    else:
        checksum_leg = onee_leg = None

    clocks = sampler.summary()
    res = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tmx / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64+f32 mixed (FP64 accumulation)", "data": "synthetic",
        "config": {"workload": args.config, "description": wdesc, "M": M, "quartets_per_build": quartets,
                   "primitive_quartets_per_build": prof["primitive_quartets"],
                   "flops_per_build_model": prof["flops"], "parallelism": f"replicas{ws}",
                   "streams": args.streams,
                   "l2": "inputs larger than L2 (D, J, K are M*M*8 bytes each)" if flush is None else
                         "L2 flushed between timed builds (256 MB write)",
                   "mixed_threshold": "per class (mixed_autotune)" if tune else args.mixed_threshold,
                   "schwarz": tau},
        "mixed_autotune": tune,
        "jk_builds_per_s": ws * steps / tmx,
        "fp64": {"value": value64, "unit": UNIT, "jk_builds_per_s": ws * steps / t64,
                 "ms_per_step": 1e3 * t64 / steps},
        "mixed_speedup_vs_fp64": t64 / tmx,
        "accuracy": {"abs_dE_Eh": abs(dE), "max_abs_dJ": dJ, "max_abs_dK": dK},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None, "traffic": traffic,
                     "kernel": (f"eri_fast_jk_kernel<float> class {dom_tag}" if cdom["fast"] else
                                f"eri_generic_cta_jk_kernel<float> class {dom_tag}") +
                               " over all quartets of the class",
                     "launch_ms": tdom,
                     "flops_per_launch_model": cdom["flops"],
                     "peak_source": "of measured: FP32 FMA-chain probe (tlno_gpu_fma_peak) on this GPU; "
                                    "MEASURED_PEAKS.json holds no FP32/FP64 CUDA-core figure",
                     "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per launch, one ncu capture "
                                       f"(profiles/dram_traffic.json entry {traffic_key!r} of {args.config})",
                     "fp64": {"achieved": achieved64, "peak": peak64, "frac": achieved64 / peak64 if peak64 else None,
                              "launch_ms": tdom64,
                              "peak_source": "of measured: DFMA-chain probe (tlno_gpu_fma_peak) on this GPU"}},
        "e2e": e2e, "gpu_launches": launches * steps,
        "incremental": incremental, "eri_checksum_stream": checksum_leg, "one_electron": onee_leg,
        "clocks": clocks, "wall_s_timed": t_wall,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(res))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--config", default="cfg4")
    ap.add_argument("--mixed-threshold", type=float, default=1e-9)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--streams", type=int, default=1,
                    help="streams the class launches of a build spread over (1..4)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the incremental, ERI-stream and one-electron legs")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep --mixed-threshold instead of autotuning the split threshold")
    ap.add_argument("--ref-sample", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.ref_sample:  # one reference sample on this process's route
        secs, desc, _, _ = _reference_sample(args.config)
        print(json.dumps({"secs": secs, "desc": desc}))
        return 0
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "cfg3":
        return run_batch(args)
    return run_native(args)


if __name__ == "__main__":
    sys.exit(main())

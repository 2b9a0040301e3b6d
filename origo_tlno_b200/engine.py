"""Python host mirror of the reference's C++ engine interfaces.

Names, argument meaning and error behaviour follow the reference:

* ``ScreeningOptions`` -- fock::ScreeningOptions
  (integrals/two_electron/fock/jk_direct.hpp:18-24), plus ``mixed_threshold``.
* ``build_direct_plan(basis, options)`` -- fock::build_direct_plan (:46-48).
* ``build_coulomb_j / build_exchange_k / build_rhf_g(plan, density, options)``
  -- jk_direct.hpp:82-96; results carry ``j`` / ``k`` / ``g`` and ``M``.
* ``build_jk_direct_for_G_rys(plan, density, options)`` --
  fock/eri_direct_jk.hpp:36-39; ``Incremental`` -- EriDirectJKIncrementalState
  (eri_direct_jk.hpp:41-135); ``build_eri_packed_for_G_rys(plan)`` -- the ERI
  checksum stream (twoe_integrals.hpp:114-119).
* ``build_one_electron_spherical_matrices(build)`` and
  ``evaluate_one_electron_matrices_sph_into(build, plan, mats)`` --
  integrals/one_electron/onee_matrices.hpp:50, 63-66.
* ``set_onee_screening_enabled`` / ``set_onee_group_pair_decay_eps`` /
  ``set_onee_nuclear_screen_eps`` -- onee_matrices.hpp:72-79,
  onee_integrals.hpp:187-188 (process-global knobs, as in the reference).

Every call runs the CUDA library (``_native``); failures raise
``TlnoError`` whose message is the reference's exception text for the same
condition.  A ``BasisBuildResult`` here is a :class:`molecules.Molecule`
(contracted shells + nuclear charges/centres).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from .molecules import Molecule

TlnoError = N.TlnoError


@dataclass
class ScreeningOptions:
    integral_threshold: float = 1.0e-12
    primitive_fastschwarz_threshold: float = 0.0
    decay_threshold: float = 0.0
    density_threshold: float = 0.0
    mixed_threshold: float = 1.0e-9

    def to_c(self) -> N.Screening:
        return N.Screening(self.integral_threshold, self.primitive_fastschwarz_threshold,
                           self.decay_threshold, self.density_threshold, self.mixed_threshold)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Context:
    """One basis on one CUDA device (tlno_gpu_context)."""

    def __init__(self, mol: Molecule, device: int = 0):
        L = N.lib()
        centers, Ls, nprim, exps, coefs = mol.soa()
        self._keep = [_f64(centers), _i32(Ls), _i32(nprim), _f64(exps), _f64(coefs),
                      _i32(mol.charges), _f64(mol.coords)]
        h = C.c_void_p()
        c, l, n, e, k, z, x = self._keep
        N.check(L.tlno_gpu_create(len(mol.shells), N.ptr(c), N.ptr(l), N.ptr(n), N.ptr(e), N.ptr(k),
                                  len(mol.charges), N.ptr(z), N.ptr(x), device, C.byref(h)))
        self.h = h
        self.mol = mol
        self.M = L.tlno_gpu_n_sph(h)
        self.device = device
        self.options: Optional[ScreeningOptions] = None

    @classmethod
    def from_components(cls, centers, ang, nprim, exps, coefs, charges, coords, device: int = 0):
        """Create from per-Cartesian-component normalised records (the
        reference's std::vector<Shell> layout)."""
        self = cls.__new__(cls)
        L = N.lib()
        self._keep = [_f64(centers), _i32(ang), _i32(nprim), _f64(exps), _f64(coefs), _i32(charges), _f64(coords)]
        c, a, n, e, k, z, x = self._keep
        h = C.c_void_p()
        N.check(L.tlno_gpu_create_from_components(len(n), N.ptr(c), N.ptr(a), N.ptr(n), N.ptr(e), N.ptr(k),
                                                  len(z), N.ptr(z), N.ptr(x), device, C.byref(h)))
        self.h = h
        self.mol = None
        self.M = L.tlno_gpu_n_sph(h)
        self.device = device
        self.options = None
        return self

    def close(self):
        if getattr(self, "h", None):
            N.lib().tlno_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- two-electron ---------------------------------------------------
    def plan(self, options: Optional[ScreeningOptions] = None):
        options = options or ScreeningOptions()
        N.check(N.lib().tlno_gpu_plan(self.h, C.byref(options.to_c())))
        self.options = options
        return self

    def profile(self) -> dict:
        p = N.Profile()
        N.check(N.lib().tlno_gpu_plan_profile(self.h, C.byref(p)))
        return {f: getattr(p, f) for f, _ in N.Profile._fields_}

    def jk(self, density, want=("J", "K"), mixed=False, validate=True,
           options: Optional[ScreeningOptions] = None):
        """J / K / G of a host density.  ``options`` are the reference's
        build-time ScreeningOptions (density and FASTSCHWARZ screening of this
        build; another integral or decay threshold re-plans)."""
        D = _f64(density)
        M = self.M
        if D.shape != (M, M):
            raise TlnoError(N.E_INVALID, "eri_ao_tensor_hgp: density must be spherical M x M row-major.")
        flags = 0
        out = {}
        J = K = G = None
        if "J" in want:
            flags |= N.WANT_J
            J = np.empty((M, M))
        if "K" in want:
            flags |= N.WANT_K
            K = np.empty((M, M))
        if "G" in want:
            flags |= N.WANT_G
            G = np.empty((M, M))
        if mixed:
            flags |= N.MIXED
        if not validate:
            flags |= N.NO_VALIDATE
        if options is None:
            N.check(N.lib().tlno_gpu_jk(self.h, N.ptr(D), N.ptr(J), N.ptr(K), N.ptr(G), flags))
        else:
            opts = options.to_c()
            if self.options is not None:
                opts.mixed_threshold = self.options.mixed_threshold
            N.check(N.lib().tlno_gpu_jk_with_options(self.h, N.ptr(D), N.ptr(J), N.ptr(K), N.ptr(G), flags,
                                                     C.byref(opts)))
            self.options = ScreeningOptions(options.integral_threshold, options.primitive_fastschwarz_threshold,
                                            options.decay_threshold, options.density_threshold,
                                            opts.mixed_threshold)
        for k, v in (("J", J), ("K", K), ("G", G)):
            if v is not None:
                out[k] = v
        return out

    def jk_device(self, d_density_ptr: int, d_J: int, d_K: int, mixed=False, validate=False):
        flags = N.WANT_J | N.WANT_K | N.DEVICE_PTRS | (N.MIXED if mixed else 0) | (0 if validate else N.NO_VALIDATE)
        N.check(N.lib().tlno_gpu_jk(self.h, d_density_ptr, d_J, d_K, None, flags))

    def eri_checksum(self):
        """(checksum, device ms) of the ERI stream: the sum of the canonical
        unique spherical ERIs that pass the plan's screen."""
        cs = C.c_double()
        ms = C.c_double()
        N.check(N.lib().tlno_gpu_eri_checksum(self.h, C.byref(cs), C.byref(ms)))
        return cs.value, ms.value

    def graph_capture(self, d_density_ptr: int, d_J: int, d_K: int, mixed=False):
        flags = N.WANT_J | N.WANT_K | (N.MIXED if mixed else 0)
        N.check(N.lib().tlno_gpu_jk_graph_capture(self.h, d_density_ptr, d_J, d_K, flags))

    def graph_launch(self):
        N.check(N.lib().tlno_gpu_jk_graph_launch(self.h))

    def synchronize(self):
        N.check(N.lib().tlno_gpu_synchronize(self.h))

    def stream(self) -> int:
        return N.lib().tlno_gpu_stream(self.h)

    def schwarz(self) -> np.ndarray:
        ns = N.lib().tlno_gpu_n_shells(self.h)
        out = np.empty(ns * (ns + 1) // 2)
        N.check(N.lib().tlno_gpu_schwarz(self.h, N.ptr(out)))
        return out

    def eri_blocks(self, quartets: Sequence[Sequence[int]]):
        """Spherical ERI blocks for shell quartets; returns a list of arrays
        shaped ((2La+1)(2Lb+1), (2Lc+1)(2Ld+1))."""
        q = _i32(np.asarray(quartets, dtype=np.int32).reshape(-1, 4))
        Ls = [s.L for s in self.mol.shells]
        sizes = [(2 * Ls[a] + 1) * (2 * Ls[b] + 1) * (2 * Ls[c] + 1) * (2 * Ls[d] + 1) for a, b, c, d in q]
        offs = np.zeros(len(q), dtype=np.int64)
        if len(q):
            offs[1:] = np.cumsum(sizes)[:-1]
        out = np.empty(max(int(sum(sizes)), 1))
        N.check(N.lib().tlno_gpu_eri_blocks(self.h, len(q), N.ptr(q), N.ptr(offs), N.ptr(out)))
        res = []
        for (a, b, c, d), o, s in zip(q, offs, sizes):
            res.append(out[o:o + s].reshape((2 * Ls[a] + 1) * (2 * Ls[b] + 1), (2 * Ls[c] + 1) * (2 * Ls[d] + 1)).copy())
        return res

    # -- one-electron ---------------------------------------------------
    def onee(self, screening=True):
        M = self.M
        S, T, V = np.empty((M, M)), np.empty((M, M)), np.empty((M, M))
        N.check(N.lib().tlno_gpu_onee(self.h, N.ptr(S), N.ptr(T), N.ptr(V), 1 if screening else 0, 0))
        return S, T, V

    def set_mixed_threshold(self, threshold: float):
        """Split threshold of the mixed-precision path without re-planning
        (recapture any J/K graph afterwards)."""
        N.check(N.lib().tlno_gpu_set_mixed_threshold(self.h, threshold))
        if getattr(self, "options", None) is not None:
            self.options.mixed_threshold = threshold

    def set_onee_thresholds(self, decay_eps: float, nuclear_eps: float):
        N.check(N.lib().tlno_gpu_set_onee_thresholds(self.h, decay_eps, nuclear_eps))

    # -- tuning ---------------------------------------------------------
    def set_tuning(self, generic_bk=64, generic_warps=0, grid_mult=8, streams=1):
        t = N.Tuning(generic_bk, generic_warps, grid_mult, streams)
        N.check(N.lib().tlno_gpu_set_tuning(self.h, C.byref(t)))

    def set_combo_generic(self, combo_id: int, force: bool):
        N.check(N.lib().tlno_gpu_set_combo_generic(self.h, combo_id, 1 if force else 0))

    def combos(self):
        n = N.check(N.lib().tlno_gpu_plan_combos(self.h, 0, None, None))
        ints = np.zeros(8 * max(n, 1), dtype=np.int32)
        dbl = np.zeros(3 * max(n, 1))
        N.check(N.lib().tlno_gpu_plan_combos(self.h, n, N.ptr(ints), N.ptr(dbl)))
        keys = ("X", "Y", "la", "lb", "lc", "ld", "fast", "n_tiles")
        out = []
        for i in range(n):
            d = dict(zip(keys, (int(v) for v in ints[8 * i:8 * i + 8])))
            d.update(quartets=dbl[3 * i], prim_quartets=dbl[3 * i + 1], flops=dbl[3 * i + 2])
            out.append(d)
        return out

    def time_combo(self, index: int, fp32: bool = False, reps: int = 3, want_j: bool = True,
                   want_k: bool = True) -> float:
        ms = C.c_double()
        mode = (1 if fp32 else 0) | (0 if want_j else 2) | (0 if want_k else 4)
        N.check(N.lib().tlno_gpu_time_combo(self.h, index, mode, reps, C.byref(ms)))
        return ms.value


class Batch:
    """Many molecules in one work queue per class (tlno_gpu_batch)."""

    def __init__(self, contexts: Sequence[Context], options: Optional[ScreeningOptions] = None):
        options = options or ScreeningOptions()
        arr = (C.c_void_p * len(contexts))(*[c.h for c in contexts])
        h = C.c_void_p()
        N.check(N.lib().tlno_gpu_batch_create(len(contexts), arr, C.byref(options.to_c()), C.byref(h)))
        self.h = h
        self.contexts = list(contexts)
        self.total = N.lib().tlno_gpu_batch_total_elements(h)
        offs = np.zeros(len(contexts) + 1, dtype=np.int64)
        N.check(N.lib().tlno_gpu_batch_offsets(h, N.ptr(offs)))
        self.offsets = offs

    def close(self):
        if getattr(self, "h", None):
            N.lib().tlno_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def profile(self) -> dict:
        p = N.Profile()
        N.check(N.lib().tlno_gpu_batch_profile(self.h, C.byref(p)))
        return {f: getattr(p, f) for f, _ in N.Profile._fields_}

    def set_tuning(self, generic_bk=64, generic_warps=0, grid_mult=8, streams=1):
        t = N.Tuning(generic_bk, generic_warps, grid_mult, streams)
        N.check(N.lib().tlno_gpu_batch_set_tuning(self.h, C.byref(t)))

    def jk(self, densities, mixed=False):
        D = np.concatenate([_f64(d).ravel() for d in densities])
        J = np.empty(self.total)
        K = np.empty(self.total)
        N.check(N.lib().tlno_gpu_batch_jk(self.h, N.ptr(D), N.ptr(J), N.ptr(K), N.MIXED if mixed else 0))
        outJ, outK = [], []
        for m, c in enumerate(self.contexts):
            a, b = self.offsets[m], self.offsets[m + 1]
            outJ.append(J[a:b].reshape(c.M, c.M))
            outK.append(K[a:b].reshape(c.M, c.M))
        return outJ, outK

    def jk_device(self, d_density: int, d_J: int, d_K: int, mixed=False):
        N.check(N.lib().tlno_gpu_batch_jk(self.h, d_density, d_J, d_K,
                                          N.DEVICE_PTRS | (N.MIXED if mixed else 0)))

    def graph_capture(self, d_density: int, d_J: int, d_K: int, mixed=False):
        N.check(N.lib().tlno_gpu_batch_graph_capture(self.h, d_density, d_J, d_K, N.MIXED if mixed else 0))

    def graph_launch(self):
        N.check(N.lib().tlno_gpu_batch_graph_launch(self.h))

    def synchronize(self):
        N.check(N.lib().tlno_gpu_batch_synchronize(self.h))

    def stream(self) -> int:
        return N.lib().tlno_gpu_batch_stream(self.h)


class Incremental:
    """Incremental dP builds of G = J - K/2 (the reference's
    EriDirectJKIncrementalState, fock/eri_direct_jk.hpp:41-135): update()
    returns "exact_rebuild", "incremental_update" or "skipped_unchanged"."""

    STATUS = {1: "exact_rebuild", 2: "incremental_update", 3: "skipped_unchanged", 0: "uninitialized"}

    def __init__(self, context: Context, base_options: Optional[ScreeningOptions] = None,
                 exact_rebuild_interval: int = 8, delta_density_threshold: float = 0.0,
                 use_first_delta_density_threshold: bool = False, first_delta_density_threshold: float = 0.0):
        base = (base_options or ScreeningOptions()).to_c()
        o = N.IncrementalOptions(base, exact_rebuild_interval, delta_density_threshold,
                                 1 if use_first_delta_density_threshold else 0, first_delta_density_threshold)
        h = C.c_void_p()
        N.check(N.lib().tlno_gpu_incremental_create(context.h, C.byref(o), C.byref(h)))
        self.h = h
        self.context = context
        self.M = context.M

    def close(self):
        if getattr(self, "h", None):
            N.lib().tlno_gpu_incremental_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def update(self, density, force_exact_rebuild: bool = False, mixed: bool = False) -> str:
        D = _f64(density)
        if D.shape != (self.M, self.M):
            raise TlnoError(N.E_INVALID, "eri_ao_tensor_hgp: incremental density must be spherical M x M row-major.")
        rc = N.check(N.lib().tlno_gpu_incremental_update(self.h, N.ptr(D), 1 if force_exact_rebuild else 0,
                                                         N.MIXED if mixed else 0))
        return self.STATUS[rc]

    def update_device(self, d_density: int, force_exact_rebuild: bool = False, mixed: bool = False) -> str:
        rc = N.check(N.lib().tlno_gpu_incremental_update(self.h, d_density, 1 if force_exact_rebuild else 0,
                                                         N.DEVICE_PTRS | (N.MIXED if mixed else 0)))
        return self.STATUS[rc]

    def g(self) -> np.ndarray:
        G = np.empty((self.M, self.M))
        N.check(N.lib().tlno_gpu_incremental_g(self.h, N.ptr(G), 0))
        return G

    def density(self) -> np.ndarray:
        D = np.empty((self.M, self.M))
        N.check(N.lib().tlno_gpu_incremental_density(self.h, N.ptr(D), 0))
        return D

    def info(self) -> dict:
        i = N.IncrementalInfo()
        N.check(N.lib().tlno_gpu_incremental_info_get(self.h, C.byref(i)))
        d = {f: getattr(i, f) for f, _ in N.IncrementalInfo._fields_}
        d["last_status"] = self.STATUS[d["last_status"]]
        return d

    def reset(self):
        N.check(N.lib().tlno_gpu_incremental_reset(self.h))

    def fail_next_update(self, stage: int):
        """Testing hook: the next update fails at `stage` (1 before the build,
        2 before the commit)."""
        N.check(N.lib().tlno_gpu_incremental_fail_next_update(self.h, stage))


# ---------------- reference-named facade ----------------

@dataclass
class DirectPlan:
    context: Context
    profile: dict


@dataclass
class CoulombJResult:
    j: np.ndarray
    M: int


@dataclass
class ExchangeKResult:
    k: np.ndarray
    M: int


@dataclass
class DirectResult:
    g: np.ndarray
    M: int


def build_direct_plan(basis: Molecule, options: Optional[ScreeningOptions] = None, device: int = 0) -> DirectPlan:
    ctx = Context(basis, device).plan(options or ScreeningOptions())
    return DirectPlan(ctx, ctx.profile())


def build_coulomb_j(plan: DirectPlan, density, options: Optional[ScreeningOptions] = None) -> CoulombJResult:
    return CoulombJResult(plan.context.jk(density, want=("J",), options=options)["J"], plan.context.M)


def build_exchange_k(plan: DirectPlan, density, options: Optional[ScreeningOptions] = None) -> ExchangeKResult:
    return ExchangeKResult(plan.context.jk(density, want=("K",), options=options)["K"], plan.context.M)


def build_rhf_g(plan: DirectPlan, density, options: Optional[ScreeningOptions] = None) -> DirectResult:
    return DirectResult(plan.context.jk(density, want=("G",), options=options)["G"], plan.context.M)


def build_jk_direct_for_G_rys(plan: DirectPlan, density, options: Optional[ScreeningOptions] = None) -> DirectResult:
    """Compatibility endpoint (fock/eri_direct_jk.hpp:36-39): G = J - K/2."""
    return build_rhf_g(plan, density, options)


def build_eri_packed_for_G_rys(plan: DirectPlan) -> float:
    """ERI checksum stream of the plan (twoe_integrals.hpp:114-119)."""
    return plan.context.eri_checksum()[0]


_ONEE = {"enabled": True, "decay": 1.0e-15, "nuclear": 1.0e-15}


def set_onee_screening_enabled(enabled: bool) -> None:
    _ONEE["enabled"] = bool(enabled)
    _ONEE["decay"] = 1.0e-15 if enabled else 0.0
    _ONEE["nuclear"] = 1.0e-15 if enabled else 0.0


def onee_screening_enabled() -> bool:
    return _ONEE["decay"] > 0.0


def set_onee_group_pair_decay_eps(eps: float) -> None:
    _ONEE["decay"] = float(eps)


def set_onee_nuclear_screen_eps(eps: float) -> None:
    _ONEE["nuclear"] = float(eps)


@dataclass
class OneElectronMatrices:
    overlap: np.ndarray
    kinetic: np.ndarray
    nuclear: np.ndarray


@dataclass
class OneElectronPlan:
    context: Context
    n_sph: int


def build_one_electron_plan(build: Molecule, device: int = 0) -> OneElectronPlan:
    ctx = Context(build, device)
    return OneElectronPlan(ctx, ctx.M)


def evaluate_one_electron_matrices_sph_into(build: Molecule, plan: OneElectronPlan,
                                            mats: Optional[OneElectronMatrices] = None) -> OneElectronMatrices:
    ctx = plan.context
    ctx.set_onee_thresholds(_ONEE["decay"], _ONEE["nuclear"])
    S, T, V = ctx.onee(screening=True)
    if mats is None:
        return OneElectronMatrices(S, T, V)
    mats.overlap, mats.kinetic, mats.nuclear = S, T, V
    return mats


def build_one_electron_spherical_matrices(build: Molecule, device: int = 0) -> OneElectronMatrices:
    return evaluate_one_electron_matrices_sph_into(build, build_one_electron_plan(build, device))


def fma_peak_tflops(fp32: bool = False, device: int = 0) -> float:
    """Measured FMA throughput (TFLOP/s) of the device."""
    v = C.c_double()
    N.check(N.lib().tlno_gpu_fma_peak(device, 1 if fp32 else 0, C.byref(v)))
    return v.value


def boys(x, maxn: int, device: int = 0) -> np.ndarray:
    x = _f64(np.atleast_1d(x))
    out = np.empty((len(x), maxn + 1))
    N.check(N.lib().tlno_gpu_boys(device, len(x), maxn, N.ptr(x), N.ptr(out)))
    return out


RYS_PATHS = {"fp64_table": 0, "fp32_table": 1, "fp32_interval": 2}


def rys_roots(T, nroots: int, fp32: bool = False, device: int = 0, path: Optional[str] = None):
    """Device Rys roots and weights; ``path`` selects one of the kernels'
    evaluation paths (RYS_PATHS), default the FP64 (or FP32) tables."""
    T = _f64(np.atleast_1d(T))
    r = np.empty((len(T), nroots))
    w = np.empty((len(T), nroots))
    mode = RYS_PATHS[path] if path else (1 if fp32 else 0)
    N.check(N.lib().tlno_gpu_rys(device, len(T), nroots, N.ptr(T), N.ptr(r), N.ptr(w), mode))
    return r, w

"""TEST INFRASTRUCTURE: ctypes wrapper of oracle/_ref/libtlno_ref.so, the
UNMODIFIED origo-tlno reference engine compiled from its own sources by
oracle/build_ref.sh together with oracle/ref_harness.cpp.

Only tests/, __graft_entry__.smoke() and bench.py (CPU baseline and the
`--impl reference` arm) may use this module, as the checker or as the timed
CPU baseline -- never as the product path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# TLNO_REF_ROUTE selects the reference build: "avx2" (its legacy tuned
# route, -march=x86-64-v3, the default) or "avx512" (its native W8 route,
# -march=x86-64-v4).  One route per process.
ROUTE = os.environ.get("TLNO_REF_ROUTE", "avx2")
if ROUTE not in ("avx2", "avx512"):
    raise ValueError(f"TLNO_REF_ROUTE must be avx2 or avx512, not {ROUTE!r}")
LIB_PATH = os.path.join(HERE, "_ref", "libtlno_ref.so" if ROUTE == "avx2" else "libtlno_ref_avx512.so")

_lib = None
_gomp = None


def _omp():
    """libgomp as loaded by the reference library (OpenMP thread control:
    the reference's G and K endpoints refuse more than one thread,
    rys_engine.ipp:16853-16857)."""
    global _gomp
    if _gomp is None:
        lib()
        _gomp = C.CDLL("libgomp.so.1")
        _gomp.omp_get_max_threads.restype = C.c_int
        _gomp.omp_set_num_threads.argtypes = [C.c_int]
    return _gomp


class single_thread:
    def __enter__(self):
        self.prev = _omp().omp_get_max_threads()
        _omp().omp_set_num_threads(1)

    def __exit__(self, *a):
        _omp().omp_set_num_threads(self.prev)


def set_threads(n: int) -> None:
    _omp().omp_set_num_threads(int(n))


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (oracle/build_ref.sh)")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.ref_last_error.restype = C.c_char_p
        L.ref_basis_create.restype = vp
        L.ref_basis_create.argtypes = [C.c_int, vp, vp, vp, vp, vp, C.c_int, vp, vp]
        L.ref_basis_destroy.argtypes = [vp]
        L.ref_basis_n_sph.argtypes = [vp]
        L.ref_basis_n_cart.argtypes = [vp]
        L.ref_basis_component_coefs.argtypes = [vp, C.c_int, vp]
        L.ref_onee_sph.argtypes = [vp, C.c_int, vp, vp, vp]
        L.ref_onee_cart.argtypes = [vp, C.c_int, vp, vp, vp]
        L.ref_jk.argtypes = [vp, vp, C.c_double, C.c_double, vp, vp, vp]
        L.ref_time_jk.argtypes = [vp, vp, C.c_double, C.c_int, vp]
        L.ref_eri_sph_block.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp]
        L.ref_schwarz_pair_max.argtypes = [vp, vp]
        L.ref_boys_single.restype = C.c_double
        L.ref_boys_single.argtypes = [C.c_int, C.c_double]
        L.ref_boys_r000_all.argtypes = [C.c_int, C.c_double, C.c_double, vp]
        L.ref_boys_hgp.restype = C.c_double
        L.ref_boys_hgp.argtypes = [C.c_int, C.c_double]
        L.ref_rys_roots.argtypes = [C.c_int, C.c_double, vp, vp]
        L.ref_rys_roots_accurate.argtypes = [C.c_int, C.c_double, vp, vp]
        L.ref_jk_opts.argtypes = [vp, vp, C.c_double, C.c_double, C.c_double, C.c_double, vp, vp, vp]
        L.ref_jk_compat.argtypes = [vp, vp, C.c_double, C.c_double, vp]
        L.ref_eri_checksum.argtypes = [vp, C.c_double, vp, vp]
        L.ref_incremental_create.restype = vp
        L.ref_incremental_create.argtypes = [vp, C.c_double, C.c_ulonglong, C.c_double, C.c_int, C.c_double]
        L.ref_incremental_destroy.argtypes = [vp]
        L.ref_incremental_update.argtypes = [vp, vp, C.c_int, vp, vp, vp, vp, vp]
        L.ref_basis_components.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
        _lib = L
    return _lib


def _chk(rc):
    if rc != 0:
        raise RuntimeError("reference: " + lib().ref_last_error().decode())


class RefBasis:
    def __init__(self, mol):
        centers, Ls, nprim, exps, coefs = mol.soa()
        self._keep = [np.ascontiguousarray(centers, dtype=np.float64), np.ascontiguousarray(Ls, dtype=np.int32),
                      np.ascontiguousarray(nprim, dtype=np.int32), np.ascontiguousarray(exps, dtype=np.float64),
                      np.ascontiguousarray(coefs, dtype=np.float64), np.ascontiguousarray(mol.charges, dtype=np.int32),
                      np.ascontiguousarray(mol.coords, dtype=np.float64)]
        c, l, n, e, k, z, x = self._keep
        self.h = lib().ref_basis_create(len(mol.shells), c.ctypes.data, l.ctypes.data, n.ctypes.data,
                                        e.ctypes.data, k.ctypes.data, len(z), z.ctypes.data, x.ctypes.data)
        if not self.h:
            raise RuntimeError("reference: " + lib().ref_last_error().decode())
        self.M = lib().ref_basis_n_sph(self.h)
        self.n_cart = lib().ref_basis_n_cart(self.h)
        self.mol = mol

    def close(self):
        if self.h:
            lib().ref_basis_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def onee(self, screening=True):
        M = self.M
        S, T, V = np.empty((M, M)), np.empty((M, M)), np.empty((M, M))
        _chk(lib().ref_onee_sph(self.h, 1 if screening else 0, S.ctypes.data, T.ctypes.data, V.ctypes.data))
        return S, T, V

    def jk(self, D, schwarz=1e-12, density_threshold=0.0, want=("J", "K", "G")):
        M = self.M
        D = np.ascontiguousarray(D, dtype=np.float64)
        out = {k: np.empty((M, M)) for k in want}
        with single_thread():
            _chk(lib().ref_jk(self.h, D.ctypes.data, schwarz, density_threshold,
                              out["J"].ctypes.data if "J" in out else None,
                              out["K"].ctypes.data if "K" in out else None,
                              out["G"].ctypes.data if "G" in out else None))
        return out

    def jk_opts(self, D, schwarz=1e-12, fastschwarz=0.0, decay=0.0, density_threshold=0.0,
                want=("J", "K", "G")):
        """J / K / G through the public facade with every ScreeningOptions field."""
        M = self.M
        D = np.ascontiguousarray(D, dtype=np.float64)
        out = {k: np.empty((M, M)) for k in want}
        with single_thread():
            _chk(lib().ref_jk_opts(self.h, D.ctypes.data, schwarz, fastschwarz, decay, density_threshold,
                                   out["J"].ctypes.data if "J" in out else None,
                                   out["K"].ctypes.data if "K" in out else None,
                                   out["G"].ctypes.data if "G" in out else None))
        return out

    def jk_compat(self, D, schwarz=1e-12, density_threshold=0.0):
        """G through build_jk_direct_for_G_rys (the compatibility endpoint)."""
        M = self.M
        D = np.ascontiguousarray(D, dtype=np.float64)
        G = np.empty((M, M))
        with single_thread():
            _chk(lib().ref_jk_compat(self.h, D.ctypes.data, schwarz, density_threshold, G.ctypes.data))
        return G

    def eri_checksum(self, schwarz=0.0):
        """(checksum, seconds) of the ERI stream endpoint."""
        cs = C.c_double()
        t = C.c_double()
        with single_thread():
            _chk(lib().ref_eri_checksum(self.h, schwarz, C.byref(cs), C.byref(t)))
        return cs.value, t.value

    def components(self):
        """Per-Cartesian-component records (centers, ang, nprim, exps, coefs)
        exactly as the reference holds its std::vector<Shell>."""
        nc = C.c_int()
        npr = C.c_int()
        _chk(lib().ref_basis_components(self.h, C.byref(nc), C.byref(npr), None, None, None, None, None))
        centers = np.empty((nc.value, 3))
        ang = np.empty((nc.value, 3), dtype=np.int32)
        nprim = np.empty(nc.value, dtype=np.int32)
        exps = np.empty(npr.value)
        coefs = np.empty(npr.value)
        _chk(lib().ref_basis_components(self.h, C.byref(nc), C.byref(npr), centers.ctypes.data, ang.ctypes.data,
                                        nprim.ctypes.data, exps.ctypes.data, coefs.ctypes.data))
        return centers, ang, nprim, exps, coefs

    def time_jk(self, D, schwarz=1e-12, reps=1):
        D = np.ascontiguousarray(D, dtype=np.float64)
        t = np.empty(reps)
        with single_thread():
            _chk(lib().ref_time_jk(self.h, D.ctypes.data, schwarz, reps, t.ctypes.data))
        return t

    def eri_block(self, a, b, c, d):
        Ls = [s.L for s in self.mol.shells]
        out = np.empty((2 * Ls[a] + 1) * (2 * Ls[b] + 1) * (2 * Ls[c] + 1) * (2 * Ls[d] + 1))
        _chk(lib().ref_eri_sph_block(self.h, a, b, c, d, out.ctypes.data))
        return out.reshape((2 * Ls[a] + 1) * (2 * Ls[b] + 1), (2 * Ls[c] + 1) * (2 * Ls[d] + 1))

    def schwarz(self):
        ns = len(self.mol.shells)
        out = np.empty(ns * (ns + 1) // 2)
        with single_thread():
            _chk(lib().ref_schwarz_pair_max(self.h, out.ctypes.data))
        return out


def boys_single(n: int, x: float) -> float:
    return lib().ref_boys_single(n, x)


def boys_r000_all(max_n: int, x: float, p: float) -> np.ndarray:
    out = np.empty(max_n + 1)
    lib().ref_boys_r000_all(max_n, x, p, out.ctypes.data)
    return out


def rys_roots(n: int, t: float, accurate: bool = False):
    r = np.empty(n)
    w = np.empty(n)
    f = lib().ref_rys_roots_accurate if accurate else lib().ref_rys_roots
    f(n, t, r.ctypes.data, w.ctypes.data)
    return r, w


class RefIncremental:
    """EriDirectJKIncrementalState of the reference on its own plan."""

    STATUS = {1: "exact_rebuild", 2: "incremental_update", 3: "skipped_unchanged"}

    def __init__(self, basis: RefBasis, schwarz=1e-12, exact_rebuild_interval=8, delta_density_threshold=0.0,
                 use_first_delta_density_threshold=False, first_delta_density_threshold=0.0):
        self.basis = basis
        self.h = lib().ref_incremental_create(basis.h, schwarz, exact_rebuild_interval, delta_density_threshold,
                                              1 if use_first_delta_density_threshold else 0,
                                              first_delta_density_threshold)
        if not self.h:
            raise RuntimeError("reference: " + lib().ref_last_error().decode())

    def update(self, D, force=False):
        M = self.basis.M
        D = np.ascontiguousarray(D, dtype=np.float64)
        G = np.empty((M, M))
        st = C.c_int()
        cnt = np.zeros(4, dtype=np.uint64)
        ld = C.c_double()
        lt = C.c_double()
        with single_thread():
            _chk(lib().ref_incremental_update(self.h, D.ctypes.data, 1 if force else 0, G.ctypes.data, C.byref(st),
                                              cnt.ctypes.data, C.byref(ld), C.byref(lt)))
        return {"status": self.STATUS.get(st.value, st.value), "G": G, "counters": [int(x) for x in cnt],
                "last_max_abs_density_delta": ld.value, "last_effective_density_threshold": lt.value}

    def close(self):
        if self.h:
            lib().ref_incremental_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------- front end (oracle/ref_frontend.cpp) ----------------

def _front():
    L = lib()
    if not getattr(L, "_front_ready", False):
        vp = C.c_void_p
        L.ref_frontend_last_error.restype = C.c_char_p
        L.ref_read_inp.argtypes = [C.c_char_p, C.c_int, vp, vp, vp, vp, vp]
        L.ref_basis_general.argtypes = [C.c_int, vp, vp, C.c_int, C.c_char_p, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.ref_raw_atom_basis.argtypes = [C.c_char_p, C.c_char_p, vp, vp, vp, vp, vp, vp, vp]
        L.ref_parse_basis_kind.argtypes = [C.c_char_p]
        L._front_ready = True
    return L


def _fchk(rc):
    if rc != 0:
        raise RuntimeError("reference: " + _front().ref_frontend_last_error().decode())


def read_inp(path):
    """(symbols, coords_bohr, charge, multiplicity) through read_inp_file."""
    n = C.c_int()
    ch = C.c_int()
    mu = C.c_int()
    _fchk(_front().ref_read_inp(path.encode(), 0, C.byref(n), None, None, C.byref(ch), C.byref(mu)))
    sym = C.create_string_buffer(8 * n.value)
    xyz = np.empty((n.value, 3))
    _fchk(_front().ref_read_inp(path.encode(), n.value, C.byref(n), sym, xyz.ctypes.data, C.byref(ch), C.byref(mu)))
    raw = sym.raw
    symbols = [raw[8 * a:8 * a + 8].split(b"\0")[0].decode() for a in range(n.value)]
    return symbols, xyz, ch.value, mu.value


def basis_general(symbols, coords, charge, basis):
    """Component records, nuclear charges and electron count of
    build_basis_general."""
    n = len(symbols)
    sym = C.create_string_buffer(b"".join(s.encode()[:7].ljust(8, b"\0") for s in symbols), 8 * n)
    xyz = np.ascontiguousarray(coords, dtype=np.float64)
    nc = C.c_int()
    npr = C.c_int()
    el = C.c_int()
    Z = np.empty(n, dtype=np.int32)
    _fchk(_front().ref_basis_general(n, sym, xyz.ctypes.data, charge, basis.encode(), C.byref(nc), C.byref(npr),
                                     None, None, None, None, None, Z.ctypes.data, C.byref(el)))
    centers = np.empty((nc.value, 3))
    ang = np.empty((nc.value, 3), dtype=np.int32)
    nprim = np.empty(nc.value, dtype=np.int32)
    exps = np.empty(npr.value)
    coefs = np.empty(npr.value)
    _fchk(_front().ref_basis_general(n, sym, xyz.ctypes.data, charge, basis.encode(), C.byref(nc), C.byref(npr),
                                     centers.ctypes.data, ang.ctypes.data, nprim.ctypes.data, exps.ctypes.data,
                                     coefs.ctypes.data, Z.ctypes.data, C.byref(el)))
    return (centers, ang, nprim, exps, coefs), Z, el.value


def raw_atom_basis(symbol, basis):
    """(charge, [(ang, exponents, raw coefficients)]) of the reference's
    per-element table."""
    ch = C.c_int()
    nr = C.c_int()
    npr = C.c_int()
    _fchk(_front().ref_raw_atom_basis(symbol.encode(), basis.encode(), C.byref(ch), C.byref(nr), C.byref(npr),
                                      None, None, None, None))
    ang = np.empty((nr.value, 3), dtype=np.int32)
    nprim = np.empty(nr.value, dtype=np.int32)
    exps = np.empty(npr.value)
    coefs = np.empty(npr.value)
    _fchk(_front().ref_raw_atom_basis(symbol.encode(), basis.encode(), C.byref(ch), C.byref(nr), C.byref(npr),
                                      ang.ctypes.data, nprim.ctypes.data, exps.ctypes.data, coefs.ctypes.data))
    out, p = [], 0
    for k in range(nr.value):
        out.append((tuple(int(v) for v in ang[k]), exps[p:p + nprim[k]].copy(), coefs[p:p + nprim[k]].copy()))
        p += nprim[k]
    return ch.value, out


def parse_basis_kind_ok(name):
    return _front().ref_parse_basis_kind(name.encode()) == 0

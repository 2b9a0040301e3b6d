"""TEST INFRASTRUCTURE: ctypes wrapper of oracle/libtlno_oracle.so, the plain
C++ restatement of the reference algorithm (oracle/tlno_oracle.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may use
it, as the checker -- never as the product path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtlno_oracle.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.orc_boys.restype = C.c_double
        L.orc_boys.argtypes = [C.c_int, C.c_double]
        L.orc_rys.argtypes = [C.c_int, C.c_double, vp, vp]
        L.orc_basis_create.restype = vp
        L.orc_basis_create.argtypes = [C.c_int, vp, vp, vp, vp, vp, C.c_int, vp, vp]
        L.orc_basis_destroy.argtypes = [vp]
        L.orc_basis_n_sph.argtypes = [vp]
        L.orc_eri_sph_block.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp]
        L.orc_schwarz.argtypes = [vp, vp]
        L.orc_jk.argtypes = [vp, vp, C.c_double, vp, vp]
        L.orc_onee.argtypes = [vp, C.c_int, vp, vp, vp]
        _lib = L
    return _lib


def boys(n: int, x: float) -> float:
    return lib().orc_boys(n, x)


def rys_roots(n: int, t: float):
    r = np.empty(n)
    w = np.empty(n)
    lib().orc_rys(n, t, r.ctypes.data, w.ctypes.data)
    return r, w


class PortBasis:
    def __init__(self, mol):
        centers, Ls, nprim, exps, coefs = mol.soa()
        self._keep = [np.ascontiguousarray(centers, dtype=np.float64), np.ascontiguousarray(Ls, dtype=np.int32),
                      np.ascontiguousarray(nprim, dtype=np.int32), np.ascontiguousarray(exps, dtype=np.float64),
                      np.ascontiguousarray(coefs, dtype=np.float64), np.ascontiguousarray(mol.charges, dtype=np.int32),
                      np.ascontiguousarray(mol.coords, dtype=np.float64)]
        c, l, n, e, k, z, x = self._keep
        self.h = lib().orc_basis_create(len(mol.shells), c.ctypes.data, l.ctypes.data, n.ctypes.data, e.ctypes.data,
                                        k.ctypes.data, len(z), z.ctypes.data, x.ctypes.data)
        self.M = lib().orc_basis_n_sph(self.h)
        self.mol = mol

    def __del__(self):
        try:
            lib().orc_basis_destroy(self.h)
        except Exception:
            pass

    def eri_block(self, a, b, c, d):
        Ls = [s.L for s in self.mol.shells]
        na, nb, nc, nd = (2 * Ls[a] + 1), (2 * Ls[b] + 1), (2 * Ls[c] + 1), (2 * Ls[d] + 1)
        out = np.empty(na * nb * nc * nd)
        lib().orc_eri_sph_block(self.h, a, b, c, d, out.ctypes.data)
        return out.reshape(na * nb, nc * nd)

    def schwarz(self):
        ns = len(self.mol.shells)
        out = np.empty(ns * (ns + 1) // 2)
        lib().orc_schwarz(self.h, out.ctypes.data)
        return out

    def jk(self, D, tau=1e-12):
        M = self.M
        D = np.ascontiguousarray(D, dtype=np.float64)
        J, K = np.empty((M, M)), np.empty((M, M))
        lib().orc_jk(self.h, D.ctypes.data, tau, J.ctypes.data, K.ctypes.data)
        return {"J": J, "K": K, "G": J - 0.5 * K}

    def onee(self, screening=True):
        M = self.M
        S, T, V = np.empty((M, M)), np.empty((M, M)), np.empty((M, M))
        lib().orc_onee(self.h, 1 if screening else 0, S.ctypes.data, T.ctypes.data, V.ctypes.data)
        return S, T, V

"""Generates the golden fixtures in tests/golden/ from the UNMODIFIED
reference engine (oracle/_ref/libtlno_ref.so, built by oracle/build_ref.sh
from the reference sources).  Run here, where the reference is present:

    python tests/golden/make_golden.py

Fixtures (float64, npz):
  cfg0.npz  -- water cfg0: S, T, V (spherical, screening on), J, K, G for
               D = C C^T (seed 1) at Schwarz 1e-12 and 0, every unique
               shell-quartet ERI block, Schwarz bounds per shell pair.
  cfg1.npz  -- cfg1 (24 atoms, M = 246): S, T, V, J, K at Schwarz 1e-12,
               Schwarz bounds, and 200 sampled ERI blocks.
  cfg2f.npz -- two heavy atoms and one H of cfg2 (shells up to f, M = 74):
               S, T, V, J, K at Schwarz 1e-12 for a random density (seed
               21), and 300 sampled ERI blocks, every one holding an f shell.
  boys.npz  -- reference Boys values F_n(x) (core/math/general_math.cpp
               boys_single) on edge and interior arguments.
  rys.npz   -- reference Rys roots/weights (production table path) for
               N = 1..9 on T in [0, 120].
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from origo_tlno_b200 import molecules as M  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def quartet_list(mol, max_n=None, seed=0):
    ns = len(mol.shells)
    pairs = [(i, j) for i in range(ns) for j in range(i + 1)]
    quads = [(a, b, c, d) for p, (a, b) in enumerate(pairs) for (c, d) in pairs[: p + 1]]
    if max_n is not None and len(quads) > max_n:
        rng = np.random.default_rng(seed)
        idx = np.sort(rng.choice(len(quads), size=max_n, replace=False))
        quads = [quads[k] for k in idx]
    return np.array(quads, dtype=np.int32)


def blocks(rb, quads):
    vals, offs = [], [0]
    for a, b, c, d in quads:
        v = rb.eri_block(int(a), int(b), int(c), int(d)).ravel()
        vals.append(v)
        offs.append(offs[-1] + v.size)
    return np.concatenate(vals), np.array(offs, dtype=np.int64)


def write_cfg2f():
    mol = M.cfg2_fragment()
    D = M.random_density(mol.n_sph, 20, seed=21)
    rb = ref.RefBasis(mol)
    S, T, V = rb.onee(screening=True)
    o = rb.jk(D, schwarz=1e-12, want=("J", "K"))
    Ls = [s.L for s in mol.shells]
    q = quartet_list(mol)
    q = q[[max(Ls[a], Ls[b], Ls[c], Ls[d]) == 3 for a, b, c, d in q]]
    rng = np.random.default_rng(9)
    q = q[np.sort(rng.choice(len(q), size=300, replace=False))]
    vals, offs = blocks(rb, q)
    np.savez_compressed(os.path.join(OUT, "cfg2f.npz"), S=S, T=T, V=V, D=D, J=o["J"], K=o["K"],
                        quartets=q, eri=vals, eri_off=offs, schwarz=rb.schwarz())


def main():
    mol = M.cfg0()
    D = M.cfg0_density()
    rb = ref.RefBasis(mol)
    S, T, V = rb.onee(screening=True)
    o = rb.jk(D, schwarz=1e-12)
    o0 = rb.jk(D, schwarz=0.0)
    q = quartet_list(mol)
    vals, offs = blocks(rb, q)
    np.savez_compressed(os.path.join(OUT, "cfg0.npz"), S=S, T=T, V=V, D=D, J=o["J"], K=o["K"], G=o["G"],
                        J0=o0["J"], K0=o0["K"], quartets=q, eri=vals, eri_off=offs, schwarz=rb.schwarz())

    mol1 = M.cfg1()
    D1 = M.density_for("cfg1", mol1)
    rb1 = ref.RefBasis(mol1)
    S1, T1, V1 = rb1.onee(screening=True)
    o1 = rb1.jk(D1, schwarz=1e-12, want=("J", "K"))
    q1 = quartet_list(mol1, max_n=200, seed=7)
    v1, off1 = blocks(rb1, q1)
    np.savez_compressed(os.path.join(OUT, "cfg1.npz"), S=S1, T=T1, V=V1, J=o1["J"], K=o1["K"],
                        quartets=q1, eri=v1, eri_off=off1, schwarz=rb1.schwarz())

    xs = np.concatenate([[0.0, 1e-16, 1e-8, 0.01, 0.005, 0.5, 1.0, 11.99, 12.0, 12.01, 25.0, 39.99, 40.0,
                          40.01, 45.0, 60.0, 100.0, 1e3, 1e4]],
                        ).astype(np.float64)
    rng = np.random.default_rng(11)
    xs = np.concatenate([xs, rng.uniform(0, 50, 200)])
    orders = np.arange(0, 17)
    F = np.array([[ref.boys_single(int(n), float(x)) for n in orders] for x in xs])
    np.savez_compressed(os.path.join(OUT, "boys.npz"), x=xs, orders=orders, F=F)

    Ts = np.concatenate([[0.0, 1e-12, 0.005, 0.01, 1.0, 28.99, 29.0, 36.99, 37.0, 75.99, 76.0, 100.0, 120.0],
                         rng.uniform(0, 80, 150)])
    R = np.zeros((9, len(Ts), 9))
    W = np.zeros((9, len(Ts), 9))
    for n in range(1, 10):
        for k, t in enumerate(Ts):
            r, w = ref.rys_roots(n, float(t))
            R[n - 1, k, :n] = r
            W[n - 1, k, :n] = w
    np.savez_compressed(os.path.join(OUT, "rys.npz"), T=Ts, roots=R, weights=W)
    write_cfg2f()
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()

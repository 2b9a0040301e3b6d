"""Writes tests/golden/cfg2.npz from the UNMODIFIED reference engine
(oracle/_ref): the full cfg2 molecule (60 atoms, shells up to f, M = 1480)
at Schwarz 1e-12 with its standard density (molecules.density_for("cfg2")),
J and K from build_coulomb_j / build_exchange_k on one core.  The matrices
are 17.5 MB each, so the fixture keeps what the GPU tests compare: the
energy terms tr(D J), tr(D K), the row sums of J and K, and 4096 sampled
elements of each (fixed positions, seed 7).  One reference build takes
tens of minutes, which is why the result is stored.

    python tests/golden/make_cfg2_golden.py
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from origo_tlno_b200 import molecules as M  # noqa: E402


def main():
    mol = M.cfg2()
    D = M.density_for("cfg2", mol)
    t0 = time.time()
    o = ref.RefBasis(mol).jk(D, schwarz=1e-12, want=("J", "K"))
    secs = time.time() - t0
    rng = np.random.default_rng(7)
    idx = rng.integers(0, mol.n_sph, size=(4096, 2))
    J, K = o["J"], o["K"]
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "cfg2.npz"),
                        trDJ=np.sum(D * J), trDK=np.sum(D * K), J_rows=J.sum(axis=1), K_rows=K.sum(axis=1),
                        idx=idx, J_samples=J[idx[:, 0], idx[:, 1]], K_samples=K[idx[:, 0], idx[:, 1]],
                        reference_seconds=secs)
    print(f"cfg2 reference J+K: {secs:.1f} s")


if __name__ == "__main__":
    main()

"""The C++ shim that keeps the reference's J/K signatures over the C ABI
(tests/shim/tlno_b200_shim.hpp), compiled against the reference's own headers
into oracle/_ref/shim_test by oracle/build_ref.sh: the reference's
fock::build_coulomb_j / build_exchange_k / build_rhf_g (plain and
density-screened), its EriDirectJKIncrementalState and the same calls
through the shim must agree to 1e-12, with identical status sequences and
error texts."""
import json
import os
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT
from origo_tlno_b200 import molecules as M

pytestmark = pytest.mark.gpu

SHIM = os.path.join(ROOT, "oracle", "_ref", "shim_test")


def _write_shells(mol, path):
    with open(path, "w") as f:
        f.write(f"{len(mol.shells)}\n")
        for s in mol.shells:
            head = " ".join(repr(float(x)) for x in s.center) + f" {int(s.L)} {len(s.exponents)} "
            f.write(head + " ".join(repr(float(x)) for x in [*s.exponents, *s.coefficients]) + "\n")


@pytest.mark.parametrize("name", ["cfg1", "water8"])
def test_cpp_shim_matches_reference(name, tmp_path):
    if not os.path.exists(SHIM):
        pytest.skip("shim test program not built (oracle/build_ref.sh)")
    mol = M.cfg1() if name == "cfg1" else M.water_cluster(8, seed=5)
    path = tmp_path / "shells.txt"
    _write_shells(mol, path)
    tau = "1e-12" if name == "cfg1" else "1e-11"
    r = subprocess.run([SHIM, str(path), tau, "1e-10"], capture_output=True, text=True, timeout=600)
    print(r.stdout, r.stderr)
    lines = r.stdout.strip().splitlines()
    assert lines, r.stderr
    res = json.loads(lines[-1])
    assert r.returncode == 0 and "error" not in res, res
    assert res["M"] == mol.n_sph
    assert res["incremental_status_match"] and res["same_error_text"]
    assert max(res["J"], res["K"], res["G"], res["G_density_screened"], res["incremental_G"]) < 1e-12

"""CPU tests (no GPU): the oracles against the reference's golden vectors,
the C-ABI library surface, host-side validation and the multi-process
replica plumbing (gloo, world size 2)."""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from tests.conftest import ROOT, load_golden
from origo_tlno_b200 import molecules as M

HEADER = os.path.join(ROOT, "include", "tlno_gpu.h")
LIB = os.path.join(ROOT, "origo_tlno_b200", "_lib", "libtlno_gpu.so")


def _declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tlno_gpu_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "native library not built (python -m origo_tlno_b200.build)"
    lib = ctypes.CDLL(LIB)
    names = _declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    from origo_tlno_b200 import _native as N
    assert set(N.EXPORTED) == set(names)


def test_library_fails_loudly_without_a_device():
    from origo_tlno_b200 import _native as N
    n = ctypes.c_int(-1)
    N.check(N.lib().tlno_gpu_device_count(ctypes.byref(n)))
    if n.value > 0:
        pytest.skip("a CUDA device is present")
    from origo_tlno_b200 import engine as E
    with pytest.raises(E.TlnoError, match="no CUDA device"):
        E.Context(M.cfg0())
    with pytest.raises(E.TlnoError, match="no CUDA device"):
        E.boys([1.0], 2)


def test_basis_validation_before_device_use():
    from origo_tlno_b200 import _native as N
    import ctypes as C
    centers = np.zeros(3)
    L = np.array([5], dtype=np.int32)
    nprim = np.array([1], dtype=np.int32)
    e = np.array([1.0])
    c = np.array([1.0])
    Z = np.array([1], dtype=np.int32)
    h = C.c_void_p()
    rc = N.lib().tlno_gpu_create(1, centers.ctypes.data, L.ctypes.data, nprim.ctypes.data, e.ctypes.data,
                                 c.ctypes.data, 1, Z.ctypes.data, centers.ctypes.data, 0, C.byref(h))
    assert rc == N.E_INVALID
    assert "L=0..4" in N.lib().tlno_gpu_last_error().decode()
    L[0] = 0
    e[0] = -1.0
    rc = N.lib().tlno_gpu_create(1, centers.ctypes.data, L.ctypes.data, nprim.ctypes.data, e.ctypes.data,
                                 c.ctypes.data, 1, Z.ctypes.data, centers.ctypes.data, 0, C.byref(h))
    assert rc == N.E_INVALID
    assert "positive" in N.lib().tlno_gpu_last_error().decode()
    e[0] = 1.0
    centers[1] = np.nan
    rc = N.lib().tlno_gpu_create(1, centers.ctypes.data, L.ctypes.data, nprim.ctypes.data, e.ctypes.data,
                                 c.ctypes.data, 1, Z.ctypes.data, np.zeros(3).ctypes.data, 0, C.byref(h))
    assert rc == N.E_INVALID
    assert "finite" in N.lib().tlno_gpu_last_error().decode()


# ---------------- oracle restatement (oracle/tlno_oracle.cpp) ----------------

@pytest.fixture(scope="module")
def port():
    from oracle import port as P
    if not P.available():
        subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile")], check=True)
    return P


def test_port_boys_against_golden(port):
    g = load_golden("boys.npz")
    F = np.array([[port.boys(int(n), float(x)) for n in g["orders"]] for x in g["x"]])
    rel = np.abs(F - g["F"]) / np.maximum(np.abs(g["F"]), 1e-300)
    assert rel.max() < 2e-13


def test_port_boys_against_mpmath(port):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.dps = 60
    for x in (0.0, 1e-12, 0.3, 2.0, 11.99, 12.0, 25.0, 39.99, 45.0, 120.0):
        for n in (0, 1, 3, 8, 16):
            exact = mpmath.quad(lambda t: t ** (2 * n) * mpmath.e ** (-x * t * t), [0, 1])
            got = port.boys(n, x)
            assert abs(got - float(exact)) <= 2e-13 * abs(float(exact)), (n, x)


def test_port_rys_against_golden(port):
    g = load_golden("rys.npz")
    for n in range(1, 10):
        for k, t in enumerate(g["T"]):
            r, w = port.rys_roots(n, float(t))
            assert np.max(np.abs(r - g["roots"][n - 1, k, :n])) < 1e-12
            assert np.max(np.abs(w - g["weights"][n - 1, k, :n])) < 1e-12


def test_port_rys_moments(port):
    # sum_i w_i r_i^k = F_k(T) for k < 2N (the reference's own self-check,
    # rys_engine.ipp:3628-3646)
    for n in (1, 3, 5, 7):
        for t in (0.0, 0.7, 5.0, 21.0, 80.0):
            r, w = port.rys_roots(n, t)
            for k in range(2 * n):
                mu = port.boys(k, t)
                assert abs(np.sum(w * r ** k) - mu) <= max(1e-13, 2e-11 * abs(mu))


def test_port_cfg0_against_golden(port):
    g = load_golden("cfg0.npz")
    pb = port.PortBasis(M.cfg0())
    S, T, V = pb.onee()
    assert np.max(np.abs(S - g["S"])) < 1e-12
    assert np.max(np.abs(T - g["T"])) < 1e-12
    assert np.max(np.abs(V - g["V"])) < 1e-12
    o = pb.jk(g["D"])
    assert np.max(np.abs(o["J"] - g["J"])) < 1e-12
    assert np.max(np.abs(o["K"] - g["K"])) < 1e-12
    assert np.max(np.abs(pb.schwarz() - g["schwarz"])) < 1e-12
    for k, (a, b, c, d) in enumerate(g["quartets"]):
        ref = g["eri"][g["eri_off"][k]:g["eri_off"][k + 1]]
        assert np.max(np.abs(pb.eri_block(a, b, c, d).ravel() - ref)) < 1e-12


def test_port_cfg1_eri_sample_against_golden(port):
    g = load_golden("cfg1.npz")
    pb = port.PortBasis(M.cfg1())
    for k in range(0, len(g["quartets"]), 10):
        a, b, c, d = g["quartets"][k]
        ref = g["eri"][g["eri_off"][k]:g["eri_off"][k + 1]]
        assert np.max(np.abs(pb.eri_block(a, b, c, d).ravel() - ref)) < 1e-12


def test_port_cfg2_fragment_f_shells_against_golden(port):
    # shells up to f: ERI blocks holding an f shell and the one-electron
    # matrices of the restatement against the reference's fixture
    g = load_golden("cfg2f.npz")
    pb = port.PortBasis(M.cfg2_fragment())
    for k in range(0, len(g["quartets"]), 5):
        a, b, c, d = g["quartets"][k]
        ref = g["eri"][g["eri_off"][k]:g["eri_off"][k + 1]]
        assert np.max(np.abs(pb.eri_block(a, b, c, d).ravel() - ref)) < 1e-12
    S, T, V = pb.onee()
    assert np.max(np.abs(S - g["S"])) < 1e-12
    assert np.max(np.abs(T - g["T"])) < 1e-12
    assert np.max(np.abs(V - g["V"])) < 1e-12


def test_port_against_compiled_reference_small(port):
    from oracle import ref
    if not ref.available():
        pytest.skip("compiled reference not built here")
    mol = M.water_cluster(2, seed=5)
    D = M.random_density(mol.n_sph, 5, seed=3)
    rb = ref.RefBasis(mol)
    pb = port.PortBasis(mol)
    o_ref = rb.jk(D, schwarz=1e-12, want=("J", "K"))
    o = pb.jk(D, tau=1e-12)
    assert np.max(np.abs(o["J"] - o_ref["J"])) < 1e-12
    assert np.max(np.abs(o["K"] - o_ref["K"])) < 1e-12
    assert np.max(np.abs(pb.schwarz() - rb.schwarz())) < 1e-12


def test_golden_fixture_self_consistency():
    g = load_golden("cfg0.npz")
    assert np.max(np.abs(g["G"] - (g["J"] - 0.5 * g["K"]))) < 1e-13
    for X in ("S", "T", "V", "J", "K"):
        assert np.max(np.abs(g[X] - g[X].T)) < 1e-13


# ---------------- host logic ----------------

def test_molecule_generators_are_deterministic_and_sized():
    a, b = M.cfg1(), M.cfg1()
    assert a.n_sph == 246 and len(a.shells) == 114
    assert np.array_equal(a.coords, b.coords)
    assert M.cfg2().n_sph == 1480
    w = M.cfg4()
    assert w.n_sph == 9600 and len(w.charges) == 1200
    ms = M.cfg3(8)
    assert len(ms) == 8 and all(3 <= len(m.charges) <= 30 for m in ms)
    d = np.min([np.linalg.norm(p - q) for i, p in enumerate(a.coords) for q in a.coords[:i]])
    assert d >= 1.0 * M.ANGSTROM_TO_BOHR - 1e-9


def test_replica_throughput_arithmetic():
    from origo_tlno_b200 import replicas
    assert replicas.throughput(100.0, 2.0, 4) == 200.0
    assert replicas.max_over_ranks([1.0, 2.0]) == [1.0, 2.0]


_GLOO_SCRIPT = r"""
import os, sys
sys.path.insert(0, {root!r})
import torch.distributed as dist
from origo_tlno_b200 import replicas
replicas.init("gloo", timeout_s=60)
ws, rank, _ = replicas.world()
t = replicas.max_over_ranks([1.0 + rank, 5.0 - rank])
assert t == [2.0, 5.0], t
v = replicas.throughput(10.0, t[0], ws)
assert v == 10.0, v
dist.barrier()
dist.destroy_process_group()
print("ok", rank)
"""


def test_replicas_gloo_world_size_2(tmp_path):
    script = tmp_path / "r.py"
    script.write_text(_GLOO_SCRIPT.format(root=ROOT))
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT="29517")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", "29517", str(script)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=240, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("ok") == 2, r.stdout


# ---------------- oracle harness: screening, incremental state, ERI stream ----------------

@pytest.fixture(scope="module")
def refw3():
    from oracle import ref
    if not ref.available():
        pytest.skip("compiled reference not built here")
    mol = M.water_cluster(3, seed=5)
    return ref, mol, ref.RefBasis(mol)


def test_ref_harness_screening_entries(refw3):
    ref, mol, rb = refw3
    D = M.random_density(mol.n_sph, 6, seed=11)
    base = rb.jk(D, schwarz=1e-12)
    same = rb.jk_opts(D, schwarz=1e-12)
    for k in ("J", "K", "G"):
        assert np.array_equal(base[k], same[k])
    # the compatibility endpoint builds the same G as the facade
    assert np.max(np.abs(rb.jk_compat(D, schwarz=1e-12) - base["G"])) < 1e-13
    # a density threshold removes quartets (results change, stay close)
    scr = rb.jk_opts(D, schwarz=1e-12, density_threshold=1e-7)
    d = np.max(np.abs(scr["J"] - base["J"]))
    assert 0.0 < d < 1e-5
    with pytest.raises(RuntimeError, match="heuristic decay"):
        rb.jk_opts(D, schwarz=0.0, decay=1e-10, density_threshold=1e-9)
    with pytest.raises(RuntimeError, match="exactly one shell-level metric"):
        rb.jk_opts(D, schwarz=1e-12, decay=1e-10)
    cs, secs = rb.eri_checksum(schwarz=0.0)
    assert np.isfinite(cs) and secs >= 0.0


def test_ref_harness_incremental_state(refw3):
    ref, mol, rb = refw3
    D0 = M.random_density(mol.n_sph, 6, seed=12)
    D1 = D0 + 1e-3 * M.random_density(mol.n_sph, 6, seed=13)
    st = ref.RefIncremental(rb, schwarz=1e-12, exact_rebuild_interval=2)
    r0 = st.update(D0)
    assert r0["status"] == "exact_rebuild" and r0["counters"] == [1, 1, 0, 0]
    assert np.max(np.abs(r0["G"] - rb.jk(D0, schwarz=1e-12)["G"])) < 1e-13
    r1 = st.update(D1)
    assert r1["status"] == "incremental_update" and r1["counters"] == [2, 1, 1, 0]
    assert np.max(np.abs(r1["G"] - rb.jk(D1, schwarz=1e-12)["G"])) < 1e-12
    r2 = st.update(D1)
    assert r2["status"] == "skipped_unchanged" and r2["counters"] == [3, 1, 1, 1]


def test_ref_harness_components_round_trip(refw3):
    ref, mol, rb = refw3
    centers, ang, nprim, exps, coefs = rb.components()
    assert len(nprim) == mol.n_cart == rb.n_cart
    assert np.all(ang.sum(axis=1) >= 0) and len(exps) == int(nprim.sum()) == len(coefs)


# ---------------- front end: .inp reader and named bases ----------------

REF_ROOT = os.environ.get("TLNO_REFERENCE_ROOT", "/root/reference")
MOLDIR = os.path.join(REF_ROOT, "test_molecules")


def _gaussian94_from_reference(ref, symbols, basis):
    """A Gaussian94 basis file written from the reference's raw tables (one
    contracted shell per run of Cartesian components of one L)."""
    names = "SPDFG"
    out = []
    for sym in sorted(set(symbols)):
        _, raw = ref.raw_atom_basis(sym, basis)
        out.append(f"{sym}     0")
        for ang, e, c in raw:
            L = sum(ang)
            if ang != (L, 0, 0):
                continue  # the first component of each shell carries the shell
            out.append(f"{names[L]}   {len(e)}   1.00")
            out += [f"  {float(x)!r}  {float(y)!r}" for x, y in zip(e, c)]
        out.append("****")
    return "\n".join(out) + "\n"


@pytest.mark.skipif(not os.path.isdir(MOLDIR), reason="reference test molecules not present")
def test_frontend_reader_matches_reference_on_every_input():
    from oracle import ref
    if not ref.available():
        pytest.skip("compiled reference not built here")
    from origo_tlno_b200 import frontend as F
    files = sorted(f for f in os.listdir(MOLDIR) if f.endswith(".inp"))
    assert len(files) >= 30
    for f in files:
        path = os.path.join(MOLDIR, f)
        mine = F.read_inp_file(path)
        sym, xyz, ch, mu = ref.read_inp(path)
        assert mine.symbols == sym, f
        assert np.array_equal(np.array(mine.coords_bohr), xyz), f
        assert (mine.charge, mine.multiplicity) == (ch, mu), f


def test_frontend_reader_errors(tmp_path):
    from origo_tlno_b200 import frontend as F
    p = tmp_path / "m.inp"
    p.write_text("* xyz 0 1\nO 0 0 0\n")
    with pytest.raises(F.FrontendError, match="Unterminated xyz block"):
        F.read_inp_file(str(p))
    p.write_text("* xyz 0 0\nO 0 0 0\n*\n")
    with pytest.raises(F.FrontendError, match="multiplicity must be at least one"):
        F.read_inp_file(str(p))
    p.write_text("* xyz 0 1\nO 0 nan 0\n*\n")
    with pytest.raises(F.FrontendError, match="bad coordinate line 2"):
        F.read_inp_file(str(p))
    p.write_text("O 0 0 0\n")
    with pytest.raises(F.FrontendError, match="Missing"):
        F.read_inp_file(str(p))
    with pytest.raises(F.FrontendError, match="Unsupported basis set: cc-pvdz"):
        F.parse_basis_kind("cc-pvdz")
    assert F.parse_basis_kind("6-31G**") == "6-31g(d,p)" and F.parse_basis_kind("def2-dzvp") == "def2-svp"


@pytest.mark.skipif(not os.path.isdir(MOLDIR), reason="reference test molecules not present")
@pytest.mark.parametrize("name,basis", [("h2o", "def2-svp"), ("glucose", "def2-svp"), ("caffeine", "def2-tzvp"),
                                        ("benzene", "6-31g**"), ("co", "sto-3g")])
def test_frontend_named_basis_matches_build_basis_general(name, basis):
    """A Gaussian94 file of the named basis, read by the front end and
    normalised by make_shell, reproduces the reference's build_basis_general
    component records (so the engine sees the reference's basis)."""
    from oracle import ref
    if not ref.available():
        pytest.skip("compiled reference not built here")
    from origo_tlno_b200 import frontend as F
    for kind in ("sto-3g", "def2-svp", "def2-tzvp", "6-31g**"):
        assert ref.parse_basis_kind_ok(kind)
    inp = F.read_inp_file(os.path.join(MOLDIR, name + ".inp"))
    spec = F.molecule_spec(inp)
    lib = F.load_basis_library(_gaussian94_from_reference(ref, spec.symbols, basis))
    mol, electrons = F.build_basis_general(spec, lib, name=name)
    (c_ref, a_ref, n_ref, e_ref, k_ref), Z, el_ref = ref.basis_general(spec.symbols, spec.coords, spec.charge, basis)
    assert electrons == el_ref and np.array_equal(mol.charges, Z)
    c, a, n, e, k = ref.RefBasis(mol).components()
    assert np.array_equal(a, a_ref) and np.array_equal(n, n_ref)
    assert np.array_equal(c, c_ref) and np.array_equal(e, e_ref)
    assert np.max(np.abs(k - k_ref) / np.abs(k_ref)) < 1e-14


def _trials(ms, err):
    return [{"ms": m, "max_abs_dJ": e, "max_abs_dK": e, "abs_dE": e} for m, e in zip(ms, err)]


def test_budget_allocation_keeps_unprofitable_classes_fp64():
    # per-class split allocation of the mixed path: a class whose FP32 split
    # saves no time stays at its first trial (FP64 only, one launch); the
    # summed per-class errors stay inside the tolerances
    from origo_tlno_b200.autotune import allocate_budget
    rows = [
        {"trials": _trials([10.0, 8.0, 6.0, 5.0], [0.0, 1e-9, 1e-8, 1e-7]), "pick": 0},  # profitable
        {"trials": _trials([4.0, 4.2, 4.5, 5.0], [0.0, 1e-10, 1e-9, 1e-8]), "pick": 0},  # FP32 slower
        {"trials": _trials([7.0, 5.0, 4.0, 3.0], [0.0, 5e-9, 2e-8, 9e-8]), "pick": 0},   # profitable
    ]
    sJ, sK, sE = allocate_budget(rows, tol_energy=1e-7, tol_jk=3e-8)
    assert rows[1]["pick"] == 0
    assert rows[0]["pick"] > 0 and rows[2]["pick"] > 0
    assert sJ <= 3e-8 and sK <= 3e-8 and sE <= 1e-7
    picked = sum(r["trials"][r["pick"]]["max_abs_dJ"] for r in rows)
    assert abs(picked - sJ) < 1e-20


def test_budget_allocation_without_budget_keeps_everything_fp64():
    from origo_tlno_b200.autotune import allocate_budget
    rows = [{"trials": _trials([10.0, 5.0], [0.0, 1e-6]), "pick": 0} for _ in range(3)]
    sJ, sK, sE = allocate_budget(rows, tol_energy=1e-7, tol_jk=1e-8)
    assert all(r["pick"] == 0 for r in rows) and sJ == sK == sE == 0.0

"""The allocation-free ERI-block entry point (tlno_gpu_eri_blocks_noalloc).

Some callers cannot allocate device memory themselves: code that lives
inside a device-memory budget owned by another allocator, or on a
latency-critical path where an allocation could synchronise the device.
This entry point serves them: it writes the same blocks as
tlno_gpu_eri_blocks into caller-owned device memory and keeps its own
scratch in one fixed device array instead of allocating.  This test calls it
through the C ABI twice in a row and checks both results against the
allocating entry point at the 1e-12 tolerance of the ERI parity tests.  It
sits in its own file, collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from origo_tlno_b200 import _native as N
from origo_tlno_b200 import engine as E
from origo_tlno_b200 import molecules as M

pytestmark = pytest.mark.gpu


def test_noalloc_blocks_match_allocating_entry_point_twice():
    import torch

    mol = M.cfg1()
    ctx = E.Context(mol)
    ns = len(mol.shells)
    rng = np.random.default_rng(3)
    quartets = np.ascontiguousarray(rng.integers(0, ns, size=(64, 4)), dtype=np.int32)
    Ls = [s.L for s in mol.shells]
    sizes = [(2 * Ls[a] + 1) * (2 * Ls[b] + 1) * (2 * Ls[c] + 1) * (2 * Ls[d] + 1) for a, b, c, d in quartets]
    offsets = np.zeros(len(quartets), dtype=np.int64)
    offsets[1:] = np.cumsum(sizes)[:-1]
    total = int(sum(sizes))

    expected = np.concatenate([b.ravel() for b in ctx.eri_blocks(quartets)])

    lib = N.lib()
    outs = [torch.full((total,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    free = []
    for d_out in outs:
        free.append(torch.cuda.mem_get_info()[0])
        rc = lib.tlno_gpu_eri_blocks_noalloc(ctx.h, len(quartets), quartets.ctypes.data, offsets.ctypes.data,
                                             C.c_void_p(d_out.data_ptr()))
        N.check(rc)
        free.append(torch.cuda.mem_get_info()[0])
        got = d_out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert float(np.max(np.abs(got - expected))) < 1e-12
    # the calls take no device memory: free memory is the same before and
    # after each of them
    assert free[0] == free[1] and free[2] == free[3], free
    ctx.close()


def test_noalloc_blocks_match_the_reference_fixture():
    """The entry point's blocks against the reference's own blocks (the
    golden fixture written from the compiled reference)."""
    import torch
    from tests.conftest import load_golden

    g = load_golden("cfg1.npz")
    ctx = E.Context(M.cfg1())
    q = np.ascontiguousarray(g["quartets"], dtype=np.int32)
    offsets = np.ascontiguousarray(g["eri_off"][:-1], dtype=np.int64)
    total = int(g["eri_off"][-1])
    d_out = torch.zeros(total, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    N.check(N.lib().tlno_gpu_eri_blocks_noalloc(ctx.h, len(q), q.ctypes.data, offsets.ctypes.data,
                                                C.c_void_p(d_out.data_ptr())))
    err = float(np.max(np.abs(d_out.cpu().numpy() - g["eri"][:total])))
    print(f"PIN noalloc_vs_reference_blocks max_abs={err:.2e}")
    assert err < 1e-12
    ctx.close()


def test_noalloc_rejects_requests_beyond_the_scratch():
    import torch

    mol = M.cfg1()
    ctx = E.Context(mol)
    # the most contracted shell, many times over: needs more than the 8 MiB scratch
    big = int(np.argmax([len(s.exponents) for s in mol.shells]))
    quartets = np.full((20000, 4), big, dtype=np.int32)
    offsets = np.zeros(len(quartets), dtype=np.int64)
    d_out = torch.zeros(16, dtype=torch.float64, device="cuda")
    rc = N.lib().tlno_gpu_eri_blocks_noalloc(ctx.h, len(quartets), quartets.ctypes.data, offsets.ctypes.data,
                                             C.c_void_p(d_out.data_ptr()))
    assert rc == N.E_INVALID
    assert "scratch" in N.lib().tlno_gpu_last_error().decode()
    ctx.close()

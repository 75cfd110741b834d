"""imc_comb_noalloc (scratch in a fixed device array inside the library) against imc_comb
(scratch in a caller workspace), both called through the C ABI on identical banks.

Two calls in a row with different meshes, bank sizes and bin layouts, so the second call
reuses the scratch the first one left behind.  Tolerance: copies, cells, groups and
weights exact (same kernels on the same inputs); per-bin comb discrepancy within 1e-9 of
the bank's energy (FP64 atomics may add in another order).  The file sorts last so the
set-up inside the first call also runs after everything else in the session.
"""
import ctypes

import numpy as np
import pytest
import torch

from radtranbook_b200 import _lib
from radtranbook_b200.engine import Bank

pytestmark = pytest.mark.gpu

NOALLOC_SCRATCH_BYTES = 8 << 20  # IMC_NOALLOC_SCRATCH_BYTES


def _mesh(nx, ny, ng, dev):
    e1 = torch.linspace(0.0, 1.0, nx + 1, dtype=torch.float64, device=dev)
    e2 = torch.linspace(0.0, 2.0, ny + 1, dtype=torch.float64, device=dev)
    vol = torch.full((nx * ny,), (1.0 / nx) * (2.0 / ny), dtype=torch.float64, device=dev)
    ge = torch.logspace(-2, 1, ng + 1, dtype=torch.float64, device=dev) if ng > 1 else None
    keep = (e1, e2, vol, ge)
    m = _lib.ImcMesh(2, nx, ny, ng, e1.data_ptr(), e2.data_ptr(), vol.data_ptr(),
                     ge.data_ptr() if ge is not None else None)
    return m, keep


def _bank(n, nbins_cell, ng, seed, dev):
    rng = np.random.default_rng(seed)
    b = Bank(n + 16, dev, multigroup=ng > 1)
    f = lambda: rng.uniform(0, 1, n)  # noqa: E731
    b.load(rng.uniform(0.1, 2.0, n), f(), f(), np.zeros(n), f(), f(), rng.integers(0, nbins_cell, n),
           rng.integers(0, ng, n) if ng > 1 else None)
    return b


def _comb_both(lib, dev, nx, ny, ng, n, n_max, step, per_group, seed):
    mesh, keep = _mesh(nx, ny, ng, dev)
    nc = nx * ny
    src = _bank(n, nc, ng, seed, dev)
    stream = torch.cuda.current_stream().cuda_stream
    nb = nc * ng

    # existing entry point, caller workspace
    out_ws = Bank(int(1.3 * n_max) + 2 * nb + 1024, dev, multigroup=ng > 1)
    ws = torch.empty(lib.imc_workspace_bytes(ctypes.byref(mesh), src.size), dtype=torch.uint8, device=dev)
    disc_ws = torch.zeros(nb, dtype=torch.float64, device=dev)
    rep_ws = _lib.ImcCombReport()
    cin, cout = src.c(), out_ws.c()
    _lib.check("imc_comb", lib.imc_comb(ctypes.byref(mesh), ctypes.byref(cin), ctypes.byref(cout), n_max, 77,
                                        step, per_group, disc_ws.data_ptr(), ws.data_ptr(), ws.numel(),
                                        ctypes.byref(rep_ws), stream))
    out_ws.size = int(cout.size)

    # no-alloc entry point
    out_na = Bank(out_ws.capacity, dev, multigroup=ng > 1)
    disc_na = torch.zeros(nb, dtype=torch.float64, device=dev)
    rep_na = _lib.ImcCombReport()
    cin, cout = src.c(), out_na.c()
    _lib.check("imc_comb_noalloc", lib.imc_comb_noalloc(ctypes.byref(mesh), ctypes.byref(cin), ctypes.byref(cout),
                                                        n_max, 77, step, per_group, disc_na.data_ptr(),
                                                        ctypes.byref(rep_na), stream))
    out_na.size = int(cout.size)
    del keep

    assert rep_na.n_in == rep_ws.n_in == n
    assert rep_na.n_out == rep_ws.n_out == out_ws.size == out_na.size
    assert rep_na.n_out > 0
    for k in ("cell", "weight", "pos1", "pos2", "dir1", "dir2", "time") + (("group",) if ng > 1 else ()):
        torch.testing.assert_close(out_na.view(k), out_ws.view(k), rtol=0, atol=0)
    e_tot = float(src.view("weight").double().sum())
    np.testing.assert_allclose(rep_na.energy_before, rep_ws.energy_before, rtol=1e-12)
    np.testing.assert_allclose(rep_na.energy_after, rep_ws.energy_after, rtol=1e-12)
    torch.testing.assert_close(disc_na, disc_ws, rtol=0, atol=1e-9 * e_tot)
    return rep_na


def test_noalloc_comb_matches_workspace_comb_twice(cuda):
    lib = _lib.load()
    # call 1: gray, per-cell bins
    _comb_both(lib, cuda, 12, 20, 1, 40000, 15000, 3, 0, seed=1)
    # call 2: multigroup, per-(cell, group) bins, larger bank: the scratch of call 1 is reused
    _comb_both(lib, cuda, 16, 16, 6, 90000, 30000, 4, 1, seed=2)


def test_noalloc_comb_rejects_inputs_beyond_its_scratch(cuda):
    lib = _lib.load()
    mesh, keep = _mesh(12, 20, 1, cuda)
    src = _bank(64, 240, 1, 3, cuda)
    out = Bank(1024, cuda)
    cin, cout = src.c(), out.c()
    n_big = 4 * NOALLOC_SCRATCH_BYTES // 4  # one 4-byte count per entry already exceeds the array
    cin.size = n_big
    cin.capacity = n_big
    assert lib.imc_workspace_bytes(ctypes.byref(mesh), n_big) > NOALLOC_SCRATCH_BYTES
    disc = torch.zeros(240, dtype=torch.float64, device=cuda)
    rep = _lib.ImcCombReport()
    st = lib.imc_comb_noalloc(ctypes.byref(mesh), ctypes.byref(cin), ctypes.byref(cout), 100, 77, 0, 0,
                              disc.data_ptr(), ctypes.byref(rep), torch.cuda.current_stream().cuda_stream)
    assert st == 8, _lib.load().imc_status_str(st)  # IMC_ERR_WORKSPACE, nothing launched
    assert lib.imc_status_str(st) == b"workspace too small"
    assert int(cout.size) == 0 and rep.n_out == 0
    del keep

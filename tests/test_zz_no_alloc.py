"""drape_pcg_noalloc: block-Jacobi PCG for callers that cannot allocate GPU memory (applications that hand every
device buffer out of their own pool, or that must stay out of the driver's allocator while running).

The test plays such a caller: it owns the matrix, right-hand side and solution buffers (allocated here with
torch, as the caller's own pool would) and asks the library to solve without it allocating anything. Two calls
in a row, on two different systems, must each agree with the allocating entry point drape_pcg on the same
system (same iteration count +-1, solutions within 1e-5) and with the f64 oracle's solution (within 1e-4), and
the device's free memory must not change across the call. info is passed with exactly the three entries the
header documents.
This file is collected last so that a failing run stopped at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

from drape_b200 import api
from tests import oracle_py

pytestmark = pytest.mark.gpu
P = ctypes.c_void_p


def _entry():
    lib = api.load()
    fn = lib.drape_pcg_noalloc
    fn.argtypes = [ctypes.c_int32, P, P, P, P, P, P, P, ctypes.c_double, ctypes.c_int32, P, P, P]
    fn.restype = ctypes.c_int
    return lib, fn


def _solve_noalloc(torch, rp, ci, vals, rhs, rtol, maxit, measure_memory=False):
    lib, fn = _entry()
    R, B = len(rp) - 1, len(ci)
    dev = torch.device("cuda", 0)
    blocks = torch.tensor(vals.astype(np.float32).reshape(B, 9), device=dev)
    a0 = blocks[:, 0:4].contiguous()
    a1 = blocks[:, 4:8].contiguous()
    a2 = blocks[:, 8].contiguous()
    b4 = torch.zeros(R, 4, dtype=torch.float32, device=dev)
    b4[:, :3] = torch.tensor(rhs.astype(np.float32).reshape(R, 3), device=dev)
    x4 = torch.full((R, 4), float("nan"), dtype=torch.float32, device=dev)  # the solve must overwrite it
    row_ptr = torch.tensor(np.asarray(rp, np.int32), device=dev)
    col_idx = torch.tensor(np.asarray(ci, np.int32), device=dev)
    info = np.zeros(3, np.int32)
    rel = ctypes.c_double()
    torch.cuda.synchronize()
    # the caller's buffers are all in place: the device's free memory just before and just after the call
    free_before = torch.cuda.mem_get_info(0)[0] if measure_memory else None
    st = fn(R, P(row_ptr.data_ptr()), P(col_idx.data_ptr()), P(a0.data_ptr()), P(a1.data_ptr()), P(a2.data_ptr()),
            P(b4.data_ptr()), P(x4.data_ptr()), rtol, maxit, None, info.ctypes.data_as(P), ctypes.byref(rel))
    assert st == 0, lib.drape_last_error(None).decode()
    free_after = torch.cuda.mem_get_info(0)[0] if measure_memory else None
    x = x4[:, :3].reshape(-1).double().cpu().numpy()
    return ((x, free_before, free_after) if measure_memory else x), int(info[0]), int(info[1])


def _check_against_both(torch, rp, ci, vals, rhs, label, measure_memory=False):
    """One no-alloc solve checked against drape_pcg (iterations +-1, solution within 1e-5) and against the f64
    oracle's own PCG solution of the same system (within 1e-4: f32 against f64). With measure_memory, the device's
    free memory is read just before and after the call: the entry point must not take any."""
    R = len(rp) - 1
    ref_ctx = api.Drape.from_arrays(np.zeros(3 * R), np.arange(R), np.ones(R), rp, ci)
    x_ref, info_ref = ref_ctx.pcg(rhs, 1e-7, 20000, blocks=vals.astype(np.float32))
    ref_ctx.close()
    x64, info64 = oracle_py.pcg(rp, ci, vals, rhs, 1e-10, 20000)
    assert info64["converged"], label
    x_new, iters, status = _solve_noalloc(torch, rp, ci, vals, rhs, 1e-7, 20000, measure_memory=measure_memory)
    if measure_memory:
        x_new, free_before, free_after = x_new
        # The driver hands out device memory in 2 MiB pages; any allocation by the call shows up as a whole page.
        assert abs(free_before - free_after) < (2 << 20), (label, free_before, free_after)
    assert status == 1 and info_ref["status"] == "converged", label
    assert abs(iters - info_ref["iterations"]) <= 1, (label, iters, info_ref["iterations"])
    err = np.linalg.norm(x_new - x_ref) / np.linalg.norm(x_ref)
    assert err <= 1e-5, (label, err)
    err64 = np.linalg.norm(x_new - x64) / np.linalg.norm(x64)
    assert err64 <= 1e-4, (label, err64)


def test_noalloc_pcg_matches_the_allocating_entry_point_on_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    for call, (kind, n) in enumerate([("tension", 33), ("dynamic", 65)]):
        rp, ci, vals, rhs = oracle_py.linear_case(kind, n)
        _check_against_both(torch, rp, ci, vals, rhs, f"{kind}-n{n}", measure_memory=call == 1)


def _grid_system(side):
    """An SPD block system on a side x side vertex grid: diagonal blocks 4.2 I plus a small symmetric coupling,
    -I to each of the four grid neighbours (rows = side^2, in row order), and a seeded right-hand side."""
    R = side * side
    rows, cols, vals = [], [], []
    rng = np.random.default_rng(5)
    sym = rng.uniform(-0.05, 0.05, (R, 3, 3))
    sym = sym + sym.transpose(0, 2, 1)
    for i in range(R):
        y, x = divmod(i, side)
        nb = []
        if y > 0:
            nb.append(i - side)
        if x > 0:
            nb.append(i - 1)
        nb.append(i)
        if x + 1 < side:
            nb.append(i + 1)
        if y + 1 < side:
            nb.append(i + side)
        for j in nb:
            rows.append(i)
            cols.append(j)
            vals.append(4.2 * np.eye(3) + sym[i] if j == i else -np.eye(3))
    rp = np.zeros(R + 1, np.int32)
    np.add.at(rp, np.asarray(rows) + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    return rp, np.asarray(cols, np.int32), np.asarray(vals).reshape(-1), rng.standard_normal(3 * R)


def test_noalloc_pcg_at_its_row_limit():
    """The largest system the work space holds (DRAPE_NOALLOC_MAX_ROWS = 65536 = 256^2 rows) solves like drape_pcg
    and the f64 oracle, without taking device memory."""
    torch = pytest.importorskip("torch")
    rp, ci, vals, rhs = _grid_system(256)
    assert len(rp) - 1 == 65536
    _check_against_both(torch, rp, ci, vals, rhs, "grid-256", measure_memory=True)


def test_noalloc_pcg_rejects_sizes_beyond_its_work_space():
    torch = pytest.importorskip("torch")
    lib, fn = _entry()
    limit = 65536
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    p = P(dummy.data_ptr())
    info = np.zeros(3, np.int32)
    st = fn(limit + 1, p, p, p, p, p, p, p, 1e-6, 10, None, info.ctypes.data_as(P), None)
    assert st == 1
    assert "65536" in lib.drape_last_error(None).decode()

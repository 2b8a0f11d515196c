"""drape_pcg_noalloc: block-Jacobi PCG for callers that cannot allocate GPU memory (applications that hand every
device buffer out of their own pool, or that must stay out of the driver's allocator while running).

The test plays such a caller: it owns the matrix, right-hand side and solution buffers (allocated here with
torch, as the caller's own pool would) and asks the library to solve without it allocating anything. Two calls
in a row, on two different systems, must each agree with the allocating entry point drape_pcg on the same
system: same iteration count (+-1) and solutions within the PCG tolerance used by the other GPU tests.
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


def _solve_noalloc(torch, rp, ci, vals, rhs, rtol, maxit):
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
    torch.cuda.synchronize()
    info = np.zeros(3, np.int32)
    rel = ctypes.c_double()
    st = fn(R, P(row_ptr.data_ptr()), P(col_idx.data_ptr()), P(a0.data_ptr()), P(a1.data_ptr()), P(a2.data_ptr()),
            P(b4.data_ptr()), P(x4.data_ptr()), rtol, maxit, None, info.ctypes.data_as(P), ctypes.byref(rel))
    assert st == 0, lib.drape_last_error(None).decode()
    return x4[:, :3].reshape(-1).double().cpu().numpy(), int(info[0]), int(info[1])


def test_noalloc_pcg_matches_the_allocating_entry_point_on_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    for kind, n in [("tension", 33), ("dynamic", 65)]:
        rp, ci, vals, rhs = oracle_py.linear_case(kind, n)
        R = len(rp) - 1
        ref_ctx = api.Drape.from_arrays(np.zeros(3 * R), np.arange(R), np.ones(R), rp, ci)
        x_ref, info_ref = ref_ctx.pcg(rhs, 1e-7, 20000, blocks=vals.astype(np.float32))
        x_new, iters, status = _solve_noalloc(torch, rp, ci, vals, rhs, 1e-7, 20000)
        assert status == 1 and info_ref["status"] == "converged"
        assert abs(iters - info_ref["iterations"]) <= 1, (iters, info_ref["iterations"])
        err = np.linalg.norm(x_new - x_ref) / np.linalg.norm(x_ref)
        assert err <= 1e-5, (kind, n, err)


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

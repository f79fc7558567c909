"""The CPIM solve that allocates no device memory, against the context solver.

capac_bicgstab_static serves callers that cannot call cudaMalloc (a host code
that owns all device memory through its own pool, or a per-step caller that
must not trigger an allocation): they pass device arrays they own, and the
solver's work space is a fixed static device array.  This test hands it the
same matrix, right-hand side and diagonal the context solver (capac_bicgstab)
used, on two calls in a row, and checks both solutions against the context
solver's at the tolerance of the tight-solve parity tests.  It sits in a file
of its own that pytest collects last.
"""
import ctypes
import os

import numpy as np
import pytest

import capacmd_b200 as cm
from conftest import golden_paths, rel_err

pytestmark = pytest.mark.gpu

TIGHT = 1e-26


def _np_ranges(par_path):
    starts, ends = [], []
    for line in open(par_path):
        w = line.split()
        if w and w[0] == "START_END_CHG":
            starts.append(int(w[1]))
            ends.append(int(w[2]))
    return np.array(starts, dtype=np.int32), np.array(ends, dtype=np.int32)


def _bind():
    L = cm.lib()
    vp = ctypes.c_void_p
    L.capac_bicgstab_static.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp,
                                        ctypes.c_double, ctypes.POINTER(ctypes.c_int), vp]
    return L


def test_static_solver_matches_context_solver(gpu_available):
    if not gpu_available:
        pytest.fail("no sm_100 GPU: GPU tests must run on a B200")
    import torch

    paths = golden_paths("t_2np")
    d = cm.Desc.from_paths(paths)
    M, n = d.n_metal, d.n_mat
    s = cm.Simulation(d, solver_tol=TIGHT)
    s.force()  # assembles the matrix, right-hand side and diagonal on the device

    # the context solver from a zero start
    s.set("vec_pq", np.zeros(n))
    it_ctx = ctypes.c_int(0)
    assert cm.lib().capac_bicgstab(s._p, ctypes.byref(it_ctx)) == 0
    x_ctx = s.get("vec_pq")
    assert it_ctx.value > 0

    # the same matrix, column by column through the context's own SpMV
    A = np.zeros((n, n))
    e = np.zeros(n)
    col = np.zeros(n)
    for k in range(n):
        e[:] = 0.0
        e[k] = 1.0
        assert cm.lib().capac_cpim_matvec(s._p, e.ctypes.data, col.ctypes.data) == 0
        A[:, k] = col
    Mp = (M + 31) // 32 * 32
    rows = lambda i: [3 * i, 3 * i + 1, 3 * i + 2, 3 * M + i]  # noqa: E731
    planes = np.zeros((M, 16, Mp))
    for i in range(M):
        ri = rows(i)
        for j in range(M):
            blk = A[np.ix_(ri, rows(j))]
            planes[i, :, j] = blk.reshape(16)
    starts, ends = _np_ranges(paths["par"])

    dev = torch.device("cuda", 0)
    mat = torch.tensor(planes.reshape(-1), dtype=torch.float64, device=dev)
    rhs = torch.tensor(s.get("vec_ext"), dtype=torch.float64, device=dev)
    diag = torch.tensor(s.get("diag_relay"), dtype=torch.float64, device=dev)
    L = _bind()
    results = []
    for call in range(2):
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        it = ctypes.c_int(0)
        rc = L.capac_bicgstab_static(mat.data_ptr(), M, Mp, len(starts), starts.ctypes.data, ends.ctypes.data,
                                     rhs.data_ptr(), diag.data_ptr(), x.data_ptr(), TIGHT, ctypes.byref(it), None)
        assert rc == 0, L.capac_last_error().decode()
        torch.cuda.synchronize()
        xs = x.cpu().numpy()
        assert it.value > 0
        assert rel_err(xs, x_ctx) < 1e-10, f"call {call}"
        results.append(xs)
    assert rel_err(results[1], results[0]) < 1e-10


def test_static_solver_rejects_oversized_systems():
    L = _bind()
    it = ctypes.c_int(0)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.capac_bicgstab_static(dummy, 5000, 5024, 0, None, None, dummy, dummy, dummy, 0.0, ctypes.byref(it),
                                 None)
    assert rc == cm.ERR_CAPACITY
    assert "16384" in L.capac_last_error().decode()

"""The CPIM solve that allocates no device memory, against the context solver.

capac_bicgstab_static serves callers that cannot call cudaMalloc (a host code
that owns all device memory through its own pool, or a per-step caller that
must not trigger an allocation): they pass device arrays they own, and the
solver's work space is a fixed static device array.  These tests hand it the
same matrix, right-hand side and diagonal the context solver (capac_bicgstab)
used, on two calls in a row, and check both solutions against the context
solver's at the tolerance of the tight-solve parity tests; then the branches
a caller meets next: a system without nanoparticles (no neutrality rows), a
warm start from the solution, a zero right-hand side (the reference's early
exit), and a breakdown, which must leave the caller's x as it was.  The file
sits on its own and pytest collects it last.
"""
import ctypes
import os

import numpy as np
import pytest

import capacmd_b200 as cm
from conftest import golden_paths, rel_err

pytestmark = pytest.mark.gpu

TIGHT = 1e-26


@pytest.fixture(autouse=True)
def _need_gpu(gpu_available):
    if not gpu_available:
        pytest.fail("no sm_100 GPU: GPU tests must run on a B200")


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


def _context_solution(paths):
    """The context solver's tight solution from a zero start, and the
    context's matrix in the static entry point's 4x4-block layout."""
    d = cm.Desc.from_paths(paths)
    M, n = d.n_metal, d.n_mat
    s = cm.Simulation(d, solver_tol=TIGHT)
    s.force()  # assembles the matrix, right-hand side and diagonal on the device
    s.set("vec_pq", np.zeros(n))
    it_ctx = ctypes.c_int(0)
    assert cm.lib().capac_bicgstab(s._p, ctypes.byref(it_ctx)) == 0
    assert it_ctx.value > 0
    # the matrix, column by column through the context's own SpMV
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
            planes[i, :, j] = A[np.ix_(ri, rows(j))].reshape(16)
    return dict(x=s.get("vec_pq"), planes=planes, Mp=Mp, M=M, n=n, rhs=s.get("vec_ext"), diag=s.get("diag_relay"))


def _static(L, case, ranges, x, tol=TIGHT):
    import torch
    starts, ends = ranges
    dev = torch.device("cuda", 0)
    mat = torch.tensor(case["planes"].reshape(-1), dtype=torch.float64, device=dev)
    rhs = torch.tensor(case["rhs"], dtype=torch.float64, device=dev)
    diag = torch.tensor(case["diag"], dtype=torch.float64, device=dev)
    xd = torch.tensor(x, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    it = ctypes.c_int(-1)
    rc = L.capac_bicgstab_static(mat.data_ptr(), case["M"], case["Mp"], len(starts), starts.ctypes.data,
                                 ends.ctypes.data, rhs.data_ptr(), diag.data_ptr(), xd.data_ptr(), tol,
                                 ctypes.byref(it), None)
    torch.cuda.synchronize()
    return rc, it.value, xd.cpu().numpy()


def test_static_solver_matches_context_solver():
    paths = golden_paths("t_2np")
    case = _context_solution(paths)
    ranges = _np_ranges(paths["par"])
    L = _bind()
    results = []
    for call in range(2):
        rc, it, xs = _static(L, case, ranges, np.zeros(case["n"]))
        assert rc == 0, L.capac_last_error().decode()
        assert it > 0
        assert rel_err(xs, case["x"]) < 1e-10, f"call {call}"
        results.append(xs)
    assert rel_err(results[1], results[0]) < 1e-10
    # warm start from the solution: the reference's iteration-0 exit or a
    # couple of iterations, and the same answer
    rc, it, xw = _static(L, case, ranges, results[1])
    assert rc == 0, L.capac_last_error().decode()
    assert it <= 2
    assert rel_err(xw, case["x"]) < 1e-10


def test_static_solver_without_nanoparticles(tmp_path):
    """NANOPARTICLES 0: no neutrality rows, the SpMV grid holds metal rows
    only and the static call passes n_nps = 0 with null range pointers."""
    src = golden_paths("t_au55w")
    paths = {}
    for k, p in src.items():
        text = open(p).read()
        if k == "par":
            text = text[:text.index("NANOPARTICLES")] + "NANOPARTICLES   0\n"
        paths[k] = os.path.join(tmp_path, os.path.basename(p))
        with open(paths[k], "w") as f:
            f.write(text)
    case = _context_solution(paths)
    assert case["n"] == 4 * case["M"]
    L = _bind()
    import torch
    dev = torch.device("cuda", 0)
    mat = torch.tensor(case["planes"].reshape(-1), dtype=torch.float64, device=dev)
    rhs = torch.tensor(case["rhs"], dtype=torch.float64, device=dev)
    diag = torch.tensor(case["diag"], dtype=torch.float64, device=dev)
    x = torch.zeros(case["n"], dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    it = ctypes.c_int(0)
    rc = L.capac_bicgstab_static(mat.data_ptr(), case["M"], case["Mp"], 0, None, None, rhs.data_ptr(),
                                 diag.data_ptr(), x.data_ptr(), TIGHT, ctypes.byref(it), None)
    torch.cuda.synchronize()
    assert rc == 0, L.capac_last_error().decode()
    assert it.value > 0
    assert rel_err(x.cpu().numpy(), case["x"]) < 1e-10


def test_static_solver_zero_rhs_and_breakdown():
    """A zero right-hand side returns at once with x untouched (the
    reference's bTb < 1e-10 exit); a system on which BiCGSTAB breaks down
    (r0 orthogonal to A r0, so alpha = rho / 0) is reported as not converged
    after the restarts, with the caller's warm start still in x."""
    L = _bind()
    M, n = 1, 4
    # one metal atom, no nanoparticle: block [[0, 1], [-1, 0]] on (p_x, p_y)
    blk = np.eye(4)
    blk[0, 0] = blk[1, 1] = 0.0
    blk[0, 1], blk[1, 0] = 1.0, -1.0
    case = dict(planes=blk.reshape(1, 16, 1), Mp=1, M=M, n=n, diag=np.ones(n))
    no_np = (np.zeros(0, dtype=np.int32), np.zeros(0, dtype=np.int32))
    x0 = np.array([0.25, -0.5, 0.125, 2.0])
    rc, it, x = _static(L, dict(case, rhs=np.zeros(n)), no_np, x0)
    assert rc == 0 and it == 0
    assert np.array_equal(x, x0)
    rc, it, x = _static(L, dict(case, rhs=np.array([1.0, 0.0, 0.0, 0.0])), no_np, np.zeros(n))
    assert rc == cm.ERR_NOT_CONVERGED
    assert np.array_equal(x, np.zeros(n))


def test_static_solver_rejects_oversized_systems():
    L = _bind()
    it = ctypes.c_int(0)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.capac_bicgstab_static(dummy, 5000, 5024, 0, None, None, dummy, dummy, dummy, 0.0, ctypes.byref(it),
                                 None)
    assert rc == cm.ERR_CAPACITY
    assert "16384" in L.capac_last_error().decode()

"""Failure paths on the GPU, each made on the host side or by a bounded wait.

* RATTLE that cannot converge (an H-H constraint longer than the two O-H
  constraints together) returns CAPAC_ERR_RATTLE with the reference's
  message (force.c:1990-1994); the resident driver exits 1 with it, as the
  reference program does.
* BiCGSTAB stopped at an iteration limit of 1 (the max_iter option standing
  in for MAX_ITER, bicg_stab.c:546-570) returns CAPAC_ERR_NOT_CONVERGED with
  the reference's message, on the persistent and the per-step solver.
* The persistent solver's grid barrier limited to one poll (the wait_polls
  option) gives up: the kernel returns, the call reports CAPAC_ERR_CUDA, and
  the next call on the same context, with the limit restored, succeeds and
  gives the answer of a fresh context.  Nothing faults, traps or hangs: every
  wait in the kernel is bounded and a block that gives up waits for its own
  copies in flight before it returns.
"""
import os
import subprocess

import numpy as np
import pytest

import capacmd_b200 as cm
from conftest import ROOT, golden_paths, impossible_constraints, rel_err, variant

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "capacmd_b200", "capacmd-gpu")


@pytest.fixture(autouse=True)
def _need_gpu(gpu_available):
    if not gpu_available:
        pytest.fail("no sm_100 GPU: GPU tests must run on a B200")


@pytest.mark.parametrize("prec", [cm.PREC_FP64, cm.PREC_MIXED])
def test_rattle_failure_is_a_status(prec, tmp_path):
    paths = variant("t_water", tmp_path, par=impossible_constraints)
    s = cm.Simulation(cm.Desc.from_paths(paths), precision=prec)
    s.md_init()
    with pytest.raises(cm.CapacError) as e:
        s.md_steps(1)
    assert e.value.code == cm.ERR_RATTLE
    assert "RATTLE_1 not converged!" in str(e.value)
    s.force()  # the context stays usable
    assert np.all(np.isfinite(s.forces()))


def test_resident_driver_exits_like_the_reference(tmp_path):
    if not os.path.exists(DRIVER):
        pytest.fail("capacmd_b200/capacmd-gpu is not built (python -m capacmd_b200.build)")
    variant("t_water", tmp_path, par=impossible_constraints)
    out = subprocess.run([DRIVER, "-gro", "init.gro", "-par", "param.txt", "-mds", "mdset.txt"], cwd=tmp_path,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 1
    assert "RATTLE_1 not converged!" in out.stdout


@pytest.mark.parametrize("solver_kernel", [0, 1])
def test_iteration_limit_is_not_converged(solver_kernel):
    d = cm.Desc.from_paths(golden_paths("t_2np"))
    s = cm.Simulation(d, solver_kernel=solver_kernel, max_iter=1)
    with pytest.raises(cm.CapacError) as e:
        s.force()
    assert e.value.code == cm.ERR_NOT_CONVERGED
    assert "bicg_stab not converged" in str(e.value)
    st = s.stats()
    assert st.solver_iterations == 2  # the check after iteration 2 exceeds the limit of 1
    # the default limit on the same system converges
    ok = cm.Simulation(d, solver_kernel=solver_kernel)
    ok.force()
    assert ok.stats().solver_iterations > 2


@pytest.mark.parametrize("prec", [cm.PREC_FP64, cm.PREC_MIXED])
def test_persistent_solver_wait_timeout(prec):
    d = cm.Desc.from_paths(golden_paths("t_2np"))
    tol = dict(solver_tol=1e-26) if prec == cm.PREC_FP64 else dict(refine_tol=1e-11)
    s = cm.Simulation(d, precision=prec, wait_polls=1, **tol)
    with pytest.raises(cm.CapacError) as e:
        s.force()
    assert e.value.code == cm.ERR_CUDA
    assert "bounded wait timed out" in str(e.value)
    s.set("wait_polls", [0])
    s.set("vec_pq", np.zeros(d.n_mat))
    s.force()
    fresh = cm.Simulation(d, precision=prec, **tol)
    fresh.force()
    assert rel_err(s.get("vec_pq"), fresh.get("vec_pq")) < 1e-9
    assert rel_err(s.forces(), fresh.forces()) < 1e-9

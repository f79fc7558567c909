"""The persistent cooperative BiCGSTAB against the launch-per-step solver.

Both run the same algorithm (bicg_stab.c:253-573) on the symmetric packed
matrix; they differ only in the order of floating-point sums, so tight solves
agree to rounding and reference-rule solves meet the same criterion.
"""
import ctypes

import numpy as np
import pytest

import capacmd_b200 as cm
from conftest import golden_paths, rel_err
from capacmd_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu(gpu_available):
    if not gpu_available:
        pytest.fail("no sm_100 GPU: GPU tests must run on a B200")


def _solve_launches(sim):
    n, ms = ctypes.c_long(), ctypes.c_double()
    assert cm.lib().capac_profile_get(sim._p, b"solve", ctypes.byref(n), ctypes.byref(ms)) == 0
    return n.value


def _pair(case, prec, tol):
    # the mixed path refines both to 1e-11, so each is within 1e-9 of the
    # FP64 solution even on the ill-conditioned vacuum cluster
    d = cm.Desc.from_paths(golden_paths(case))
    coop = cm.Simulation(d, precision=prec, solver_tol=tol, solver_kernel=0, refine_tol=1e-11)
    step = cm.Simulation(d, precision=prec, solver_tol=tol, solver_kernel=1, refine_tol=1e-11)
    for s in (coop, step):
        assert cm.lib().capac_profile_enable(s._p, 1) == 0
        s.force()
    return d, coop, step


@pytest.mark.parametrize("case", ["t_au55w", "t_2np", "c1_field"])
@pytest.mark.parametrize("prec", [cm.PREC_FP64, cm.PREC_MIXED])
def test_persistent_solver_matches_stepwise_tight(case, prec):
    d, coop, step = _pair(case, prec, 1e-26 if prec == cm.PREC_FP64 else 0.0)
    assert _solve_launches(coop) > 0, "persistent solver did not run"
    assert _solve_launches(step) == 0
    # FP64: both solve to rTr < 1e-26 bTb; mixed: both refine to a relative
    # residual of 1e-11
    bar = 1e-10 if prec == cm.PREC_FP64 else 1e-8
    assert rel_err(coop.get("vec_pq"), step.get("vec_pq")) < bar
    assert rel_err(coop.forces(), step.forces()) < bar


@pytest.mark.parametrize("case", ["t_au55w", "t_2np", "c1_field"])
def test_persistent_solver_meets_reference_rule(case):
    d, coop, step = _pair(case, cm.PREC_FP64, 0.0)
    st_c, st_s = coop.stats(), step.stats()
    # rTr < 1e-8 bTb (bicg_stab.c:303, 523)
    assert st_c.solver_rel_residual < 1e-4
    assert st_s.solver_rel_residual < 1e-4
    # same algorithm; the iterate under the 1e-4 rule is sensitive to the
    # order of floating-point sums, so counts agree only roughly
    assert st_c.solver_iterations <= 1.5 * st_s.solver_iterations + 5
    assert st_s.solver_iterations <= 1.5 * st_c.solver_iterations + 5
    # the answer is the reference's up to the 1e-4 stopping rule
    assert rel_err(coop.get("vec_pq"), step.get("vec_pq")) < 1e-2


def test_persistent_solver_zero_field_exit():
    # Au147 in vacuum without a field: bTb = 0, the reference's early exit
    d, coop, step = _pair("c1", cm.PREC_FP64, 0.0)
    assert np.all(coop.get("vec_pq") == 0.0)
    assert np.all(step.get("vec_pq") == 0.0)
    assert coop.stats().solver_iterations == 0


def test_persistent_solver_md_steps():
    # several solves in a row, warm-started, through the integrator
    d = cm.Desc.from_paths(golden_paths("c1_field"))
    coop = cm.Simulation(d, solver_tol=1e-26, solver_kernel=0)
    step = cm.Simulation(d, solver_tol=1e-26, solver_kernel=1)
    for s in (coop, step):
        s.md_init()
        s.md_steps(5)
    assert rel_err(coop.positions(), step.positions()) < 1e-11
    assert rel_err(coop.get("vec_pq"), step.get("vec_pq")) < 1e-9


@pytest.mark.parametrize("case", ["t_au55w", "t_2np", "c1_field", "t_au13"])
def test_grouped_solver_matches_ungrouped(case, monkeypatch):
    """The mixed path's persistent solver in the block-Jacobi groups' order
    (tiles assembled in that order, reductions fused with the inverse blocks)
    against the same solver in the reference order: both refine to 1e-11 and
    agree with an FP64 solve to rTr < 1e-26 bTb within the mixed path's bar."""
    d = cm.Desc.from_paths(golden_paths(case))
    grouped = cm.Simulation(d, precision=cm.PREC_MIXED, refine_tol=1e-11)
    monkeypatch.setenv("CAPAC_SOLVER_UNGROUPED", "1")
    plain = cm.Simulation(d, precision=cm.PREC_MIXED, refine_tol=1e-11)
    monkeypatch.delenv("CAPAC_SOLVER_UNGROUPED")
    f64 = cm.Simulation(d, solver_tol=1e-26)
    assert grouped.get("solver_layout")[0] == 1.0, grouped.get("solver_layout")
    assert plain.get("solver_layout")[0] == 0.0
    for s in (grouped, plain, f64):
        s.force()
    x64 = f64.get("vec_pq")
    assert rel_err(grouped.get("vec_pq"), x64) < 1e-8
    assert rel_err(plain.get("vec_pq"), x64) < 1e-8
    assert rel_err(grouped.forces(), plain.forces()) < 1e-8
    assert grouped.stats().solver_rel_residual <= 1e-11
    # MD through several warm-started solves and a preconditioner refresh
    grouped.md_init()
    plain.md_init()
    for _ in range(12):
        grouped.md_steps(1)
        plain.md_steps(1)
    assert rel_err(grouped.get("vec_pq"), plain.get("vec_pq")) < 1e-7
    assert rel_err(grouped.get("rx"), plain.get("rx")) < 1e-9


@pytest.mark.parametrize("case", ["t_au55w", "t_2np", "c1_field"])
def test_tmem_tiles_match_streamed(case, monkeypatch):
    """The grouped solver with the first tiles of each block held in tensor
    memory for the whole solve (one block per SM) gives the same solution as
    the one that streams every tile each pass (two blocks per SM): the same
    FP32 tile products, summed over a different split of the tiles among
    blocks, so the solutions agree to rounding and the iteration counts
    match."""
    d = cm.Desc.from_paths(golden_paths(case))
    held = cm.Simulation(d, precision=cm.PREC_MIXED, refine_tol=1e-11)  # every tile fits: held by default
    monkeypatch.setenv("CAPAC_SOLVER_STREAM", "1")
    streamed = cm.Simulation(d, precision=cm.PREC_MIXED, refine_tol=1e-11)
    monkeypatch.delenv("CAPAC_SOLVER_STREAM")
    assert streamed.get("solver_layout")[1] == 0.0
    assert held.get("solver_layout")[1] > 0.0, held.get("solver_layout")
    for s in (streamed, held):
        s.force()
    assert abs(held.stats().solver_iterations - streamed.stats().solver_iterations) <= 1
    assert rel_err(held.get("vec_pq"), streamed.get("vec_pq")) < 1e-12
    held.md_init()
    streamed.md_init()
    for _ in range(6):
        held.md_steps(1)
        streamed.md_steps(1)
    assert rel_err(held.get("rx"), streamed.get("rx")) < 1e-11


@pytest.mark.parametrize("precond", [2, 3])
@pytest.mark.parametrize("case", ["t_2np", "c1_field", "c2"])
def test_two_level_inner_solves(case, precond):
    """inner_precond 2 and 3: the block-Jacobi inverse with a coarse
    correction on each group's charge sum (3: and its dipole sums) and the
    nanoparticle constraints (multiplicative: Z c + K (v - A Z c),
    c = E^-1 Z^T v).  The refined
    solution meets the same bars against a tight FP64 solve as the
    block-Jacobi inner solves, through MD steps and preconditioner refreshes."""
    paths = configs.cached(case) if case == "c2" else golden_paths(case)
    d = cm.Desc.from_paths(paths)
    two = cm.Simulation(d, precision=cm.PREC_MIXED, refine_tol=1e-11, inner_precond=precond)
    bj = cm.Simulation(d, precision=cm.PREC_MIXED, refine_tol=1e-11, inner_precond=1)
    f64 = cm.Simulation(d, solver_tol=1e-26)
    for s in (two, bj, f64):
        s.force()
    x64 = f64.get("vec_pq")
    assert rel_err(two.get("vec_pq"), x64) < 1e-8
    assert rel_err(two.forces(), bj.forces()) < 1e-8
    assert two.stats().solver_rel_residual <= 1e-11
    two.md_init()
    bj.md_init()
    for _ in range(12):
        two.md_steps(1)
        bj.md_steps(1)
    assert rel_err(two.get("vec_pq"), bj.get("vec_pq")) < 1e-7
    assert rel_err(two.get("rx"), bj.get("rx")) < 1e-9
    assert two.stats().solver_rel_residual <= 1e-11


@pytest.mark.parametrize("case", ["c2", "t_2np"])
def test_coarse_inversion_by_a_cluster(case, monkeypatch):
    """The coarse matrix E inverted by a cluster of CTAs exchanging rows
    through distributed shared memory gives the same solve as the inversion
    by one block (the same pivots and operations)."""
    paths = configs.cached(case) if case == "c2" else golden_paths(case)
    d = cm.Desc.from_paths(paths)
    cl = cm.Simulation(d, precision=cm.PREC_MIXED, refine_tol=1e-11)
    monkeypatch.setenv("CAPAC_COARSE_ONE_BLOCK", "1")
    one = cm.Simulation(d, precision=cm.PREC_MIXED, refine_tol=1e-11)
    monkeypatch.delenv("CAPAC_COARSE_ONE_BLOCK")
    for s in (cl, one):
        s.set("vec_pq", np.zeros(d.n_mat))
        s.force()
    assert cl.get("solver_layout")[4] >= 8, cl.get("solver_layout")
    assert one.get("solver_layout")[4] == 1.0
    assert cl.stats().solver_iterations == one.stats().solver_iterations
    assert rel_err(cl.get("vec_pq"), one.get("vec_pq")) < 1e-12


@pytest.mark.parametrize("prec", [cm.PREC_FP64, cm.PREC_MIXED])
def test_tile_l2_policy_changes_no_result(prec, monkeypatch):
    """The persistent solvers stream their matrix tiles with an L2
    evict-first policy by default, so the vectors, partial sums and
    preconditioner blocks of the reduction phases stay in L2.  The policy
    only steers the cache: the solve is bit for bit the one without it
    (CAPAC_TILE_L2=0) and with part of the tiles kept (CAPAC_TILE_L2=0.5).
    The mixed arms use the full cluster list, whose pair sums run in a fixed
    order (the half list's atomic adds vary the order from run to run)."""
    d = cm.Desc.from_paths(configs.cached("c2"))
    extra = {"pair_list": 3} if prec == cm.PREC_MIXED else {}
    sims = []
    for v in (None, "0", "0.5"):
        if v is None:
            monkeypatch.delenv("CAPAC_TILE_L2", raising=False)
        else:
            monkeypatch.setenv("CAPAC_TILE_L2", v)
        sims.append(cm.Simulation(d, precision=prec, refine_tol=1e-11, **extra))
    monkeypatch.delenv("CAPAC_TILE_L2", raising=False)
    for s in sims:
        s.force()
        s.md_init()
        s.md_steps(3)
    x0 = sims[0].get("vec_pq")
    for s in sims[1:]:
        assert s.stats().solver_iterations == sims[0].stats().solver_iterations
        assert np.array_equal(s.get("vec_pq"), x0)
        assert np.array_equal(s.get("rx"), sims[0].get("rx"))

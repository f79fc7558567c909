"""Mixed-precision path against the FP64 GPU path (tight solve).

Mixed = FP32 pair arithmetic (FP64 coordinate differences, compensated FP32
per-lane force sums), FP32 CPIM matrix storage and SpMV (FP64 accumulation),
FP64 iterative refinement to relative residual 1e-10.  Bars from the
workload's specification: forces within 1e-5 relative, induced charges and
dipoles within 1e-8 relative of the FP64 solution.
"""
import numpy as np
import pytest

import capacmd_b200 as cm
from capacmd_b200 import configs
from conftest import golden_paths, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu(gpu_available):
    if not gpu_available:
        pytest.fail("no sm_100 GPU: GPU tests must run on a B200")


# Au147 in vacuum under a field is ill-conditioned: the default FP64 residual
# target of 1e-10 leaves the induced charges 1.6e-8 from the FP64 solution,
# so it is refined to 1e-11 (the 452k-atom system meets 6e-10 at 1e-10)
REFINE = {"c1_field": 1e-11}


def _both(paths, case=None):
    d = cm.Desc.from_paths(paths)
    f64 = cm.Simulation(d, precision=cm.PREC_FP64, solver_tol=1e-24)
    mix = cm.Simulation(d, precision=cm.PREC_MIXED, refine_tol=REFINE.get(case, 1e-10))
    f64.force()
    mix.force()
    return d, f64, mix


@pytest.mark.parametrize("case", ["t_au55w", "t_2np", "c1_field", "t_water", "c1", "t_morse_buck"])
def test_mixed_forces_and_charges(case):
    d, f64, mix = _both(golden_paths(case), case)
    assert rel_err(mix.forces(), f64.forces()) < 1e-5
    if d.n_mat > 0:
        assert rel_err(mix.get("vec_pq"), f64.get("vec_pq")) < 1e-8
        st = mix.stats()
        if np.any(f64.get("vec_ext") != 0):
            assert st.solver_rel_residual <= 1e-10
    # the total nearly cancels (e.g. +34 kJ/mol from terms of +-600), so the
    # bar is relative to the magnitude of the terms
    p64, pmx = f64.get("potential")[1:], mix.get("potential")[1:]
    assert abs(pmx.sum() - p64.sum()) <= 1e-5 * np.abs(p64).sum()


@pytest.mark.parametrize("prec", [cm.PREC_FP64, cm.PREC_MIXED])
def test_symmetric_and_full_block_layouts_agree(prec):
    d = cm.Desc.from_paths(golden_paths("t_2np"))
    sym = cm.Simulation(d, precision=prec, matrix_layout=0, solver_tol=1e-26)
    full = cm.Simulation(d, precision=prec, matrix_layout=1, solver_tol=1e-26)
    sym.force()
    full.force()
    x = np.random.default_rng(1).normal(size=d.n_mat)
    ys, yf = np.zeros(d.n_mat), np.zeros(d.n_mat)
    assert cm.lib().capac_cpim_matvec(sym._p, x.ctypes.data, ys.ctypes.data) == 0
    assert cm.lib().capac_cpim_matvec(full._p, x.ctypes.data, yf.ctypes.data) == 0
    assert rel_err(ys, yf) < (1e-13 if prec == cm.PREC_FP64 else 1e-6)
    # FP64 solves to rTr < 1e-26 bTb; the mixed path refines both to the same
    # FP64 residual target, which bounds the charges by the 1e-8 bar
    bar = 1e-9 if prec == cm.PREC_FP64 else 1e-8
    assert rel_err(sym.get("vec_pq"), full.get("vec_pq")) < bar
    assert rel_err(sym.forces(), full.forces()) < bar


def test_mixed_medium_system():
    d, f64, mix = _both(configs.cached("c4"))
    assert rel_err(mix.forces(), f64.forces()) < 1e-5
    assert rel_err(mix.get("vec_pq"), f64.get("vec_pq")) < 1e-8


def test_mixed_md_runs_and_conserves_energy_nve():
    # c1 field variant: NVE, CPIM active in vacuum
    d = cm.Desc.from_paths(golden_paths("c1_field"))
    mix = cm.Simulation(d, precision=cm.PREC_MIXED, refine_tol=REFINE["c1_field"])
    mix.md_init()
    e = []
    for _ in range(50):
        mix.md_steps(1)
        e.append(mix.get("potential")[0] + 0.5 * mix.get("thermo")[0])
    e = np.array(e)
    assert np.all(np.isfinite(e))
    assert np.max(np.abs(e - e[0])) / np.abs(e[0]) < 1e-4

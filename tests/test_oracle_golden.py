"""The C restatement (oracle/capac_oracle.c) pinned against the reference.

tests/golden/<case>/ref.npz was produced by the reference sources themselves
(tests/golden/make_golden.py).  Inputs are parsed by the product's parser, so
these tests pin the parser too.

Quantities that do not pass through the BiCGSTAB solve must agree to rounding
(1e-12).  The solve itself stops at relative residual 1e-4 (bicg_stab.c:303)
and its iterate is not a continuous function of rounding (see
test_host.py::test_reference_solve_is_not_continuous_in_rounding), so forces are compared with the reference's own
induced vector fed in (force_given_pq), and the oracle's own solution is
checked against the reference's stopping criterion.
"""
import numpy as np
import pytest

import capacmd_b200 as cm
from oracle.oracle import Oracle
from conftest import GOLDEN_CASES, golden_paths, golden_ref, large_case, rel_err, slot_rel_err


def _setup(case):
    d = cm.Desc.from_paths(golden_paths(case))
    o = Oracle(d)
    assert o.force() == 0
    return d, o, golden_ref(case)


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_pair_set_matches_reference(case):
    d, o, g = _setup(case)
    cnt, h = o.pair_fingerprint()
    assert cnt == int(g["pair_count"])
    assert h == int(g["pair_hash"])


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_solve_inputs_match_reference(case):
    d, o, g = _setup(case)
    if d.n_mat == 0:
        pytest.skip("no CPIM system")
    assert rel_err(o.get("vec_ext"), g["vec_ext"]) < 1e-13
    assert rel_err(o.get("diag_relay"), g["diag_relay"]) == 0.0
    assert rel_err(o.get("inv_sqrt_dens"), g["inv_sqrt_dens"]) < 1e-14
    assert rel_err(o.matvec(g["mv_x"]), g["mv_y"]) < 1e-13


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_forces_given_reference_pq(case):
    d, o, g = _setup(case)
    if d.n_mat > 0:
        o.set("vec_pq", g["vec_pq"])
    assert o.force_given_pq() == 0
    for k in ("fx", "fy", "fz"):
        assert rel_err(o.get(k), g[k]) < 1e-12, k
    assert slot_rel_err(o.get("potential"), g["potential"]) < 1e-11
    assert rel_err(o.get("virial"), g["virial"]) < 1e-12


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_solution_meets_reference_criterion(case):
    d, o, g = _setup(case)
    if d.n_mat == 0:
        pytest.skip("no CPIM system")
    b = g["vec_ext"]
    for x in (o.get("vec_pq"), g["vec_pq"]):
        r = b - o.matvec(x)
        bb = float(b @ b)
        if bb < 1e-10:  # zero right-hand side: the reference skips the solve
            assert np.all(x == 0.0)
        else:
            assert float(r @ r) < 1e-8 * bb


@pytest.mark.parametrize("case", ["t_water", "c1", "t_morse_buck"])
def test_md_trace_matches_reference_without_solve_noise(case):
    # no permanent charges near metal / zero field / no CPIM: no solve noise
    d, o, g = _setup(case)
    o.md_init()
    pots = []
    for _ in range(len(g["md_potential"])):
        assert o.md_steps(1) == 0
        pots.append(o.get("potential"))
    pots = np.array(pots)
    assert rel_err(pots[:, 0], g["md_potential"][:, 0]) < 1e-10
    for k in ("rx", "ry", "rz", "vx", "vy", "vz"):
        assert rel_err(o.get(k), g["md_" + k]) < 1e-10, k


@pytest.mark.parametrize("case", ["t_au55w", "t_2np", "c1_field"])
def test_md_trace_close_to_reference_with_solve(case):
    # the solve stops at relative residual 1e-4, so traces agree to that level
    d, o, g = _setup(case)
    o.md_init()
    pots = []
    for _ in range(len(g["md_potential"])):
        assert o.md_steps(1) == 0
        pots.append(o.get("potential"))
    pots = np.array(pots)
    assert rel_err(pots[:, 0], g["md_potential"][:, 0]) < 1e-5
    assert rel_err(o.get("rx"), g["md_rx"]) < 1e-7


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_cell_fingerprint_matches_reference(case):
    # boxes under three cells of rc per edge take the all-pairs loop
    d, o, g = _setup(case)
    assert o.pair_fingerprint(cells=True) == (int(g["pair_count"]), int(g["pair_hash"]))


def test_large_system_cell_fingerprint_and_sampled_forces():
    """The 91k-atom two-particle system in a field, against the reference's
    own force call on it (the reference counts its pairs in 64 bits here;
    mpi-main.c:406 overflows for N >= 46,342): the cell search finds the
    reference's pair set, and the sampled nonbonded pass plus every other
    term gives the reference's forces on the sampled atoms."""
    paths, g = large_case("c3")
    d = cm.Desc.from_paths(paths)
    o = Oracle(d)
    assert o.pair_fingerprint(cells=True) == (int(g["pair_count"]), int(g["pair_hash"]))
    o.set_sample(g["sample"])
    o.set("vec_pq", g["vec_pq"])
    assert o.force_given_pq() == 0
    f = o.forces()[g["sample"]]
    assert rel_err(f, g["sample_f"]) < 1e-12
    assert rel_err(o.get("vec_ext"), g["vec_ext"]) < 1e-13
    assert rel_err(o.get("inv_sqrt_dens"), g["inv_sqrt_dens"]) < 1e-14
    assert rel_err(o.matvec(g["mv_x"]), g["mv_y"]) < 1e-13
    # every term outside the pair loop: Sutton-Chen [1], CPIM [9..14]
    p, gp = o.get("potential"), g["potential"]
    for k in (1, 9, 10, 11, 12, 13, 14):
        assert abs(p[k] - gp[k]) <= 1e-11 * max(abs(gp[k]), 1e-300), k


def test_large_system_cell_traversal_matches_reference():
    """The restatement's nonbonded pass through cells (systems of 2,048 atoms
    or more) on the 91k-atom system, against the reference's force call:
    forces, every energy slot and the virial."""
    paths, g = large_case("c3")
    o = Oracle(cm.Desc.from_paths(paths))
    o.set("vec_pq", g["vec_pq"])
    assert o.force_given_pq() == 0
    f = o.forces()
    assert rel_err(f[g["sample"]], g["sample_f"]) < 1e-12
    assert abs((f * f).sum() / float(g["f_sumsq"]) - 1.0) < 1e-12
    # sums over 33M pairs of both signs in another order: ~1e-11
    assert slot_rel_err(o.get("potential")[1:], g["potential"][1:]) < 1e-10
    assert rel_err(o.get("virial"), g["virial"]) < 1e-10

"""Bonded terms and virtual sites against the reference's own outputs.

tests/golden/t_bonded holds the reference's first force call and 10 MD steps
on a system with every bonded term it supports (harmonic and Morse bonds,
1-4 pairs of both kinds, harmonic and Urey-Bradley angles, RB and periodic
dihedrals of multiplicity 1 to 4), rigid 4-site waters with a funct-4
virtual site and flexible waters around a CPIM gold cluster.  Bars as in the
parity tests: pair set identical; forces, the 15 energy slots and the virial
within 1e-10 relative for the reference's induced vector; the 10-step energy
and position trace within 1e-8 (each program stops BiCGSTAB at the
reference's 1e-4 rule, whose iterate carries rounding at that level).
"""
import numpy as np
import pytest

import capacmd_b200 as cm
from conftest import golden_paths, golden_ref, rel_err, slot_rel_err

pytestmark = pytest.mark.gpu

CASE = "t_bonded"


@pytest.fixture(autouse=True)
def _need_gpu(gpu_available):
    if not gpu_available:
        pytest.fail("no sm_100 GPU: GPU tests must run on a B200")


def _sim(prec=cm.PREC_FP64, **kw):
    d = cm.Desc.from_paths(golden_paths(CASE))
    return d, cm.Simulation(d, precision=prec, **kw)


def test_pair_set_identical():
    d, s = _sim()
    g = golden_ref(CASE)
    ref = (int(g["pair_count"]), int(g["pair_hash"]))
    assert s.pair_fingerprint(from_list=True) == ref
    assert s.pair_fingerprint(from_list=False) == ref


def test_forces_energies_virial_given_reference_pq():
    d, s = _sim()
    g = golden_ref(CASE)
    s.force()
    s.set("vec_pq", g["vec_pq"])
    cm.lib().capac_force_given_pq(s._p)
    for k in ("fx", "fy", "fz"):
        assert rel_err(s.get(k), g[k]) < 1e-10, k
    pot = s.get("potential")
    for slot in (2, 3, 4, 7, 8):  # bonds, angles, dihedrals, Coulomb and vdW with 1-4
        assert pot[slot] != 0.0
    assert slot_rel_err(pot[1:], g["potential"][1:]) < 1e-10
    assert rel_err(s.get("virial"), g["virial"]) < 1e-10


def test_virtual_sites_are_placed_and_carry_no_force():
    d, s = _sim()
    s.force()
    g = golden_ref(CASE)
    # the reference's first force call placed the sites: its positions are
    # those of init.gro with the sites rebuilt; the sites' own force is zero
    f = s.forces()
    mass = d.get("mass")
    assert np.all(f[mass == 0.0] == 0.0)
    assert np.count_nonzero(mass == 0.0) == 30


def test_md_trace_matches_reference():
    d, s = _sim()
    g = golden_ref(CASE)
    s.md_init()
    pots = []
    for _ in range(len(g["md_potential"])):
        s.md_steps(1)
        pots.append(s.get("potential").copy())
    pots = np.array(pots)
    assert rel_err(pots[:, 0], g["md_potential"][:, 0]) < 1e-8
    for slot in (2, 3, 4):
        assert rel_err(pots[:, slot], g["md_potential"][:, slot]) < 1e-8, slot
    for k in ("rx", "ry", "rz", "vx"):
        assert rel_err(s.get(k), g["md_" + k]) < 1e-8, k


def test_mixed_path_with_bonded_terms():
    d, f64 = _sim(solver_tol=1e-24)
    _, mix = _sim(cm.PREC_MIXED)
    f64.force()
    mix.force()
    assert rel_err(mix.forces(), f64.forces()) < 1e-5
    assert rel_err(mix.get("vec_pq"), f64.get("vec_pq")) < 1e-8

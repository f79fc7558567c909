"""Parsing of bonded terms and virtual sites (file.c:715-969), on the CPU."""
import numpy as np

import capacmd_b200 as cm
from conftest import golden_paths


def test_bonded_terms_are_parsed_per_kind():
    d = cm.Desc.from_paths(golden_paths("t_bonded"))
    counts = d.get("bonded_counts")
    kinds = d.get("bonded_kinds")
    # 20 chains: 2 harmonic + 1 Morse bonds, one 1-4 pair of each kind,
    # 2 harmonic + 1 Urey-Bradley angles, 5 dihedrals (1 RB, 4 periodic as
    # RB); 10 flexible waters: 2 harmonic bonds, 1 Urey-Bradley angle;
    # 30 rigid 4-site waters: 3 constraints and 1 virtual site each
    assert list(counts) == [20 * 13 + 10 * 3, 30, 30 * 3]
    expect = np.zeros(8)
    expect[cm.BT_BOND_HARMONIC] = 20 * 2 + 10 * 2
    expect[cm.BT_BOND_MORSE] = 20
    expect[cm.BT_PAIR_14] = 20
    expect[cm.BT_PAIR_USER] = 20
    expect[cm.BT_ANGLE_HARMONIC] = 20 * 2
    expect[cm.BT_ANGLE_UB] = 20 + 10
    expect[cm.BT_DIHEDRAL_RB] = 20 * 5
    assert np.array_equal(kinds, expect)


def test_periodic_dihedral_as_rb_coefficients():
    # V = k (1 + cos(n phi - phi0)) expanded in cos(psi), psi = phi - 180
    import ctypes
    lib = cm.lib()
    lib.capac_dihedral_periodic_to_rb.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                  ctypes.POINTER(ctypes.c_double)]
    phi = np.linspace(0.1, 3.0, 7)
    for n in (1, 2, 3, 4):
        for phi0 in (0.0, 180.0):
            c = (ctypes.c_double * 6)()
            assert lib.capac_dihedral_periodic_to_rb(phi0, 2.5, n, c) == 0
            # the reference's convention: RB in cos(psi) with the odd signs flipped
            v_rb = c[0] - c[1] * np.cos(phi) + c[2] * np.cos(phi) ** 2 - c[3] * np.cos(phi) ** 3 \
                + c[4] * np.cos(phi) ** 4 - c[5] * np.cos(phi) ** 5
            v = 2.5 * (1 + np.cos(n * phi - np.deg2rad(phi0)))
            assert np.allclose(v_rb, v, atol=1e-12), (n, phi0)
    c = (ctypes.c_double * 6)()
    assert lib.capac_dihedral_periodic_to_rb(90.0, 1.0, 2, c) < 0
    assert lib.capac_dihedral_periodic_to_rb(0.0, 1.0, 5, c) < 0

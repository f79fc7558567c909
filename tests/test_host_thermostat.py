"""The Berendsen thermostat (no counterpart in the reference) in the oracle,
and the library's check of its input.

Weak coupling scales every velocity once a step by
lambda = sqrt(1 + dt/tau (T0/T - 1)) (Berendsen et al., J. Chem. Phys. 81,
3684 (1984)).  Two limits pin the restatement: tau -> infinity leaves the
step an NVE step bit for bit, and tau = dt sets the temperature to T0 in one
step (up to the centre-of-mass removal that follows, which the conserved
momentum makes negligible).
"""
import numpy as np
import pytest

import capacmd_b200 as cm
from oracle.oracle import Oracle
from conftest import berendsen, variant


def _run(paths, steps):
    o = Oracle(cm.Desc.from_paths(paths))
    assert o.force() == 0
    o.md_init()
    temps = []
    for _ in range(steps):
        assert o.md_steps(1) == 0
        temps.append(o.get("thermo")[1])
    return o, np.array(temps)


def _nve(text: str) -> str:
    return text.replace("ensemble          nvt", "ensemble          nve")


def test_infinite_coupling_time_is_nve(tmp_path):
    a, _ = _run(variant("t_water", tmp_path / "b", mds=berendsen(1e300)), 5)
    b, _ = _run(variant("t_water", tmp_path / "n", mds=_nve), 5)
    for k in ("rx", "ry", "vx", "vz"):
        assert np.array_equal(a.get(k), b.get(k))


def test_coupling_time_of_one_step_sets_the_reference_temperature(tmp_path):
    _, temps = _run(variant("t_water", tmp_path, mds=berendsen(0.001, 320.0)), 4)
    # lambda^2 is held to [0.64, 1.5625]: 300 K -> 320 K is inside it
    assert np.max(np.abs(temps - 320.0)) < 1e-9 * 320.0


def test_temperature_relaxes_towards_the_reference(tmp_path):
    _, hot = _run(variant("t_water", tmp_path / "h", mds=berendsen(0.005, 400.0)), 30)
    _, free = _run(variant("t_water", tmp_path / "n", mds=_nve), 30)
    # the lattice start releases potential energy: without a thermostat the
    # water heats past 1000 K in 30 fs; coupled with tau = 5 fs it peaks
    # near 600 K and is brought back towards 400 K
    assert free.max() > 1000.0
    assert hot.max() < 0.65 * free.max()
    assert abs(hot[-1] - 400.0) < 60.0 and abs(hot[-1] - 400.0) < 0.5 * abs(hot.max() - 400.0)


def test_non_positive_coupling_time_is_rejected(tmp_path):
    d = cm.Desc.from_paths(variant("t_water", tmp_path, mds=berendsen(0.0)))
    with pytest.raises(cm.CapacError) as e:
        cm.Simulation(d)
    assert e.value.code == cm.ERR_INVALID

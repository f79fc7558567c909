"""The Berendsen thermostat on the GPU against the oracle's restatement.

The reference has no Berendsen thermostat (its MD loop thermostats only with
the Nose-Hoover chain), so the oracle's formula is the one pinned: on the CPU
at its two limits (tests/test_host_thermostat.py), and here against the
device path over coupled steps, through the C ABI.
"""
import pytest

import capacmd_b200 as cm
from oracle.oracle import Oracle
from conftest import berendsen, rel_err, variant

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu(gpu_available):
    if not gpu_available:
        pytest.fail("no sm_100 GPU: GPU tests must run on a B200")


def test_berendsen_md_trace(tmp_path):
    """The Berendsen thermostat (no counterpart in the reference) against
    the oracle's restatement: 20 steps of the water system coupled to 400 K
    with tau = 5 fs, so every step scales the velocities by several per cent."""
    d = cm.Desc.from_paths(variant("t_water", tmp_path, mds=berendsen(0.005, 400.0)))
    s, o = cm.Simulation(d), Oracle(d)
    s.md_init()
    assert o.force() == 0
    o.md_init()
    ts, to = [], []
    for _ in range(20):
        s.md_steps(1)
        assert o.md_steps(1) == 0
        ts.append(s.get("thermo")[1])
        to.append(o.get("thermo")[1])
    assert to[-1] > 350.0  # the coupling is active: heated from 300 K towards 400 K
    assert rel_err(ts, to) < 1e-9
    for k in ("rx", "vx", "vz"):
        assert rel_err(s.get(k), o.get(k)) < 1e-9

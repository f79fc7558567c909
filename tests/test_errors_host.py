"""Failure paths of the reference, pinned on the CPU.

The reference reports a failure with printf and exit(1); the library returns
a status instead.  These tests fix what the reference itself does on the
inputs the GPU error-path tests use, and that the C restatement agrees.
"""
import os
import subprocess

import pytest

import capacmd_b200 as cm
from oracle.oracle import Oracle
from conftest import ROOT, impossible_constraints, variant

REF = os.path.join(ROOT, "oracle", "_ref", "mpi-main")


def test_impossible_constraints(tmp_path):
    paths = variant("t_water", tmp_path, par=impossible_constraints)
    o = Oracle(cm.Desc.from_paths(paths))
    assert o.force() == 0
    o.md_init()
    assert o.md_steps(1) == cm.ERR_RATTLE
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/mpi-main is built only where the reference sources are")
    out = subprocess.run([REF], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert out.returncode == 1
    assert "RATTLE_1 not converged!" in out.stdout

"""A plain C99 host program against include/capacmd.h and the library.

The boundary is meant for host code written in C, as the reference's own
driver is: this compiles a small C program with gcc in strict C99 (warnings
as errors), links it against libcapacmd_gpu.so, and runs it on a golden
input.  It parses the reference's three input files through the C ABI, reads
the description's fields and sizes from C, takes the derived constants, and
creates a context; without a GPU that last call must return
CAPAC_ERR_NO_DEVICE with a message, as every entry point reports failures by
status instead of exiting.
"""
import os
import shutil
import subprocess

import pytest

import capacmd_b200 as cm
from conftest import ROOT, berendsen, golden_paths, variant

C_SOURCE = r"""
#include <stdio.h>
#include "capacmd.h"

int main(int argc, char **argv)
{
    capac_desc *d = NULL;
    capac_consts k;
    capac_options o;
    capac_ctx *ctx = NULL;
    int n_atoms, n_mols, n_metal, n_nps, n_mat, rc;
    if (argc != 4) return 2;
    if (capac_desc_load(argv[1], argv[2], argv[3], &d) != CAPAC_OK) {
        printf("load failed: %s\n", capac_last_error());
        return 3;
    }
    if (capac_desc_info(d, &n_atoms, &n_mols, &n_metal, &n_nps, &n_mat) != CAPAC_OK) return 4;
    if (capac_desc_derive(d, &k) != CAPAC_OK) return 5;
    printf("atoms %d mols %d metal %d nps %d n_mat %d\n", n_atoms, n_mols, n_metal, n_nps, n_mat);
    printf("ensemble %d tau %.6g ref_temp %.6g dt %.6g ndf %d\n", d->ensemble, d->tau_temp, d->ref_temp, d->dt,
           k.ndf);
    capac_options_default(&o);
    rc = capac_create(d, &o, &ctx);
    printf("create %d %s\n", rc, rc == CAPAC_OK ? "" : capac_last_error());
    if (ctx) capac_destroy(ctx);
    capac_desc_free(d);
    return 0;
}
"""


@pytest.fixture(scope="module")
def c_program(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    out = tmp_path_factory.mktemp("c_host")
    src = out / "host.c"
    src.write_text(C_SOURCE)
    exe = out / "host"
    libdir = os.path.dirname(cm.LIB_PATH)
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
           str(src), "-o", str(exe), "-L", libdir, "-lcapacmd_gpu", f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return str(exe)


def _run(exe, paths):
    r = subprocess.run([exe, paths["gro"], paths["par"], paths["mds"]], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout.splitlines()


def test_c_program_parses_and_reports_by_status(c_program, gpu_available):
    lines = _run(c_program, golden_paths("t_2np"))
    d = cm.Desc.from_paths(golden_paths("t_2np"))
    assert lines[0] == (f"atoms {d.n_atoms} mols {d.n_mols} metal {d.n_metal} nps {d.n_nps} "
                        f"n_mat {d.n_mat}")
    assert lines[1].startswith(f"ensemble {cm.NVT} ")
    rc = int(lines[2].split()[1])
    if gpu_available:
        assert rc == cm.OK
    else:
        assert rc == cm.ERR_NO_DEVICE and len(lines[2].split()) > 2


def test_c_program_reads_the_thermostat_settings(c_program, tmp_path):
    lines = _run(c_program, variant("t_water", tmp_path, mds=berendsen(0.005, 400.0)))
    words = lines[1].split()
    assert int(words[1]) == cm.BERENDSEN
    assert float(words[3]) == 0.005 and float(words[5]) == 400.0

"""Host-side checks that need no GPU: the C ABI library, the input parser,
the workload generator, and the solver-sensitivity property that sets how
charge parity is stated."""
import ctypes
import os
import re
import shutil

import numpy as np
import pytest

import capacmd_b200 as cm
from capacmd_b200 import configs
from oracle.oracle import Oracle
from conftest import ROOT, golden_paths, golden_ref


# ------------------------------------------------------------------ C ABI

def _declared_functions():
    src = open(os.path.join(ROOT, "include", "capacmd.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(capac_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(cm.LIB_PATH)
    names = _declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_every_state_name_is_documented():
    """Every name capac_get answers (the library's name table and its
    diagnostics) appears in the header's description of capac_get."""
    api = open(os.path.join(ROOT, "capacmd_b200", "csrc", "api.cu")).read()
    body = api[api.index("int capac_get(capac_ctx *c, const char *name, double *out)"):]
    body = body[:body.index("\nint capac_set(")]
    names = set(re.findall(r'n == "([a-z_0-9A-Z]+)"', body)) | set(re.findall(r'\{"([a-z_0-9]+)", c->', api))
    hdr = open(os.path.join(ROOT, "include", "capacmd.h")).read()
    doc = hdr[hdr.index("/* State transfer."):hdr.index("int capac_get(")]
    assert len(names) > 20
    missing = sorted(n for n in names if n not in doc)
    assert not missing, missing


def test_python_constants_match_the_header():
    """Every status, precision, bonded-term and thermostat value the Python
    mirror names equals the header's #define of the same name."""
    src = open(os.path.join(ROOT, "include", "capacmd.h")).read()
    defs = {k: int(v) for k, v in re.findall(r"#define CAPAC_([A-Z_0-9]+)\s+\(?(-?\d+)\)?", src)}
    checked = 0
    for name, value in vars(cm).items():
        if isinstance(value, int) and not isinstance(value, bool) and name in defs:
            assert value == defs[name], name
            checked += 1
    for name in ("OK", "ERR_INVALID", "ERR_CAPACITY", "PREC_MIXED", "BT_DIHEDRAL_RB", "NVT", "BERENDSEN"):
        assert name in defs and getattr(cm, name) == defs[name], name
    assert checked >= 20


def test_options_mirror_matches_library_defaults():
    """The Python Options structure has the C layout: every field read back
    from capac_options_default is the documented default."""
    o = cm.Options()
    cm.lib().capac_options_default(ctypes.byref(o))
    assert (o.precision, o.device, o.skin) == (cm.PREC_FP64, 0, 0.2)
    assert (o.list_every, o.max_neighbors, o.solver_tol, o.refine_tol) == (0, 0, 0.0, 1e-10)
    assert (o.matrix_layout, o.predictor, o.solver_kernel, o.inner_precond, o.pair_list) == (0, 3, 0, 3, 0)
    assert (o.max_iter, o.wait_polls) == (0, 0)
    src = open(os.path.join(ROOT, "include", "capacmd.h")).read()
    body = src[src.index("typedef struct capac_options {"):src.index("} capac_options;")]
    fields = re.findall(r"^\s*(?:int|double)\s+(\w+);", body, flags=re.M)
    assert fields == [f[0] for f in cm.Options._fields_]


def test_library_reports_no_device_without_gpu(gpu_available):
    if gpu_available:
        pytest.skip("a GPU is present")
    d = cm.Desc.from_paths(golden_paths("t_au13"))
    with pytest.raises(cm.CapacError) as e:
        cm.Simulation(d)
    assert e.value.code == cm.ERR_NO_DEVICE


# ----------------------------------------------------------------- parser

def test_parser_reads_reference_layout():
    d = cm.Desc.from_paths(golden_paths("t_2np"))
    assert d.n_atoms == 1310 and d.n_metal == 110 and d.n_nps == 2 and d.n_mat == 442
    q = d.get("charge")
    assert np.all(q[:110] == 0.0)
    assert np.allclose(q[110:113], [-0.834, 0.417, 0.417])
    assert np.allclose(d.get("box"), [4.2, 4.2, 4.2])
    # ndf = 3N - 3 - constraints (mpi-main.c:548)
    assert d.consts.ndf == 3 * 1310 - 3 - 3 * 400


def test_parser_matches_reference_state():
    g = golden_ref("t_au55w")
    d = cm.Desc.from_paths(golden_paths("t_au55w"))
    o = Oracle(d)
    assert o.force() == 0
    o.md_init()
    # kinetic energy and temperature after the reference's start-up COM
    # removal (mpi-main.c:629-636) start from the parsed velocities
    th = o.get("thermo")
    assert g["thermo"][3] == d.consts.ndf
    assert abs(th[0] - g["thermo"][0]) <= 1e-12 * abs(g["thermo"][0])
    assert abs(th[1] - g["thermo"][1]) <= 1e-12 * abs(g["thermo"][1])


def test_parser_errors(tmp_path):
    with pytest.raises(cm.CapacError) as e:
        cm.Desc(str(tmp_path / "none.gro"), str(tmp_path / "none.par"), str(tmp_path / "none.mds"))
    assert e.value.code == cm.ERR_IO
    p = golden_paths("t_au13")
    bad = tmp_path / "param.txt"
    txt = open(p["par"]).read().replace("NONBONDED", "NONBONDEX")
    bad.write_text(txt)
    with pytest.raises(cm.CapacError) as e:
        cm.Desc(p["gro"], str(bad), p["mds"])
    assert e.value.code == cm.ERR_IO and "NONBONDED" in str(e.value)
    short = tmp_path / "init.gro"
    short.write_text("".join(open(p["gro"]).readlines()[:5]))
    with pytest.raises(cm.CapacError) as e:
        cm.Desc(str(short), p["par"], p["mds"])
    assert e.value.code == cm.ERR_IO
    # an atom count that is not the topology's: the reference's own check and
    # wording (mpi-main.c:527-532)
    lines = open(p["gro"]).readlines()
    n = int(lines[1])
    lines[1] = f"{n + 1}\n"
    other = tmp_path / "other.gro"
    other.write_text("".join(lines))
    with pytest.raises(cm.CapacError) as e:
        cm.Desc(str(other), p["par"], p["mds"])
    assert e.value.code == cm.ERR_IO and f"groNAtoms({n + 1}) not equal to nAtoms({n})" in str(e.value)


@pytest.mark.parametrize("section,line", [("SOL_BONDS", "0 1 7 0.1 1000.0"),
                                          ("SOL_DIHEDRALS", "0 1 2 0 9 90.0 1.0 2")])
def test_unsupported_bonded_function_types_are_refused(tmp_path, section, line):
    """Function types the reference rejects (file.c:755-760, force.c:1260-1340)."""
    p = golden_paths("t_water")
    txt = open(p["par"]).read()
    old = re.search(rf"(?m)^{section}\s+0$", txt).group(0)
    txt = txt.replace(old, f"{section}   1\n{line}")
    par = tmp_path / "param.txt"
    par.write_text(txt)
    with pytest.raises(cm.CapacError) as e:
        cm.Desc(p["gro"], str(par), p["mds"])
    assert e.value.code == cm.ERR_UNSUPPORTED


# -------------------------------------------------------------- workloads

@pytest.mark.parametrize("shells,count", [(1, 13), (3, 147), (4, 309), (5, 561), (8, 2057)])
def test_mackay_icosahedron_sizes(shells, count):
    x = configs.icosahedron(shells)
    assert len(x) == count
    d = np.sqrt(((x[:, None] - x[None]) ** 2).sum(-1)) if count < 600 else None
    if d is not None:
        np.fill_diagonal(d, np.inf)
        assert abs(d.min() - configs.AU_NN * 0.9511) < 0.01  # radial spacing of Mackay shells


def test_workload_geometry(tmp_path):
    p = configs.write("t_2np", str(tmp_path / "w"))
    d = cm.Desc.from_paths(p)
    r = np.stack([d.get("rx"), d.get("ry"), d.get("rz")], 1)
    M = d.n_metal
    w = r[M:].reshape(-1, 3, 3)
    oh = np.linalg.norm(w[:, 1] - w[:, 0], axis=1)
    hh = np.linalg.norm(w[:, 2] - w[:, 1], axis=1)
    assert np.allclose(oh, 0.1, atol=1e-9) and np.allclose(hh, 0.163299, atol=1e-5)
    L = d.get("box")[0]
    dd = r[M:, None, :] - r[None, :M, :]
    dd -= L * np.round(dd / L)
    assert np.sqrt((dd ** 2).sum(-1)).min() >= 0.3
    # deterministic for a seed
    p2 = configs.write("t_2np", str(tmp_path / "w2"))
    assert open(p["gro"]).read() == open(p2["gro"]).read()


def test_large_workload_sizes():
    # sizes of the measured workloads without writing files
    assert len(configs.icosahedron(8)) == 2057
    w = configs.WORKLOADS
    assert w["c5"].n_waters == 150000 and w["c5"].box == 16.5
    assert w["c3"].n_waters == 30000 and w["c3"].efield_vnm[2] == 0.5


# ------------------------------------------------- solver sensitivity

def _bicgstab(A, b, diag, n4, tol, pert=0.0):
    """Jacobi-preconditioned BiCGSTAB as in bicg_stab.c:253-573, in numpy."""
    n = len(b)
    x = np.zeros(n)
    bTb = b @ b
    r0 = b - A(x)
    r = r0.copy()
    p = np.zeros(n)
    v = np.zeros(n)
    K = np.where(np.arange(n) < n4, 1.0 / diag, 1.0)
    rho_old = alpha = omega = 1.0
    for it in range(1000):
        rho = r0 @ r
        if it == 1:
            rho *= 1.0 + pert
        beta = (rho / rho_old) * (alpha / omega)
        p = r + beta * (p - omega * v)
        y = K * p
        v = A(y)
        alpha = rho / (r0 @ v)
        s = r - alpha * v
        z = K * s
        t = A(z)
        Kt = K * t
        omega = (Kt @ z) / (Kt @ Kt)
        x = x + alpha * y + omega * z
        r = s - omega * t
        rho_old = rho
        if r @ r < tol * bTb:
            return x
    raise AssertionError("no convergence")


def test_reference_solve_is_not_continuous_in_rounding():
    """A 1e-15 relative change of one inner product moves the reference-
    criterion iterate far more than 1e-10, while at a tight tolerance both runs
    meet at the solution: charge/dipole parity at 1e-10 is therefore stated
    against a tight solve."""
    g = golden_ref("c1_field")
    d = cm.Desc.from_paths(golden_paths("c1_field"))
    o = Oracle(d)
    o.force()
    A, b, diag, n4 = o.matvec, g["vec_ext"], g["diag_relay"], 4 * d.n_metal
    xa = _bicgstab(A, b, diag, n4, 1e-8)
    xb = _bicgstab(A, b, diag, n4, 1e-8, pert=1e-15)
    assert np.abs(xa - xb).max() / np.abs(xa).max() > 1e-8
    ta = _bicgstab(A, b, diag, n4, 1e-26)
    tb = _bicgstab(A, b, diag, n4, 1e-26, pert=1e-15)
    assert np.abs(ta - tb).max() / np.abs(ta).max() < 1e-10


def test_oracle_tight_solve_matches_dense_solution():
    d = cm.Desc.from_paths(golden_paths("t_au55w"))
    o = Oracle(d, solver_tol=1e-26)
    assert o.force() == 0
    n = d.n_mat
    A = np.stack([o.matvec(e) for e in np.eye(n)], 1)
    x = np.linalg.solve(A, o.get("vec_ext"))
    assert np.abs(o.get("vec_pq") - x).max() / np.abs(x).max() < 1e-10


def test_fp32_erfc_fit_error_bound():
    """The mixed path's FP32 erfc (exp(-x^2) times a fitted polynomial in
    t = 1 / (1 + x / 2)) against the exact erfc on [0, 5], evaluated with
    FP32 rounding at every step as the kernel does."""
    import math
    import re
    src = open(os.path.join(ROOT, "capacmd_b200", "csrc", "k_pair.cu")).read()
    body = src[src.index("erfc_from_gauss_f(float x, float gauss)"):]
    body = body[:body.index("return gauss * r;")]
    coef = [float(c) for c in re.findall(r"([-+]?\d\.\d+e[-+]\d+)f", body)]
    assert len(coef) == 10  # Horner order: highest degree first
    x = np.linspace(0.0, 5.0, 200001).astype(np.float32)
    t = (np.float32(1.0) / (np.float32(0.5) * x + np.float32(1.0))).astype(np.float32)
    gauss = np.exp(-(x.astype(np.float64) ** 2)).astype(np.float32)
    exact = np.array([math.erfc(float(v)) for v in x])
    # the kernel's reciprocal is the hardware approximation (within one ulp):
    # t exact, and one ulp either side
    for tt in (t, np.nextafter(t, np.float32(2.0)), np.nextafter(t, np.float32(0.0))):
        r = np.float32(coef[0]) * np.ones_like(x)
        for c in coef[1:]:
            r = (r * tt + np.float32(c)).astype(np.float32)
        approx = (gauss * r).astype(np.float64)
        rel = np.abs(approx / exact - 1.0)
        assert rel.max() < 6e-7  # a few FP32 ulp, as the library erfcf

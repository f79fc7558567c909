"""Cluster-pair list of the mixed path against the atom list and the reference.

The mixed path walks a list per cluster of four atoms (k_list.cu, k_pair.cu)
when the box is large enough for the cluster's shared minimum image; every
member keeps exactly the atom list's pairs (the reference's r^2 rounding and
exclusions at the build, the cut-off in FP32 every step).  Checked here: the
pair set equals the reference's (count and hash of all pairs inside the
cut-off, mpi_nonb_pair force.c:1419-1473), forces, energies and virial equal
the atom-list kernel's within FP32 rounding and the FP64 path's within the
mixed path's 1e-5 bar, through list rebuilds in MD, and the gradients that
switch the build to full atom rows.
"""
import numpy as np
import pytest

import capacmd_b200 as cm
from capacmd_b200 import configs
from conftest import golden_paths, golden_ref, large_case, rel_err

pytestmark = pytest.mark.gpu

# boxes with rc + cluster extent + skin below half the shortest edge
CLUSTER_CASES = ["t_au13", "t_2np", "c1", "c1_field"]
ATOM_CASES = ["t_au55w", "t_water"]


@pytest.fixture(autouse=True)
def _need_gpu(gpu_available):
    if not gpu_available:
        pytest.fail("no sm_100 GPU: GPU tests must run on a B200")


def _mixed(paths, **kw):
    d = cm.Desc.from_paths(paths)
    return d, cm.Simulation(d, precision=cm.PREC_MIXED, **kw)


def _uses_clusters(sim) -> bool:
    return sim.get("pair_list")[0] == 1.0


@pytest.mark.parametrize("case", CLUSTER_CASES + ATOM_CASES)
def test_path_choice_and_pair_set(case):
    d, s = _mixed(golden_paths(case))
    g = golden_ref(case)
    ref = (int(g["pair_count"]), int(g["pair_hash"]))
    assert s.pair_fingerprint(from_list=True) == ref
    assert _uses_clusters(s) == (case in CLUSTER_CASES)
    _, a = _mixed(golden_paths(case), pair_list=1)
    assert a.pair_fingerprint(from_list=True) == ref
    assert not _uses_clusters(a)


def test_medium_system_pair_set():
    p = configs.cached("c2")
    d, s = _mixed(p)
    fp = s.pair_fingerprint(from_list=True)
    assert _uses_clusters(s)
    assert fp == s.pair_fingerprint(from_list=False)
    st = s.stats()
    _, a = _mixed(p, pair_list=1)
    a.force()
    sa = a.stats()
    # a cluster's list is shared by its members: fewer entries than the
    # atom list
    assert 0 < st.list_entries < sa.list_entries
    assert st.max_neighbors <= st.list_capacity


@pytest.mark.parametrize("case", ["t_2np", "c1_field", "c2"])
def test_cluster_forces_match_atom_list_and_fp64(case):
    paths = configs.cached(case) if case == "c2" else golden_paths(case)
    d, cl = _mixed(paths, refine_tol=1e-11)
    _, at = _mixed(paths, refine_tol=1e-11, pair_list=1)
    f64 = cm.Simulation(d, precision=cm.PREC_FP64, solver_tol=1e-24)
    for s in (cl, at, f64):
        s.force()
    assert _uses_clusters(cl) and not _uses_clusters(at)
    # FP32 rounding of the differences: one more rounding than the atom kernel
    assert rel_err(cl.forces(), at.forces()) < 2e-6
    assert rel_err(cl.forces(), f64.forces()) < 1e-5
    pc, pa, p64 = cl.get("potential"), at.get("potential"), f64.get("potential")
    # the pair energies nearly cancel (FP32 terms of +-100 kJ/mol summing to
    # tens): bars relative to the magnitude of the terms, as for the mixed path
    scale = np.abs(p64[1:]).sum()
    for k in (7, 8):  # Coulomb and van der Waals sums of the pair kernel
        assert abs(pc[k] - p64[k]) <= 1e-5 * scale
        assert abs(pa[k] - p64[k]) <= 1e-5 * scale
    assert abs(pc[1:].sum() - p64[1:].sum()) <= 1e-5 * scale
    assert rel_err(cl.get("virial"), at.get("virial")) < 1e-5
    if d.n_mat:
        assert rel_err(cl.get("vec_pq"), f64.get("vec_pq")) < 1e-8


def test_cluster_md_through_rebuilds():
    p = configs.cached("c2")
    d, cl = _mixed(p)
    _, at = _mixed(p, pair_list=1)
    f64 = cm.Simulation(d, precision=cm.PREC_FP64)
    for s in (cl, at, f64):
        s.md_init()
    e = {id(s): [] for s in (cl, at, f64)}
    for _ in range(60):
        for s in (cl, at, f64):
            s.md_steps(1)
            e[id(s)].append(s.get("potential")[0])
    assert cl.stats().list_builds >= 2
    assert _uses_clusters(cl)
    ec, ea, e64 = (np.array(e[id(s)]) for s in (cl, at, f64))
    scale = np.abs(e64).max()
    assert np.abs(ec - ea).max() <= 1e-5 * scale
    assert np.abs(ec - e64).max() <= 1e-5 * scale
    # 60 fs of trajectories that differ by FP32 rounding from the first step
    assert rel_err(cl.get("rx"), f64.get("rx")) < 1e-5
    assert rel_err(at.get("rx"), f64.get("rx")) < 1e-5


def test_gradients_on_the_cluster_path():
    """The force-matching gradient walks every atom row: the build switches
    to full atom rows and the pair kernel stays on the clusters."""
    paths = golden_paths("t_2np")
    d, cl = _mixed(paths, refine_tol=1e-11)
    _, at = _mixed(paths, refine_tol=1e-11, pair_list=1)
    for s in (cl, at):
        s.set("vec_pq", np.zeros(d.n_mat))
        s.force()
    # residuals F - target of half the forces, so that the two paths' FP32
    # force rounding (~1e-6 of the largest force) moves the loss little
    target = at.forces() * 0.5
    lc, gc, rc_ = cl.force_match_grad(target, positions=True)
    la, ga, ra = at.force_match_grad(target, positions=True)
    assert _uses_clusters(cl)
    assert lc == pytest.approx(la, rel=1e-5)
    for name in cm.PARAMS:
        assert abs(gc[name] - ga[name]) <= 1e-5 * abs(ga[name]) + 1e-12, name
    assert rel_err(rc_, ra) < 1e-5
    # the pair kernel still runs on the clusters after the full rebuild
    cl.md_init()
    cl.md_steps(5)
    assert _uses_clusters(cl)


@pytest.mark.parametrize("case", CLUSTER_CASES + ["c2"])
def test_half_cluster_list(case):
    """The default cluster list (pair_list 0, as 2): every pair listed once,
    by the lower-numbered cluster of its atoms, and applied to both ends.  The
    pair set is still the reference's; forces, energies and virial agree with
    the full cluster list (pair_list 3) within FP32 rounding of the pair
    terms."""
    paths = configs.cached(case) if case == "c2" else golden_paths(case)
    d, full = _mixed(paths, refine_tol=1e-11, pair_list=3)
    _, half = _mixed(paths, refine_tol=1e-11)
    ref = full.pair_fingerprint(from_list=False)
    if case != "c2":
        g = golden_ref(case)
        assert ref == (int(g["pair_count"]), int(g["pair_hash"]))
    assert half.pair_fingerprint(from_list=True) == ref
    assert _uses_clusters(half)
    for s in (full, half):
        s.force()
    assert half.stats().list_entries < full.stats().list_entries
    assert rel_err(half.forces(), full.forces()) < 2e-6
    pf, ph = full.get("potential"), half.get("potential")
    scale = np.abs(pf[1:]).sum()
    assert np.abs(ph - pf).max() <= 1e-6 * scale
    assert rel_err(half.get("virial"), full.get("virial")) < 1e-5
    if d.n_mat:
        assert rel_err(half.get("vec_pq"), full.get("vec_pq")) < 1e-8


def test_half_cluster_list_md_through_rebuilds():
    p = configs.cached("c2")
    d, full = _mixed(p, pair_list=3)
    _, half = _mixed(p, pair_list=2)
    for s in (full, half):
        s.md_init()
    ef, eh = [], []
    for _ in range(60):
        full.md_steps(1)
        half.md_steps(1)
        ef.append(full.get("potential")[0])
        eh.append(half.get("potential")[0])
    assert half.stats().list_builds >= 2
    assert _uses_clusters(half)
    ef, eh = np.array(ef), np.array(eh)
    assert np.abs(ef - eh).max() <= 1e-5 * np.abs(ef).max()
    assert rel_err(half.get("rx"), full.get("rx")) < 1e-5


def test_full_cluster_list_repeats_exactly():
    """pair_list 3 (every pair from both ends, fixed grid-stride order) gives
    run-to-run identical forces, energies and virial; the default half list
    agrees with it within FP32 rounding and does not use more entries."""
    p = configs.cached("c2")
    d, a = _mixed(p, pair_list=3)
    _, b = _mixed(p, pair_list=3)
    _, h = _mixed(p)
    for s in (a, b, h):
        s.set("vec_pq", np.zeros(d.n_mat))
        s.force()
    assert np.array_equal(a.forces(), b.forces())
    assert np.array_equal(a.get("potential"), b.get("potential"))
    assert np.array_equal(a.get("virial"), b.get("virial"))
    assert rel_err(h.forces(), a.forces()) < 2e-6
    assert h.stats().list_entries < a.stats().list_entries


def test_cluster_pair_list_at_91k_atoms():
    """pair_list 4: i-cluster x j-cluster pairs, each member pair once.  At
    91k atoms (box large enough for the composite minimum image) the list
    holds the reference's pair set, and forces, energies, virial and induced
    vector agree with the full cluster list within FP32 rounding of the pair
    terms and with a tight FP64 solve within the mixed path's bars."""
    paths, g = large_case("c3")
    d, cp = _mixed(paths, refine_tol=1e-11, pair_list=4)
    _, full = _mixed(paths, refine_tol=1e-11, pair_list=3)
    assert cp.pair_fingerprint(from_list=True) == (int(g["pair_count"]), int(g["pair_hash"]))
    assert cp.get("pair_list")[0] == 2.0
    f64 = cm.Simulation(d, precision=cm.PREC_FP64, solver_tol=1e-24)
    for s in (cp, full, f64):
        s.force()
    assert rel_err(cp.forces(), full.forces()) < 2e-6
    assert rel_err(cp.forces(), f64.forces()) < 1e-5
    pc, pf, p64 = cp.get("potential"), full.get("potential"), f64.get("potential")
    scale = np.abs(p64[1:]).sum()
    assert np.abs(pc - pf).max() <= 1e-6 * scale
    assert abs(pc[1:].sum() - p64[1:].sum()) <= 1e-5 * scale
    assert rel_err(cp.get("virial"), full.get("virial")) < 1e-5
    M = d.n_metal
    x, x64 = cp.get("vec_pq"), f64.get("vec_pq")
    assert rel_err(x[3 * M:4 * M], x64[3 * M:4 * M]) < 1e-8
    assert rel_err(x[:3 * M], x64[:3 * M]) < 1e-8


def test_cluster_pair_list_md_through_rebuilds():
    """40 MD steps at 91k atoms on the cluster-pair list against the full
    cluster list: energies within FP32 rounding, the pair set still the
    reference's rule after the rebuilds (checked against all pairs)."""
    paths, _ = large_case("c3")
    d, cp = _mixed(paths, pair_list=4)
    _, full = _mixed(paths, pair_list=3)
    for s in (cp, full):
        s.md_init()
    ec, ef = [], []
    for _ in range(40):
        cp.md_steps(1)
        full.md_steps(1)
        ec.append(cp.get("potential")[0])
        ef.append(full.get("potential")[0])
    assert cp.stats().list_builds >= 2
    assert cp.get("pair_list")[0] == 2.0
    ec, ef = np.array(ec), np.array(ef)
    assert np.abs(ec - ef).max() <= 1e-5 * np.abs(ef).max()
    assert rel_err(cp.get("rx"), full.get("rx")) < 1e-5
    assert cp.pair_fingerprint(from_list=True) == cp.pair_fingerprint(from_list=False)


def test_cluster_pair_list_falls_back_in_a_small_box():
    """Where the box is too small for the composite minimum image the build
    takes the half cluster list instead, with the same pair set."""
    p = configs.cached("c2")
    d, cp = _mixed(p, pair_list=4)
    assert cp.pair_fingerprint(from_list=True) == cp.pair_fingerprint(from_list=False)
    assert cp.get("pair_list")[0] == 1.0


@pytest.mark.parametrize("case", ["t_2np", "c2"])
def test_pairs_overlapped_with_the_solve(case, monkeypatch):
    """CAPAC_OVERLAP: the mixed path runs the nonbonded pairs on a second
    stream while the CPIM stages and solve run, then the CPIM forces on water
    atoms over the clusters next to metal; against the same path in one
    stream: forces, energies, virial and induced vector agree within FP32
    rounding, through MD steps and list rebuilds."""
    paths = configs.cached(case) if case == "c2" else golden_paths(case)
    monkeypatch.setenv("CAPAC_OVERLAP", "1")
    d, ovl = _mixed(paths, refine_tol=1e-11)
    monkeypatch.delenv("CAPAC_OVERLAP")
    _, one = _mixed(paths, refine_tol=1e-11)
    for s in (ovl, one):
        s.set("vec_pq", np.zeros(d.n_mat))
        s.force()
    assert _uses_clusters(ovl)
    # the pair force and the CPIM force of a water atom are rounded to FP32
    # separately here and as one sum on one stream
    assert rel_err(ovl.forces(), one.forces()) < 1e-6
    po, p1 = ovl.get("potential"), one.get("potential")
    assert np.abs(po - p1).max() <= 1e-12 * np.abs(p1[1:]).sum()
    assert rel_err(ovl.get("virial"), one.get("virial")) < 1e-12
    assert rel_err(ovl.get("vec_pq"), one.get("vec_pq")) < 1e-12
    for s in (ovl, one):
        s.md_init()
    for _ in range(30):
        ovl.md_steps(1)
        one.md_steps(1)
    assert rel_err(ovl.get("rx"), one.get("rx")) < 1e-7
    assert abs(ovl.get("potential")[0] - one.get("potential")[0]) <= 1e-7 * abs(one.get("potential")[0])


@pytest.mark.parametrize("case", ["c2", "t_2np"])
def test_split_pair_launch_matches_one_launch(case, monkeypatch):
    """The half-list pair launch split in two (the pair terms over every
    cluster, then the water-side CPIM term over the clusters next to metal)
    gives the energies and virial of the single launch to rounding and its
    forces to FP32 rounding (the single launch adds a pair's CPIM force to
    its pair force in FP32 before the FP64 sum, the split adds both in FP64);
    left to itself the context splits only when fewer than 8% of the clusters
    are next to metal."""
    paths = configs.cached(case) if case == "c2" else golden_paths(case)
    d = cm.Desc.from_paths(paths)
    sims = {}
    for v in ("1", "0", None):
        if v is None:
            monkeypatch.delenv("CAPAC_PAIR_SPLIT", raising=False)
        else:
            monkeypatch.setenv("CAPAC_PAIR_SPLIT", v)
        sims[v] = _mixed(paths)[1]
    monkeypatch.delenv("CAPAC_PAIR_SPLIT", raising=False)
    for s in sims.values():
        s.set("vec_pq", np.zeros(d.n_mat))
        s.force()
    if not _uses_clusters(sims["1"]):
        pytest.skip("the box is too small for the cluster list")
    on, off, auto = sims["1"], sims["0"], sims[None]
    assert on.get("pair_split")[0] == 1.0 and off.get("pair_split")[0] == 0.0
    share = auto.get("pair_split")
    assert share[0] == (1.0 if share[1] < 0.08 * share[2] else 0.0)
    assert rel_err(on.forces(), off.forces()) < 1e-6
    p_on, p_off = on.get("potential"), off.get("potential")
    m = np.abs(p_off) > 0
    assert np.all(np.abs(p_on[m] - p_off[m]) <= 1e-12 * np.abs(p_off[m]))
    assert rel_err(on.get("virial"), off.get("virial")) < 1e-12

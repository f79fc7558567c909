"""Energy and force-matching gradients against central finite differences.

capac_energy_grad returns the total dE/dθ for the metal's nine parameters
(capacitance, polarizability, the two Gaussian widths, the five Sutton-Chen
constants) and dE/dr; capac_force_match_grad returns the force-matching loss
and its parameter gradient.  Each is checked against a Richardson-
extrapolated central difference of the same quantity recomputed by the GPU
(FP64 path; every evaluation solves the CPIM system from a zero start to
rTr < 1e-24 bTb, so the reference's warm-start early exit cannot freeze the
induced vector).  Bar: 1e-6 relative, with an absolute floor scaled by the
summed magnitude of the energy terms for gradients that nearly vanish.

The reference's forces are -dE/dr at fixed induced vector, which is checked
too; the total dE/dr differs from -F because the reported energy is not
stationary in the induced vector at the solution.
"""
import numpy as np
import pytest

import capacmd_b200 as cm
from conftest import golden_paths, rel_err

pytestmark = pytest.mark.gpu

TIGHT = 1e-24
CPIM_CASES = ["t_au55w", "t_2np", "c1_field", "t_au13"]


@pytest.fixture(autouse=True)
def _need_gpu(gpu_available):
    if not gpu_available:
        pytest.fail("no sm_100 GPU: GPU tests must run on a B200")


def _sim(case, prec=cm.PREC_FP64, **kw):
    d = cm.Desc.from_paths(golden_paths(case))
    return d, cm.Simulation(d, precision=prec, solver_tol=TIGHT, **kw)


def _cold_force(sim):
    if sim.desc.n_mat > 0:
        sim.set("vec_pq", np.zeros(sim.desc.n_mat))
    sim.force()


def _energy(sim):
    _cold_force(sim)
    p = sim.get("potential")[1:]
    return p.sum(), np.abs(p).sum()


def _richardson(central, h):
    return (4 * central(h / 2) - central(h)) / 3


def _fd_param(sim, name, fn, rel_step=1e-3):
    th = sim.param_get(name)

    def central(h):
        sim.param_set(name, th + h)
        vp = fn()
        sim.param_set(name, th - h)
        vm = fn()
        sim.param_set(name, th)
        return (vp - vm) / (2 * h)

    return _richardson(central, rel_step * abs(th))


@pytest.mark.parametrize("case", CPIM_CASES)
def test_energy_param_gradient_matches_finite_differences(case):
    d, sim = _sim(case)
    e0, scale = _energy(sim)
    g, _ = sim.energy_grad(positions=False)
    assert set(g) == set(cm.PARAMS)
    for name in cm.PARAMS:
        th = sim.param_get(name)
        fd = _fd_param(sim, name, lambda: _energy(sim)[0])
        assert abs(g[name] - fd) <= 1e-6 * abs(fd) + 1e-10 * scale / abs(th), (name, g[name], fd)
    # back at the original parameters (setting a width decouples it, 0 ties
    # it to C or alpha again): the same energy and gradient
    sim.param_set("cpim_rq", 0.0)
    sim.param_set("cpim_rp", 0.0)
    e1, _ = _energy(sim)
    assert abs(e1 - e0) <= 1e-12 * scale
    g1, _ = sim.energy_grad(positions=False)
    for name in cm.PARAMS:
        assert abs(g1[name] - g[name]) <= 1e-9 * abs(g[name]) + 1e-12 * scale / abs(sim.param_get(name))


def _probe_atoms(sim, d):
    """Metal atoms 0, 1, M-1 and the two permanent charges nearest to metal atom 0."""
    r = sim.positions()
    atoms = [0, 1, d.n_metal - 1]
    if d.n_atoms > d.n_metal:
        q = d.get("charge")
        dist = np.linalg.norm(r - r[0], axis=1)
        dist[: d.n_metal] = np.inf
        dist[q == 0] = np.inf
        atoms += [int(k) for k in np.argsort(dist)[:2]]
    return atoms


@pytest.mark.parametrize("case", ["t_au55w", "c1_field", "t_2np"])
def test_energy_position_gradient_matches_finite_differences(case):
    d, sim = _sim(case)
    _, scale = _energy(sim)
    f = sim.forces()
    x0 = sim.get("vec_pq").copy()
    _, grad = sim.energy_grad()
    r0 = {k: sim.get(k).copy() for k in ("rx", "ry", "rz")}
    h = 1e-5  # nm

    def displaced(i, k, s, fn):
        r = r0[k].copy()
        r[i] += s
        sim.set(k, r)
        v = fn()
        sim.set(k, r0[k])
        return v

    def fixed_x_energy():
        sim.set("vec_pq", x0)
        cm.lib().capac_force_given_pq(sim._p)
        return sim.get("potential")[1:].sum()

    for i in _probe_atoms(sim, d):
        for a, k in enumerate(("rx", "ry", "rz")):
            total = _richardson(lambda hh: (displaced(i, k, hh, lambda: _energy(sim)[0]) -
                                            displaced(i, k, -hh, lambda: _energy(sim)[0])) / (2 * hh), h)
            assert abs(grad[i, a] - total) <= 1e-6 * abs(total) + 1e-9 * scale, (i, k, grad[i, a], total)
            # the reference's force is the gradient at fixed induced vector
            explicit = _richardson(lambda hh: (displaced(i, k, hh, fixed_x_energy) -
                                               displaced(i, k, -hh, fixed_x_energy)) / (2 * hh), h)
            assert abs(-f[i, a] - explicit) <= 1e-6 * abs(explicit) + 1e-9 * scale, (i, k, -f[i, a], explicit)


def test_energy_gradient_without_metal_is_minus_force():
    d, sim = _sim("t_water")
    sim.force()
    g, grad = sim.energy_grad()
    assert all(v == 0.0 for v in g.values())
    assert np.array_equal(grad, -sim.forces())


@pytest.mark.parametrize("case", ["t_au55w", "t_2np"])
def test_force_match_gradient_matches_finite_differences(case):
    d, sim = _sim(case)
    _, scale = _energy(sim)
    f0 = sim.forces()
    # targets: the forces at parameters perturbed by seeded 5% noise
    rng = np.random.default_rng(3)
    th0 = {n: sim.param_get(n) for n in cm.PARAMS}
    for n in ("cpff_capac", "cpff_polar", "qsc_eps", "qsc_c", "qsc_a"):
        sim.param_set(n, th0[n] * (1 + 0.05 * rng.standard_normal()))
    _cold_force(sim)
    target = sim.forces()
    for n in ("cpff_capac", "cpff_polar", "qsc_eps", "qsc_c", "qsc_a"):
        sim.param_set(n, th0[n])
    _cold_force(sim)
    assert rel_err(sim.forces(), f0) < 1e-12

    def loss():
        _cold_force(sim)
        return np.mean((sim.forces() - target) ** 2)

    l0, g = sim.force_match_grad(target)
    assert l0 == pytest.approx(loss(), rel=1e-12)
    l0, g = sim.force_match_grad(target)
    gmax = max(abs(v) * abs(th0[n]) for n, v in g.items())
    for name in cm.PARAMS:
        fd = _fd_param(sim, name, loss)
        assert abs(g[name] - fd) <= 1e-6 * abs(fd) + 1e-9 * gmax / abs(th0[name]), (name, g[name], fd)


def test_width_follows_capacitance_unless_set():
    d, sim = _sim("t_au55w")
    cap, pol = sim.param_get("cpff_capac"), sim.param_get("cpff_polar")
    # R_q = sqrt(2/pi) capac, R_p = (sqrt(2/pi) polar / 3)^(1/3) (mpi-main.c:315-323)
    assert sim.param_get("cpim_rq") == pytest.approx(np.sqrt(2 / np.pi) * cap, rel=1e-15)
    assert sim.param_get("cpim_rp") == pytest.approx((np.sqrt(2 / np.pi) * pol / 3) ** (1 / 3), rel=1e-15)
    sim.param_set("cpff_capac", 2 * cap)
    assert sim.param_get("cpim_rq") == pytest.approx(np.sqrt(2 / np.pi) * 2 * cap, rel=1e-15)
    sim.param_set("cpim_rq", 1.5)
    assert sim.param_get("cpim_rq") == 1.5
    assert sim.param_get("cpff_capac") == 2 * cap
    sim.param_set("cpff_capac", cap)  # a decoupled width stays
    assert sim.param_get("cpim_rq") == 1.5
    sim.param_set("cpim_rq", 0.0)  # tied again
    assert sim.param_get("cpim_rq") == pytest.approx(np.sqrt(2 / np.pi) * cap, rel=1e-15)
    with pytest.raises(cm.CapacError):
        sim.param_set("cpff_polar", -1.0)
    with pytest.raises(cm.CapacError):
        sim.param_get("no_such_parameter")
    # gradients refer to a solved state
    with pytest.raises(cm.CapacError):
        sim.energy_grad()


def test_decoupled_width_gradient_matches_finite_differences():
    """With R_q set on its own, dE/dC no longer carries the width term."""
    d, sim = _sim("t_2np")
    sim.param_set("cpim_rq", 1.05 * sim.param_get("cpim_rq"))
    _, scale = _energy(sim)
    g, _ = sim.energy_grad(positions=False)
    for name in ("cpff_capac", "cpim_rq"):
        fd = _fd_param(sim, name, lambda: _energy(sim)[0])
        assert abs(g[name] - fd) <= 1e-6 * abs(fd) + 1e-10 * scale / abs(sim.param_get(name)), (name, g[name], fd)


def test_setting_a_parameter_back_restores_the_solution():
    d, a = _sim("t_2np")
    _cold_force(a)
    cap = a.param_get("cpff_capac")
    a.param_set("cpff_capac", 1.1 * cap)
    _cold_force(a)
    a.param_set("cpff_capac", cap)
    _cold_force(a)
    _, b = _sim("t_2np")
    _cold_force(b)
    assert rel_err(a.get("vec_pq"), b.get("vec_pq")) < 1e-10
    assert rel_err(a.forces(), b.forces()) < 1e-10


def test_mixed_gradients_match_fp64():
    d, f64 = _sim("t_2np")
    _, mix = _sim("t_2np", prec=cm.PREC_MIXED, refine_tol=1e-11)
    _cold_force(f64)
    _cold_force(mix)
    g64, r64 = f64.energy_grad()
    gmx, rmx = mix.energy_grad()
    for name in cm.PARAMS:
        assert abs(gmx[name] - g64[name]) <= 1e-6 * abs(g64[name]) + 1e-12, name
    assert rel_err(rmx, r64) < 1e-5


@pytest.mark.parametrize("case", ["t_au55w", "t_water", "c1_field"])
def test_force_match_position_gradient_matches_finite_differences(case):
    d, sim = _sim(case)
    _energy(sim)
    f0 = sim.forces()
    rng = np.random.default_rng(5)
    target = f0 + 0.05 * np.abs(f0).mean() * rng.standard_normal(f0.shape)

    def loss():
        _cold_force(sim)
        return np.mean((sim.forces() - target) ** 2)

    l0 = loss()
    l1, _, grad = sim.force_match_grad(target, positions=True)
    assert l1 == pytest.approx(l0, rel=1e-12)
    r0 = {k: sim.get(k).copy() for k in ("rx", "ry", "rz")}
    # t_water's oxygens sit on a lattice with pair offsets of exactly half the
    # box, where the single minimum-image shift makes the force jump: probe
    # hydrogens there
    atoms = _probe_atoms(sim, d) if d.n_metal > 0 else [1, 2, d.n_atoms - 2, d.n_atoms - 1]
    gscale = np.abs(grad).max()
    for i in atoms:
        for a, k in enumerate(("rx", "ry", "rz")):
            def central(hh):
                v = []
                for s in (hh, -hh):
                    r = r0[k].copy()
                    r[i] += s
                    sim.set(k, r)
                    v.append(loss())
                sim.set(k, r0[k])
                return (v[0] - v[1]) / (2 * hh)
            fd = _richardson(central, 1e-5)
            assert abs(grad[i, a] - fd) <= 1e-6 * abs(fd) + 1e-8 * gscale, (i, k, grad[i, a], fd)


def test_torch_autograd_wrappers():
    torch = pytest.importorskip("torch")
    from capacmd_b200 import fit
    d, sim = _sim("t_au55w")
    _cold_force(sim)
    f0 = sim.forces()
    target = torch.from_numpy(f0 * 1.01 + 0.1)
    params = fit.current_params(sim).requires_grad_(True)
    pos = torch.from_numpy(sim.positions()).requires_grad_(True)
    loss = fit.force_match_loss(sim, params, target, positions=pos)
    loss.backward()
    l_ref, g_ref, r_ref = sim.force_match_grad(target.numpy(), positions=True)
    assert loss.item() == pytest.approx(l_ref, rel=1e-12)
    for k, name in enumerate(cm.PARAMS):
        want = 0.0 if name in ("cpim_rq", "cpim_rp") else g_ref[name]  # tied widths: inside C and alpha
        assert params.grad[k].item() == pytest.approx(want, rel=1e-9, abs=1e-12)
    assert np.allclose(pos.grad.numpy(), r_ref, rtol=1e-9, atol=1e-12)
    e = fit.energy(sim, params.detach().requires_grad_(True))
    assert e.item() == pytest.approx(sim.get("potential")[1:].sum(), rel=1e-14)

"""Force-matching fit on the 3.1k-atom system (Au147 + 1,000 waters, seed 3).

Frames are taken every 100 steps from an FP64 run; the targets are FP64
forces at parameters perturbed by seeded 5% Gaussian noise (capacitance,
polarizability, Sutton-Chen eps, c, a; the Gaussian widths follow C and
alpha).  The loss is the force-matching MSE summed over the frames; its
gradient with respect to all nine parameters, taken with the mixed-precision
forward pass (FP32 pairs and matrix, FP64 refinement) and the FP64 adjoint,
and with the FP64 forward pass, is checked against FP64 central finite
differences.  A relative step of 1e-6 would drown in the FP64 solver's
floor (the induced vector is exact to ~1e-11 relative here, which moves the
loss by ~1e-10 of itself from one solve to the next), so the differences
use relative steps 1e-3 and 5e-4 with Richardson extrapolation (truncation
O(h^4)).  Four frames keep the test short; the frame count does not change
what is checked.
"""
import numpy as np
import pytest

import capacmd_b200 as cm
from capacmd_b200 import configs
from conftest import rel_err

pytestmark = pytest.mark.gpu

FRAMES, EVERY = 4, 100
TIGHT = 1e-22  # the 3.1k-atom system's FP64 BiCGSTAB floor is near 7e-12 relative
NOISY = ("cpff_capac", "cpff_polar", "qsc_eps", "qsc_c", "qsc_a")


@pytest.fixture(autouse=True)
def _need_gpu(gpu_available):
    if not gpu_available:
        pytest.fail("no sm_100 GPU: GPU tests must run on a B200")


@pytest.fixture(scope="module")
def fit_case():
    d = cm.Desc.from_paths(configs.cached("c4"))
    run = cm.Simulation(d, precision=cm.PREC_FP64, solver_tol=TIGHT)
    run.md_init()
    frames = []
    for _ in range(FRAMES):
        run.md_steps(EVERY)
        frames.append({k: run.get(k).copy() for k in ("rx", "ry", "rz")})
    run.close()
    ref = cm.Simulation(d, precision=cm.PREC_FP64, solver_tol=TIGHT)
    theta0 = {n: ref.param_get(n) for n in cm.PARAMS}
    rng = np.random.default_rng(3)
    for n in NOISY:
        ref.param_set(n, theta0[n] * (1.0 + 0.05 * rng.standard_normal()))
    targets = [_forces_at(ref, fr) for fr in frames]
    ref.close()
    return d, theta0, frames, targets


def _forces_at(sim, frame):
    for k, v in frame.items():
        sim.set(k, v)
    sim.set("vec_pq", np.zeros(sim.desc.n_mat))
    sim.force()
    return sim.forces()


def _loss_and_grad(sim, frames, targets, positions=False):
    total, grad, pos = 0.0, dict.fromkeys(cm.PARAMS, 0.0), []
    for fr, t in zip(frames, targets):
        _forces_at(sim, fr)
        out = sim.force_match_grad(t, positions=positions)
        total += out[0]
        for n in cm.PARAMS:
            grad[n] += out[1][n]
        if positions:
            pos.append(out[2])
    return total, grad, pos


def _loss(sim, frames, targets):
    return sum(np.mean((_forces_at(sim, fr) - t) ** 2) for fr, t in zip(frames, targets))


def test_force_matching_gradient_mixed_forward_fp64_adjoint(fit_case):
    d, theta0, frames, targets = fit_case
    f64 = cm.Simulation(d, precision=cm.PREC_FP64, solver_tol=TIGHT)
    mix = cm.Simulation(d, precision=cm.PREC_MIXED, refine_tol=1e-10)
    l64, g64, _ = _loss_and_grad(f64, frames, targets)
    lmx, gmx, _ = _loss_and_grad(mix, frames, targets)
    assert lmx == pytest.approx(l64, rel=1e-5)
    assert l64 > 0.0
    worst64 = worst_mx = 0.0
    for name in cm.PARAMS:
        th = f64.param_get(name)

        def central(h):
            f64.param_set(name, th + h)
            lp = _loss(f64, frames, targets)
            f64.param_set(name, th - h)
            lm = _loss(f64, frames, targets)
            f64.param_set(name, th)
            if name in ("cpim_rq", "cpim_rp"):
                f64.param_set(name, 0.0)  # tied again
            return (lp - lm) / (2 * h)

        h = 1e-3 * abs(th)
        fd = (4 * central(h / 2) - central(h)) / 3
        scale = max(abs(fd), 1e-9 * l64 / abs(th))
        worst64 = max(worst64, abs(g64[name] - fd) / scale)
        worst_mx = max(worst_mx, abs(gmx[name] - fd) / scale)
        assert abs(g64[name] - fd) <= 1e-6 * scale, (name, g64[name], fd)
        # the FP32 forward pass moves F by ~1e-7 of |F| against F - F_target
        # of ~5%; measured 4e-7 at worst
        assert abs(gmx[name] - fd) <= 1e-6 * scale, (name, gmx[name], fd)
    print(f"force-matching gradient vs FP64 FD: FP64 adjoint {worst64:.2e}, mixed forward {worst_mx:.2e}")


def test_force_matching_position_gradient_on_a_frame(fit_case):
    d, theta0, frames, targets = fit_case
    sim = cm.Simulation(d, precision=cm.PREC_FP64, solver_tol=TIGHT)
    _, _, pos = _loss_and_grad(sim, frames[:1], targets[:1], positions=True)
    grad = pos[0]
    fr, t = frames[0], targets[0]
    r = np.stack([fr["rx"], fr["ry"], fr["rz"]], 1)
    q = d.get("charge")
    dist = np.linalg.norm(r - r[0], axis=1)
    dist[: d.n_metal] = np.inf
    dist[q == 0] = np.inf
    atoms = [0, d.n_metal - 1, int(np.argmin(dist)), d.n_atoms - 1]
    for i in atoms:
        for a, k in enumerate(("rx", "ry", "rz")):
            def central(h):
                v = []
                for s in (h, -h):
                    f2 = dict(fr)
                    f2[k] = fr[k].copy()
                    f2[k][i] += s
                    v.append(np.mean((_forces_at(sim, f2) - t) ** 2))
                return (v[0] - v[1]) / (2 * h)
            fd = (4 * central(5e-6) - central(1e-5)) / 3
            assert abs(grad[i, a] - fd) <= 1e-6 * abs(fd) + 1e-8 * np.abs(grad).max(), (i, k, grad[i, a], fd)
    assert rel_err(_forces_at(sim, fr), _forces_at(sim, fr)) == 0.0

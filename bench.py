"""Throughput of CapacMD's per-timestep force-and-solve path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c5] [--precision mixed|fp64]
    python bench.py --impl reference ...      # the reference's own CPU code, same workload

Metric: atom-steps/s -- atoms x MD steps per second of device time, one MD
step being the reference loop (mpi-main.c:874-1013: thermostat, half kicks,
drift, RATTLE, and one mpi_force with Sutton-Chen, CPIM RHS, matrix, BiCGSTAB
and CPIM forces) run resident on the GPU.  Default workload: the 452k-atom
system (Au2057 icosahedron in 150,000 rigid waters, 16.5 nm periodic box,
seeded synthetic inputs written in the reference's file formats).

Multi-GPU runs (torchrun) are independent replicas: every rank integrates its
own copy and nothing is exchanged per step (the path does not shard); value is
the sum over ranks, timed as the slowest rank.

The headline arm is the mixed-precision form (FP32 pair terms, FP32 matrix
and SpMV, FP64 refinement to relative residual 1e-10).  Beside it the plain
FP64 path (the reference's algorithm and 1e-4 solver rule) runs the same
steps, the FP64 path also at the mixed path's residual target, and an
accuracy block compares the arms, at the final state, with an FP64 solve to
rTr < 1e-24 bTb.

Printed: one JSON line with value, e2e (the drop-in mpi_force call with host
buffers, copies included), the roofline of the dominant kernel from CUDA-event
timings inside the timed region, the CPU baseline (reference code on a bounded
sample), clocks sampled during the timed region and the kernel-launch count.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD_DESC = {
    "c5": "Au2057 icosahedron + 150,000 rigid 3-site waters, 452,057 atoms, 16.5 nm periodic box, nvt 300 K",
    "c3": "2 x Au561 + 30,000 waters, 91,122 atoms, 9.65 nm box, 0.5 V/nm field along z",
    "c2": "Au309 + 3,000 waters, 9,309 atoms, 4.5 nm box, nvt 300 K",
    "c4": "Au147 + 1,000 waters, 3,147 atoms, 3.1 nm box",
    "c1": "Au147 in vacuum, 147 atoms, nve",
}


def max_over_ranks(ms: float, device) -> float:
    """The slowest rank's time: independent replicas are timed together as
    the slowest one (every rank takes part in the same all-reduce)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(n_atoms: int, steps: int, world: int, ms: float) -> float:
    """Whole-job atom-steps/s of `world` replicas of an n_atoms system, each
    running `steps` MD steps, timed as the slowest replica's ms."""
    return n_atoms * steps * world / (ms / 1e3)


def _peaks() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, n in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(sim, cls: str, n_atoms: int, n_metal: int, precision: str) -> float:
    """HBM bytes one launch of a kernel class must move at minimum.

    pair: the list (4 B per entry) plus, per atom, its packed position/charge
          (32 B, 16 B mixed), list length, type, metal flag, and the force
          read-modify-write (48 B);
    spmv: the symmetric packed 4x4-block CPIM matrix (10 entries per unordered
          metal pair in 32 x 32-atom tiles over the upper triangle; 8 B, 4 B
          mixed), the per-tile partial sums written and read back (nT^2 x 128 x
          8 B each way) and the input and output vectors.
    """
    st = sim.stats()
    w = 4 if precision == "mixed" else 8
    if cls == "pair":
        return 4.0 * st.list_entries + n_atoms * (32 + 4 + 4 + 1 + 48)
    if cls == "spmv":
        nt = (n_metal + 31) // 32
        tiles = nt * (nt + 1) // 2
        return 10.0 * w * 1024 * tiles + 2 * nt * nt * 128 * 8.0 + 2 * 4 * n_metal * 8.0
    if cls == "matrix":
        mp = (n_metal + 31) // 32 * 32
        return 16.0 * 8 * n_metal * mp
    return float("nan")


def cpu_reference_sample(paths: dict, n_atoms: int, target_nb_s: float = 6.0) -> dict:
    """The reference code (oracle/_ref) on a bounded sample of the workload.

    One warm-up force call, then positions drift by dt*v (so the BiCGSTAB warm
    start is as in MD) and one force call is timed with its nonbonded pair loop
    restricted to the last fraction f of the pair index -- the share one rank of
    a 1/f-rank MPI run owns; all other phases run in full.  Per-step time =
    rest + nonbonded/f (the pair loop is uniform O(N^2) work)."""
    from oracle import oracle as O
    if not O.ref_available():
        return {"unavailable": "reference library oracle/_ref/libcapref.so not built"}
    ref = O.open_reference(paths, first_force=False)
    P = n_atoms * (n_atoms - 1) / 2
    frac = min(1.0, target_nb_s / (11e-9 * P))
    O.time_sampled_force(ref, frac)  # warm-up: COO allocation, cold solve
    dt = 0.001
    for a, v in (("rx", "vx"), ("ry", "vy"), ("rz", "vz")):
        ref.set(a, ref.get(a) + dt * ref.get(v))
    t, ph = O.time_sampled_force(ref, frac)
    nb = ph[4]
    step = (t - nb) + nb / frac
    return {"step_s": step, "frac": frac, "wall_s": t, "nonbonded_s": nb, "phases": ph.tolist()}


def run_reference_arm(args, world: int, rank: int) -> int:
    if rank != 0:
        return 0
    from capacmd_b200 import configs
    wl = args.workload
    paths = configs.cached(wl)
    n_atoms = int(open(paths["gro"]).readlines()[1])
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU library not built (oracle/_ref)"}))
        return 0
    ref = O.open_reference(paths, first_force=False)
    P = n_atoms * (n_atoms - 1) / 2
    frac = min(1.0, 4.0 / (11e-9 * P))
    steps = min(args.steps, 3)
    O.time_sampled_force(ref, frac)  # one warm-up call
    per_step = []
    for _ in range(steps):
        for a, v in (("rx", "vx"), ("ry", "vy"), ("rz", "vz")):
            ref.set(a, ref.get(a) + 0.001 * ref.get(v))
        t, ph = O.time_sampled_force(ref, frac)
        per_step.append((t - ph[4]) + ph[4] / frac)
    step_s = float(np.mean(per_step))
    value = n_atoms / step_s
    sample = (f"{steps} force calls of the {n_atoms}-atom workload after one warm-up call, positions drifted "
              f"by dt*v between calls; nonbonded pair loop restricted to the last {frac:.4%} of the pair index "
              f"(the reference's own rank partition), other phases in full; step time = rest + nonbonded/fraction")
    print(json.dumps({
        "impl": "reference", "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s",
        "n_gpus": world, "steps": steps, "warmup": 1, "ms_per_step": step_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_DESC.get(wl, wl), "name": wl, "parallelism": "1 host thread"},
        "cpu_baseline": {"value": value, "unit": "atom-steps/s", "cores": 1, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c5", choices=sorted(WORKLOAD_DESC))
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-compare", action="store_true", help="skip the comparison arms and the accuracy block")
    ap.add_argument("--drift-steps", type=int, default=1000,
                    help="NVE steps per run of the 9.3k-atom system for the energy-drift figures (0: skip)")
    ap.add_argument("--drift-only", action="store_true",
                    help="run the energy-drift study alone (12 runs of --drift-steps) and print its JSON")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-calls", type=int, default=20)
    ap.add_argument("--solver-kernel", type=int, default=0, choices=[0, 1],
                    help="0: persistent cooperative BiCGSTAB launch per solve, 1: a launch per vector step")
    ap.add_argument("--pair-list", type=int, default=0, choices=[0, 1, 2, 3, 4],
                    help="mixed path nonbonded list: 0 (= 2) clusters with every pair once, 1 one list per "
                         "atom, 3 clusters with every pair from both ends, 4 cluster pairs")
    ap.add_argument("--inner-precond", type=int, default=3, choices=[0, 1, 2, 3],
                    help="mixed path inner solves: 0 Jacobi, 1 block-Jacobi, 2 (3) block-Jacobi with a coarse "
                         "correction on group charges (and dipoles)")
    ap.add_argument("--predictor", type=int, default=3, choices=[0, 1, 2, 3],
                    help="mixed path warm start: order of the polynomial extrapolation of past solutions")
    ap.add_argument("--solver-phases", action="store_true",
                    help="time the persistent solver's phases in-kernel (globaltimer, block 0) and report them")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.solver_phases:
        os.environ["CAPAC_SOLVER_PHASES"] = "1"  # read when the context is created

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference_arm(args, world, rank)

    import torch
    import torch.distributed as dist
    import capacmd_b200 as cm
    from capacmd_b200 import configs

    torch.cuda.set_device(local)
    if args.drift_only:
        print(json.dumps(nve_drift(cm, configs, args.drift_steps, local)))
        return 0
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    if rank == 0:
        paths = configs.cached(args.workload)
    if world > 1:
        dist.barrier()
    paths = configs.cached(args.workload)

    prec = cm.PREC_MIXED if args.precision == "mixed" else cm.PREC_FP64
    desc = cm.Desc.from_paths(paths)
    sim = cm.Simulation(desc, precision=prec, device=local, solver_kernel=args.solver_kernel,
                        predictor=args.predictor, pair_list=args.pair_list, inner_precond=args.inner_precond)
    N, M = desc.n_atoms, desc.n_metal
    sim.md_init()
    sim.md_steps(args.warmup)

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.15)
    cm.lib().capac_profile_enable(sim._p, 1)
    l0 = sim.kernel_launches()
    ms = ctypes_time(sim, args.steps)
    launches = sim.kernel_launches() - l0
    prof = {}
    for cls in ("pair", "spmv", "matrix", "cpim_metal", "cpim_rhs", "qsc", "list_build", "solver_vec", "resid",
                "solve"):
        prof[cls] = profile_get(sim, cls)
    n_spmv = spmv_effective(sim, 0)
    cm.lib().capac_profile_enable(sim._p, 0)
    clk = clocks.stop()
    torch.cuda.synchronize()
    if world > 1:
        ms = max_over_ranks(ms, "cuda")
        dist.barrier()
    value = replica_value(N, args.steps, world, ms)
    st = sim.stats()

    # dominant kernel and its roofline, and the persistent solve's beside it
    peak, peak_kind = _peaks()

    def kernel_roofline(cls):
        n_launch, tot_ms = prof[cls]
        if cls == "spmv":
            n_launch = n_spmv or n_launch
        avg_s = tot_ms / max(n_launch, 1) / 1e3
        if cls == "solve":
            # one launch = a whole solve: its SpMV products plus the BiCGSTAB
            # vector updates (19 n doubles per iteration beyond the products)
            iters = max(n_spmv - n_launch, 0) / 2
            bytes_launch = (n_spmv * algorithmic_bytes(sim, "spmv", N, M, args.precision)
                            + iters * 19 * desc.n_mat * 8.0) / max(n_launch, 1)
        else:
            bytes_launch = algorithmic_bytes(sim, cls, N, M, args.precision)
        achieved = bytes_launch / avg_s / 1e9 if avg_s > 0 else None
        r = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
             "frac": achieved / peak if achieved else None, "traffic": _traffic(args.workload, args.precision, cls),
             "kernel": cls, "algorithmic_bytes_per_launch": bytes_launch, "avg_launch_ms": avg_s * 1e3,
             "launches": n_launch, "peak_kind": peak_kind}
        if r["traffic"] and r["traffic"] < 0.5 * bytes_launch:
            r["note"] = (f"operands stay in the 126 MB L2 across the launch: measured DRAM traffic is "
                         f"{r['traffic'] / bytes_launch:.0%} of the algorithmic bytes, so the launch is "
                         f"bound by L2 and latency, not HBM")
        if cls == "pair" and args.precision == "mixed":
            ia = _issue_active("pair")
            r["note"] = ("FP32 pair terms on the CUDA cores, one list pass per step: bound by instruction issue "
                         "and latency, not by bytes" + (f" (ncu issue active {ia:.0%} of peak on the 91k-atom "
                                                         f"workload, profiles/k_pair_cl_half_c3.md)" if ia else ""))
        return r

    dom = max(("pair", "spmv", "matrix", "solve"), key=lambda k: prof[k][1])
    roofline = kernel_roofline(dom)
    roofline_solve = kernel_roofline("solve") if dom != "solve" and prof["solve"][0] > 0 else None

    # the other precision on the same workload and step count, the FP64 path
    # also at the mixed path's residual target, and the accuracy of the arms
    # against a tight FP64 solve at the final state
    compare, accuracy = None, None
    if not args.no_compare and world == 1:
        compare, accuracy = compare_arms(args, cm, desc, sim, prec, local)
        if args.drift_steps > 0:
            accuracy["nve_drift"] = nve_drift(cm, configs, args.drift_steps, local)
        accuracy["gradients"] = gradient_timing(cm, configs, local)

    # end to end through the drop-in mpi_force with pinned host buffers
    e2e = None
    if not args.no_e2e:
        e2e = e2e_drop_in(sim, desc, args.e2e_calls, prec, local, torch)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference_sample(paths, N)
        if "unavailable" in r:
            cpu = {"value": None, "unit": "atom-steps/s", "cores": 1, "kind": "reference", "sample": r["unavailable"]}
        else:
            cpu = {"value": N / r["step_s"], "unit": "atom-steps/s", "cores": 1, "kind": "reference",
                   "sample": (f"one reference force call (after a warm-up call) of the {N}-atom workload with the "
                              f"nonbonded pair loop restricted to the last {r['frac']:.4%} of the pair index, other "
                              f"phases in full; step = rest + nonbonded/fraction = {r['step_s']:.1f} s")}

    if rank == 0:
        ps = sim.phase_times()
        line = {
            "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 pair/SpMV + f64 refinement",
            "data": "synthetic",
            "config": {"workload": WORKLOAD_DESC[args.workload], "name": args.workload,
                       "atoms": N, "metal_atoms": M, "cpim_unknowns": desc.n_mat, "precision": args.precision,
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (neighbour list and CPIM matrix > 126 MB)"},
            "ns_per_day": args.steps / (ms / 1e3) * 0.001 * 86.4,  # steps/s x dt(ps) x s/day / ps-per-ns
            "solver": {"iterations_last": st.solver_iterations, "sweeps_last": st.solver_outer,
                       "initial_rel_residual_last": st.solver_initial_rel_residual,
                       "rel_residual_last": st.solver_rel_residual,
                       "ms_per_solve": (prof["spmv"][1] + prof["solver_vec"][1] + prof["resid"][1]
                                        + prof["solve"][1]) / args.steps,
                       "layout": "group order" if sim.get("solver_layout")[0] else "reference order",
                       "tiles_in_tensor_memory_per_block": int(sim.get("solver_layout")[1]),
                       "inner_stalls": int(sim.get("inner_stalls")[0])},
            "pair_launch": (lambda ps: {"split": bool(ps[0]), "clusters_next_to_metal": int(ps[1]),
                                        "clusters": int(ps[2])})(sim.get("pair_split")),
            "kernel_ms": {k: v[1] for k, v in prof.items()},
            **({"solver_phase_us": solver_phases(sim)} if args.solver_phases else {}),
            "phase_ms_last_force": {"list": ps[10], "qsc": ps[1], "cpim_vec": ps[6], "cpim_matrix": ps[5],
                                    "cpim_solve": ps[7], "nonbonded": ps[4], "cpim_force": ps[8]},
            "roofline": roofline, **({"roofline_solve": roofline_solve} if roofline_solve else {}),
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "gpu_launches": launches,
            "compare": compare, "accuracy": accuracy,
        }
        print(json.dumps(line))
    sim.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def solver_phases(sim) -> dict:
    """Mean microseconds per iteration of the persistent solver's phases
    (block 0's view, %globaltimer marks), over the iterations timed."""
    ph = sim.get("solver_phases")
    # two-level inner solves: each reduction's first step (with its grid
    # barrier) under "V reduction" / "T reduction", its coarse step (with the
    # next barrier) under "K v pass" / "K t pass"
    names = ["P tile pass", "P grid barrier", "V reduction (+ K v)", "K v pass", "alpha + S tile pass + barrier",
             "T reduction (+ K t)", "K t pass", "dot sums + scalars"]
    out = {n: ph[k] / 1e3 for k, n in enumerate(names)}
    out["iterations_timed"] = ph[8]
    out["total"] = float(sum(ph[:8]) / 1e3)
    return out


def compare_arms(args, cm, desc, sim, prec, device) -> tuple[dict, dict]:
    """Time the other precision (and FP64 at the mixed residual target) over
    the same steps; measure every arm's errors at its own final state."""
    N = desc.n_atoms

    def rel(a, b):
        nb = float(np.linalg.norm(b))
        return float(np.linalg.norm(a - b) / nb) if nb > 0 else 0.0

    def state_errors(x):
        """x's forces, charges, dipoles and energy against an FP64 solve to
        rTr < 1e-24 bTb from a zero start at x's positions."""
        x.force()
        ref = cm.Simulation(desc, precision=cm.PREC_FP64, device=device, solver_tol=1e-24)
        for a in ("rx", "ry", "rz"):
            ref.set(a, x.get(a))
        ref.force()
        M = desc.n_metal
        ex, er = x.get("potential")[1:], ref.get("potential")[1:]
        out = {"force": rel(x.forces(), ref.forces()),
               "energy_vs_sum_abs_terms": float(abs(ex.sum() - er.sum()) / max(np.abs(er).sum(), 1e-300))}
        if desc.n_mat > 0:
            qx, qr = x.get("vec_pq"), ref.get("vec_pq")
            out["charges"] = rel(qx[3 * M:4 * M], qr[3 * M:4 * M])
            out["dipoles"] = rel(qx[:3 * M], qr[:3 * M])
        ref.close()
        return out

    acc = {"reference": "each arm at its own final MD state against the FP64 path at the same positions "
                        "solved to rTr < 1e-24 bTb from a zero start",
           "headline": state_errors(sim)}
    arms = {}
    other = cm.PREC_FP64 if prec == cm.PREC_MIXED else cm.PREC_MIXED
    specs = [("fp64_plain" if other == cm.PREC_FP64 else "mixed", other, 0.0, 0)]
    if desc.n_mat > 0:
        # rTr < 1e-20 bTb: relative residual 1e-10, the mixed path's target
        specs.append(("fp64_equal_residual", cm.PREC_FP64, 1e-20, 0))
    if prec == cm.PREC_MIXED:
        # the other cluster list: every pair once (2) against four atoms sharing each neighbour (0)
        other_list = 3 if args.pair_list in (0, 2) else 0  # the full cluster list against the half one
        specs.append((f"mixed_pair_list_{other_list}", cm.PREC_MIXED, 0.0, other_list))
    for name, p, tol, plist in specs:
        s2 = cm.Simulation(desc, precision=p, device=device, solver_tol=tol, solver_kernel=args.solver_kernel,
                           predictor=args.predictor, pair_list=plist, inner_precond=args.inner_precond)
        s2.md_init()
        s2.md_steps(args.warmup)
        ms2 = ctypes_time(s2, args.steps)
        st2 = s2.stats()
        arms[name] = {"value": N * args.steps / (ms2 / 1e3), "unit": "atom-steps/s",
                      "ms_per_step": ms2 / args.steps, "solver_iterations_last": st2.solver_iterations,
                      "solver_rel_residual_last": st2.solver_rel_residual}
        acc[name] = state_errors(s2)
        s2.close()
    return arms, acc


def nve_drift(cm, configs, steps: int, device: int, every: int = 10) -> dict:
    """Total-energy drift of NVE runs of the 9.3k-atom system (Au309 in 3,000
    waters, dt 1 fs), three seeds (initial configuration and velocities) per
    arm: the mixed path, the FP64 path at the reference's solver rule, the
    FP64 path solved to rTr < 1e-22 bTb, and the mixed path without CPIM (the
    floor of the integrator and RATTLE).  Per run: the slope of a
    least-squares line through E_pot + E_kin sampled every `every` steps, per
    atom and per ns.  Per arm: the mean over the seeds and its standard
    error; per seed the mixed-minus-tight difference (same initial state),
    with its mean, standard error and 95% interval (Student t, 2 degrees of
    freedom).  The reference's CPIM forces are the gradient of its energy at
    fixed induced vector, and that energy is not stationary in the induced
    vector, so even exact solves do not conserve it: the tight FP64 arm is
    the floor the CPIM arms are compared with."""
    seeds = (("c2_nve", "c2_nve_nocpim_s1"), ("c2_nve_s2", "c2_nve_nocpim_s2"), ("c2_nve_s3", "c2_nve_nocpim_s3"))
    out = {"workload": "Au309 + 3,000 waters (9,309 atoms), nve, dt 1 fs, seeds 1-3", "steps": steps,
           "unit": "kJ/mol per atom per ns"}
    arms = (("mixed", cm.PREC_MIXED, {}, 0), ("fp64_plain", cm.PREC_FP64, {}, 0),
            ("fp64_tight", cm.PREC_FP64, {"solver_tol": 1e-22}, 0), ("mixed_no_cpim", cm.PREC_MIXED, {}, 1))
    runs = {name: [] for name, *_ in arms}
    for name, p, kw, variant in arms:
        for pair in seeds:
            d = cm.Desc.from_paths(configs.cached(pair[variant]))
            s = cm.Simulation(d, precision=p, device=device, **kw)
            s.md_init()
            t, e = [], []
            for k in range(steps // every + 1):
                if k:
                    s.md_steps(every)
                t.append(k * every * 1e-3)  # ps
                e.append(s.get("potential")[0] + 0.5 * s.get("thermo")[0])
            t, e = np.array(t), np.array(e)
            fit = np.polyfit(t, e, 1)
            runs[name].append({"drift": float(fit[0]) * 1e3 / d.n_atoms,
                               "rms_fluctuation": float(np.std(e - np.polyval(fit, t))), "e_start": float(e[0])})
            s.close()
    t95 = 4.303  # Student t, 2 degrees of freedom
    for name, rs in runs.items():
        v = np.array([r["drift"] for r in rs])
        out[name] = {"drift_mean": float(v.mean()), "drift_se": float(v.std(ddof=1) / np.sqrt(len(v))),
                     "runs": rs}
    diff = np.array([a["drift"] - b["drift"] for a, b in zip(runs["mixed"], runs["fp64_tight"])])
    se = float(diff.std(ddof=1) / np.sqrt(len(diff)))
    out["mixed_minus_fp64_tight"] = {"mean": float(diff.mean()), "se": se,
                                     "ci95": [float(diff.mean() - t95 * se), float(diff.mean() + t95 * se)],
                                     "per_seed": diff.tolist()}
    return out


def gradient_timing(cm, configs, device: int, calls: int = 10) -> dict:
    """Wall time per gradient call on the 3.1k-atom system (Au147 + 1,000
    waters): one mixed-precision force evaluation with a solve from zero,
    then capac_energy_grad (parameters and positions) or
    capac_force_match_grad (parameters and positions); each call includes its
    adjoint solve and the host copies of its results."""
    d = cm.Desc.from_paths(configs.cached("c4"))
    s = cm.Simulation(d, precision=cm.PREC_MIXED, device=device)
    zero = np.zeros(d.n_mat)

    def fresh():
        s.set("vec_pq", zero)
        s.force()

    fresh()
    target = s.forces() * 1.05
    out = {"workload": f"Au147 + 1,000 waters ({d.n_atoms:,} atoms), mixed forward", "unit": "ms per call"}
    for name, fn in (("force", lambda: None), ("energy_grad", lambda: s.energy_grad()),
                     ("force_match_grad", lambda: s.force_match_grad(target, positions=True))):
        fresh()
        fn()  # warm-up (workspace, graphs)
        t = []
        for _ in range(calls):
            fresh()
            t0 = time.perf_counter()
            fn()
            t.append(time.perf_counter() - t0)
        out[name] = statistics.median(t) * 1e3
    t = []
    for _ in range(calls):
        s.set("vec_pq", zero)
        t0 = time.perf_counter()
        s.force()
        t.append(time.perf_counter() - t0)
    out["force"] = statistics.median(t) * 1e3
    s.close()
    return out


def ctypes_time(sim, steps: int) -> float:
    import ctypes
    import capacmd_b200 as cm
    out = ctypes.c_double(0.0)
    lib = cm.lib()
    lib.capac_time_md_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    cm._check(lib.capac_time_md_steps(sim._p, int(steps), ctypes.byref(out)))
    return out.value


def profile_get(sim, cls: str) -> tuple[int, float]:
    import ctypes
    import capacmd_b200 as cm
    lib = cm.lib()
    lib.capac_profile_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_long),
                                      ctypes.POINTER(ctypes.c_double)]
    n, ms = ctypes.c_long(0), ctypes.c_double(0.0)
    cm._check(lib.capac_profile_get(sim._p, cls.encode(), ctypes.byref(n), ctypes.byref(ms)))
    return int(n.value), float(ms.value)


def spmv_effective(sim, launched: int) -> int:
    """SpMV launches that did work (the solver over-issues a few per solve that
    return immediately once it has converged)."""
    n, _ = profile_get(sim, "spmv_effective")
    return n if n > 0 else launched


def _issue_active(kernel: str):
    """ncu issue-active fraction of the mixed path's kernel on the 91k-atom
    workload, if its capture summary is committed (profiles/ncu_traffic.json)."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            return json.load(f)["issue_active"]["c3"]["mixed"].get(kernel)
    except Exception:
        return None


def _traffic(workload: str, precision: str, kernel: str):
    """DRAM bytes per launch measured by ncu for this kernel, workload and
    precision, if a capture summary is committed (profiles/ncu_traffic.json)."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            return json.load(f).get(workload, {}).get(precision, {}).get(kernel)
    except Exception:
        return None


def e2e_drop_in(sim, desc, calls: int, prec: int, device: int, torch) -> dict:
    """atom-steps/s through capac_mpi_force with pinned host buffers: positions
    (and the induced-vector warm start) copied in, forces, energies, virial and
    the induced vector copied out, every call.  The positions of successive
    calls are successive frames of the workload's own MD (the resident
    simulation, stepped outside the timed region, as the drop-in mode's caller
    integrates between its force calls); the calls go to a second context, so
    each sees one real step's displacement and keeps its own induced vector as
    the warm start, as the reference's caller does.  Only the calls are timed."""
    import capacmd_b200 as cm
    N, n = desc.n_atoms, max(desc.n_mat, 1)

    def pinned(k):
        return torch.empty(k, dtype=torch.float64, pin_memory=True).numpy()

    drop = cm.Simulation(desc, precision=prec, device=device)
    rx, ry, rz = pinned(N), pinned(N), pinned(N)
    fx, fy, fz, pot, vir, pq = pinned(N), pinned(N), pinned(N), pinned(15), pinned(9), pinned(n)
    pq[:] = sim.get("vec_pq") if desc.n_mat else 0.0
    lib = cm.lib()
    ptr = lambda a: a.ctypes.data  # noqa: E731

    def call():
        cm._check(lib.capac_mpi_force(drop._p, ptr(rx), ptr(ry), ptr(rz), ptr(fx), ptr(fy), ptr(fz), ptr(pot),
                                      ptr(vir), ptr(pq) if desc.n_mat else None, None, None, None))

    rx[:], ry[:], rz[:] = sim.get("rx"), sim.get("ry"), sim.get("rz")
    call()  # first call: list, matrix and preconditioner set-up of the new context
    h2d = 3 * N * 8 + desc.n_mat * 8
    d2h = 3 * N * 8 + 15 * 8 + 9 * 8 + desc.n_mat * 8
    elapsed = 0.0
    for _ in range(calls):
        sim.md_steps(1)
        rx[:], ry[:], rz[:] = sim.get("rx"), sim.get("ry"), sim.get("rz")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        call()
        elapsed += time.perf_counter() - t0
    drop.close()
    return {"value": N * calls / elapsed, "unit": "atom-steps/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "calls": calls, "ms_per_call": elapsed / calls * 1e3,
            "what": "one drop-in mpi_force per MD step (host positions in, host forces/energies/virial/vec_pq "
                    "out) on successive frames of the workload's own trajectory, the induced vector carried "
                    "between calls by the caller; the integration between calls is the caller's, untimed"}


if __name__ == "__main__":
    sys.exit(main())

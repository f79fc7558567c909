"""Generate the golden fixtures under tests/golden/ from the reference itself.

The reference CapacMD ships no tests or expected outputs, so its own sources,
compiled in place by ``make -C oracle ref`` (single-rank MPI stub, unmodified
physics), are run on small seeded inputs and their outputs are stored:

    tests/golden/<case>/{init.gro,param.txt,mdset.txt}   inputs (our generator)
    tests/golden/<case>/ref.npz                          reference outputs

ref.npz holds, after the reference's first force call: forces, the 15
potential slots, the virial, the CPIM vectors (vec_pq, vec_ext, diag_relay),
inv_sqrt_dens, the pair-set fingerprint, one product of the reference's COO
matrix with a seeded probe vector; and the per-step potential and thermostat
record of 10 MD steps plus the final positions and velocities.

Run in the build container (needs the reference sources):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from capacmd_b200 import configs  # noqa: E402
from oracle.oracle import RefSim  # noqa: E402

CASES = ["t_au13", "t_au55w", "t_2np", "t_water", "c1", "c1_field", "t_bonded"]
MD_STEPS = 10


def make(case: str) -> None:
    out = os.path.join(HERE, case)
    paths = configs.write(case, out, steps=MD_STEPS)
    ref = RefSim(paths)
    rec = {}
    for k in ("fx", "fy", "fz", "potential", "virial", "vec_pq", "vec_ext", "diag_relay", "inv_sqrt_dens",
              "thermo", "vQ"):
        rec[k] = ref.get(k)
    cnt, h = ref.pair_fingerprint()
    rec["pair_count"] = np.array(cnt, dtype=np.int64)
    rec["pair_hash"] = np.array(h, dtype=np.uint64)
    n = ref.n_mat
    if n > 0:
        probe = np.random.default_rng(123).normal(size=n)
        rec["mv_x"] = probe
        rec["mv_y"] = ref.matvec(probe)
    pots, thermo = [], []
    for _ in range(MD_STEPS):
        ref.md_steps(1)
        pots.append(ref.get("potential"))
        thermo.append(ref.get("thermo"))
    rec["md_potential"] = np.array(pots)
    rec["md_thermo"] = np.array(thermo)
    for k in ("rx", "ry", "rz", "vx", "vy", "vz", "fx", "fy", "fz", "vec_pq"):
        rec["md_" + k] = ref.get(k)
    np.savez_compressed(os.path.join(out, "ref.npz"), **rec)
    print(f"{case}: {ref.n_atoms} atoms, n_mat {n}, pairs {cnt}")


def main() -> int:
    for c in (sys.argv[1:] or CASES):
        make(c)
    return 0


if __name__ == "__main__":
    sys.exit(main())

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

Large systems (``c3``, the 91k-atom two-particle system in a field) keep
their inputs out of the repository: the seeded generator rebuilds them, and
ref.npz stores the SHA-256 of the three generated files so a test can tell
that it runs on the same input.  Their record holds one force call (no MD),
with the forces of a seeded sample of atoms (every metal atom plus 3,000
others) and the sum of squares of all forces.  One reference force call on
c3 takes about two minutes on one core.

Run in the build container (needs the reference sources):
    python tests/golden/make_golden.py            # small cases
    python tests/golden/make_golden.py c3         # the large case
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from capacmd_b200 import configs  # noqa: E402
from conftest import input_digest  # noqa: E402
from oracle.oracle import RefSim  # noqa: E402

CASES = ["t_au13", "t_au55w", "t_2np", "t_water", "c1", "c1_field", "t_bonded", "t_morse_buck"]
LARGE = ["c3"]
MD_STEPS = 10
SAMPLE_OTHERS = 3000


def sample_atoms(n_atoms: int, n_metal: int, metal_min: int = 0) -> np.ndarray:
    """Every metal atom plus a seeded sample of the others, sorted."""
    rest = np.setdiff1d(np.arange(n_atoms), np.arange(metal_min, metal_min + n_metal))
    pick = np.random.default_rng(2024).choice(rest, size=min(SAMPLE_OTHERS, len(rest)), replace=False)
    return np.sort(np.concatenate([np.arange(metal_min, metal_min + n_metal), pick])).astype(np.int64)


def make_large(case: str) -> None:
    out = os.path.join(HERE, case)
    os.makedirs(out, exist_ok=True)
    paths = configs.write(case, os.path.join(ROOT, "build", "configs", case))
    ref = RefSim(paths)
    rec = {"input_sha256": np.array(input_digest(paths))}
    for k in ("potential", "virial", "vec_pq", "vec_ext", "diag_relay", "inv_sqrt_dens"):
        rec[k] = ref.get(k)
    f = ref.forces()
    idx = sample_atoms(ref.n_atoms, paths["n_metal"])
    rec["sample"] = idx
    rec["sample_f"] = f[idx]
    rec["f_sumsq"] = np.array((f * f).sum())
    rec["f_absmax"] = np.array(np.abs(f).max())
    cnt, h = ref.pair_fingerprint()
    rec["pair_count"] = np.array(cnt, dtype=np.int64)
    rec["pair_hash"] = np.array(h, dtype=np.uint64)
    probe = np.random.default_rng(123).normal(size=ref.n_mat)
    rec["mv_x"] = probe
    rec["mv_y"] = ref.matvec(probe)
    np.savez_compressed(os.path.join(out, "ref.npz"), **rec)
    print(f"{case}: {ref.n_atoms} atoms, n_mat {ref.n_mat}, pairs {cnt}")


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
        (make_large if c in LARGE else make)(c)
    return 0


if __name__ == "__main__":
    sys.exit(main())

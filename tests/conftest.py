import hashlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["t_au13", "t_au55w", "t_2np", "t_water", "c1", "c1_field", "t_morse_buck"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the built CUDA library")


def golden_paths(case: str) -> dict:
    d = os.path.join(GOLDEN, case)
    return {"gro": os.path.join(d, "init.gro"), "par": os.path.join(d, "param.txt"),
            "mds": os.path.join(d, "mdset.txt")}


def golden_ref(case: str) -> dict:
    with np.load(os.path.join(GOLDEN, case, "ref.npz")) as z:
        return {k: z[k] for k in z.files}


def input_digest(paths: dict) -> str:
    """SHA-256 over the three input files, in the order gro, param, mdset."""
    h = hashlib.sha256()
    for k in ("gro", "par", "mds"):
        with open(paths[k], "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def large_case(case: str) -> tuple[dict, dict]:
    """Inputs of a large golden case, rebuilt by the seeded generator (their
    files are not stored), with the reference's record of them; fails if the
    generator no longer writes the inputs the record was made from."""
    from capacmd_b200 import configs
    paths = configs.cached(case)
    g = golden_ref(case)
    assert input_digest(paths) == str(g["input_sha256"]), f"{case}: generated inputs differ from the golden's"
    return paths, g


def rel_err(a, b) -> float:
    """max |a - b| / max |b| (normwise relative error)."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    if b.size == 0:
        return 0.0
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / scale) if scale > 0 else float(np.max(np.abs(a)))


def slot_rel_err(a, b) -> float:
    """Largest relative error over the non-zero potential slots."""
    a, b = np.asarray(a), np.asarray(b)
    m = np.abs(b) > 0
    if not m.any():
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a[m] - b[m]) / np.abs(b[m])))


@pytest.fixture(scope="session")
def gpu_available() -> bool:
    try:
        import torch
        if not torch.cuda.is_available():
            return False
        return torch.cuda.get_device_capability(0)[0] == 10
    except Exception:
        return False


def variant(case: str, out_dir: str, par=None, mds=None) -> dict:
    """A golden case's three inputs written to out_dir under the reference
    program's default names, with param.txt / mdset.txt text passed through
    the given functions."""
    src = golden_paths(case)
    names = {"gro": "init.gro", "par": "param.txt", "mds": "mdset.txt"}
    edit = {"par": par, "mds": mds}
    os.makedirs(str(out_dir), exist_ok=True)
    out = {}
    for k, p in src.items():
        text = open(p).read()
        if edit.get(k):
            new = edit[k](text)
            assert new != text, f"{k}: the edit changed nothing"
            text = new
        out[k] = os.path.join(str(out_dir), names[k])
        with open(out[k], "w") as f:
            f.write(text)
    return out


def impossible_constraints(text: str) -> str:
    """t_water's param.txt with an H-H constraint longer than the two O-H
    constraints together: no geometry satisfies it, so RATTLE cannot converge
    (the reference stops with "RATTLE_1 not converged!", force.c:1990-1994)."""
    return text.replace("1 2   0.163298", "1 2   0.300000")


def berendsen(tau: float, ref_t: float | None = None):
    """An mdset.txt edit selecting the Berendsen thermostat with coupling time
    tau (ps) and, if given, another reference temperature (K)."""
    def edit(text: str) -> str:
        out = []
        for line in text.splitlines():
            key = line.split()[0] if line.split() else ""
            if key == "ensemble":
                line = "ensemble          berendsen"
            elif key == "tau_T_in_ps":
                line = f"tau_T_in_ps       {tau!r}"
            elif key == "ref_T_in_K" and ref_t is not None:
                line = f"ref_T_in_K        {ref_t!r}"
            out.append(line)
        return "\n".join(out) + "\n"
    return edit

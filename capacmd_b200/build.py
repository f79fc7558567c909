"""Build the CUDA library in-tree (sm_100a) and the CPU oracles.

    python -m capacmd_b200.build [--reference DIR]

builds the library, the resident driver and the C oracle; with the reference
sources given (--reference, else the CAPAC_REFERENCE_SRC environment
variable) also the reference compiled in place (oracle/_ref).

The library is ``capacmd_b200/libcapacmd_gpu.so``: host C++ (input parsing,
orchestration, C ABI) and the sm_100a kernels, linked against the CUDA runtime.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "build", "obj")
LIB = os.path.join(PKG, "libcapacmd_gpu.so")
DRIVER = os.path.join(PKG, "capacmd-gpu")

SOURCES = ["io.cpp", "api.cu", "k_list.cu", "k_pair.cu", "k_cpim.cu", "k_md.cu", "k_cpim_sym.cu", "k_solve_static.cu", "k_solve_coop.cu",
           "k_precond.cu", "k_coarse.cu", "k_grad.cu", "k_grad_forces.cu", "k_bonded.cu"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _flags() -> list[str]:
    return ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
            "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall", f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}",
            "--expt-relaxed-constexpr"]


def _compile(src: str, verbose: bool) -> str:
    out = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "capacmd.h"))
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return out
    cmd = [nvcc()] + _flags() + ["-c", path, "-o", out]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return out


def build_library(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB] + objs + [
            "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def build_driver(verbose: bool = False) -> str:
    """The resident driver (reference command line and files, run on the GPU)."""
    src = os.path.join(PKG, "driver", "capacmd_gpu.cpp")
    deps = [src, LIB, os.path.join(ROOT, "include", "capacmd.h")]
    if os.path.exists(DRIVER) and os.path.getmtime(DRIVER) >= max(os.path.getmtime(d) for d in deps):
        return DRIVER
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", f"-I{os.path.join(ROOT, 'include')}", src, "-o", DRIVER,
           f"-L{PKG}", "-lcapacmd_gpu", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return DRIVER


def reference_dir(reference: str | None = None) -> str | None:
    """The reference source folder: the argument, else $CAPAC_REFERENCE_SRC;
    None when neither names an existing folder."""
    ref = reference or os.environ.get("CAPAC_REFERENCE_SRC")
    return ref if ref and os.path.isdir(ref) else None


def build_oracle(verbose: bool = False, reference: str | None = None) -> None:
    """Compile the C restatement and, where the reference sources are given,
    the reference itself (oracle/_ref)."""
    odir = os.path.join(ROOT, "oracle")
    subprocess.run(["make", "-s", "-C", odir], check=True)
    ref = reference_dir(reference)
    if ref:
        subprocess.run(["make", "-s", "-C", odir, "ref", f"REF={ref}"], check=True)
        if os.path.exists(LIB):
            # the reference driver with its mpi_force calls sent to this library
            subprocess.run(["make", "-s", "-C", odir, "dropin", f"REF={ref}"], check=True)


def main() -> int:
    verbose = "-v" in sys.argv
    reference = sys.argv[sys.argv.index("--reference") + 1] if "--reference" in sys.argv[:-1] else None
    build_library(verbose)
    build_driver(verbose)
    build_oracle(verbose, reference)
    print(LIB)
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""ctypes wrappers of the two CPU oracles (test infrastructure only).

``Oracle``  -- oracle/liboracle.so, our plain-C restatement of the reference
               path (oracle/capac_oracle.c); takes a parsed ``capacmd_b200.Desc``.
``RefSim``  -- oracle/_ref/libcapref.so, the reference sources compiled in
               place with a single-rank MPI stub (oracle/ref_harness.cpp);
               reads the three input files itself.  Present only where the
               reference sources were available at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product library never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libcapref.so")

_orc = None
_ref = None


def _orc_lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            raise FileNotFoundError(f"{ORACLE_LIB} missing: run `make -C oracle`")
        L = ctypes.CDLL(ORACLE_LIB)
        vp, cp = ctypes.c_void_p, ctypes.c_char_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [vp, ctypes.c_double]
        for f in ("orc_destroy", "orc_md_init", "orc_zero", "orc_nonbonded", "orc_qsc", "orc_cpff_vec_ext",
                  "orc_cpff_mat_relay", "orc_cpff_force"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = None
        for f in ("orc_force", "orc_force_given_pq", "orc_bicgstab", "orc_iterations", "orc_step"):
            getattr(L, f).argtypes = [vp]
        L.orc_md_steps.argtypes = [vp, ctypes.c_int]
        L.orc_get.argtypes = [vp, cp, vp]
        L.orc_set.argtypes = [vp, cp, vp]
        L.orc_matvec.argtypes = [vp, vp, vp]
        L.orc_matvec.restype = None
        L.orc_pair_fingerprint.argtypes = [vp, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_ulonglong)]
        L.orc_pair_fingerprint.restype = None
        L.orc_pair_fingerprint_cells.argtypes = L.orc_pair_fingerprint.argtypes
        L.orc_pair_fingerprint_cells.restype = None
        L.orc_set_sample.argtypes = [vp, vp, ctypes.c_int]
        _orc = L
    return _orc


class Oracle:
    """The C restatement on a parsed description (capacmd_b200.Desc)."""

    def __init__(self, desc, solver_tol: float = 1e-8):
        self.desc = desc  # keeps the description alive
        self.n_atoms = desc.n_atoms
        self.n_mat = desc.n_mat
        self._p = _orc_lib().orc_create(desc.ptr, solver_tol)
        if not self._p:
            raise MemoryError("orc_create failed")

    def __del__(self):
        try:
            if self._p:
                _orc_lib().orc_destroy(self._p)
                self._p = None
        except Exception:
            pass

    def force(self) -> int:
        return _orc_lib().orc_force(self._p)

    def force_given_pq(self) -> int:
        return _orc_lib().orc_force_given_pq(self._p)

    def md_init(self) -> None:
        _orc_lib().orc_md_init(self._p)

    def md_steps(self, n: int) -> int:
        return _orc_lib().orc_md_steps(self._p, int(n))

    def stage(self, name: str):
        return getattr(_orc_lib(), "orc_" + name)(self._p)

    def iterations(self) -> int:
        return _orc_lib().orc_iterations(self._p)

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(max(self.n_atoms, self.n_mat, 16))
        n = _orc_lib().orc_get(self._p, name.encode(), out.ctypes.data)
        if n < 0:
            raise KeyError(name)
        return out[:n].copy()

    def set(self, name: str, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        if _orc_lib().orc_set(self._p, name.encode(), v.ctypes.data) < 0:
            raise KeyError(name)

    def matvec(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x)
        _orc_lib().orc_matvec(self._p, x.ctypes.data, y.ctypes.data)
        return y

    def forces(self) -> np.ndarray:
        return np.stack([self.get("fx"), self.get("fy"), self.get("fz")], 1)

    def pair_fingerprint(self, cells: bool = False) -> tuple[int, int]:
        """Count and hash of the reference's pair set: all-pairs loop, or
        (cells=True) the same set found through a cell search."""
        c, h = ctypes.c_long(0), ctypes.c_ulonglong(0)
        fn = _orc_lib().orc_pair_fingerprint_cells if cells else _orc_lib().orc_pair_fingerprint
        fn(self._p, ctypes.byref(c), ctypes.byref(h))
        return c.value, h.value

    def set_sample(self, atoms) -> None:
        """Form nonbonded forces only on these atoms in later force calls
        (all their pairs; no pair energies or virial); empty restores."""
        self._sample = np.ascontiguousarray(atoms, dtype=np.int64)
        if _orc_lib().orc_set_sample(self._p, self._sample.ctypes.data, len(self._sample)) != 0:
            raise ValueError("sample index out of range")


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _ref_lib():
    global _ref
    if _ref is None:
        L = ctypes.CDLL(REF_LIB)
        vp, cp = ctypes.c_void_p, ctypes.c_char_p
        L.capref_open.restype = vp
        L.capref_open.argtypes = [cp, cp, cp]
        for f in ("capref_force",):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = None
        L.capref_md_steps.argtypes = [vp, ctypes.c_int]
        L.capref_md_steps.restype = None
        L.capref_time_md_steps.argtypes = [vp, ctypes.c_int]
        L.capref_time_md_steps.restype = ctypes.c_double
        for f in ("capref_n_atoms", "capref_n_mat", "capref_n_metal", "capref_step"):
            getattr(L, f).argtypes = [vp]
        L.capref_nnz.argtypes = [vp]
        L.capref_nnz.restype = ctypes.c_long
        L.capref_get.argtypes = [vp, cp, vp]
        L.capref_set.argtypes = [vp, cp, vp]
        L.capref_matvec.argtypes = [vp, vp, vp]
        L.capref_matvec.restype = None
        L.capref_pair_fingerprint.argtypes = [vp, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_ulonglong)]
        L.capref_pair_fingerprint.restype = None
        _ref = L
    return _ref


class RefSim:
    """The reference sources themselves (single rank), opened on input files.

    Opening performs the reference's first force call (mpi-main.c:614) and its
    start-up thermostat bookkeeping (mpi-main.c:629-655)."""

    def __init__(self, paths: dict):
        L = _ref_lib()
        self._p = L.capref_open(paths["gro"].encode(), paths["par"].encode(), paths["mds"].encode())
        if not self._p:
            raise RuntimeError("reference failed to open the inputs")
        self.n_atoms = L.capref_n_atoms(self._p)
        self.n_mat = L.capref_n_mat(self._p)

    def force(self) -> None:
        _ref_lib().capref_force(self._p)

    def md_steps(self, n: int) -> None:
        _ref_lib().capref_md_steps(self._p, int(n))

    def time_md_steps(self, n: int) -> float:
        return _ref_lib().capref_time_md_steps(self._p, int(n))

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(max(self.n_atoms, self.n_mat, 16))
        n = _ref_lib().capref_get(self._p, name.encode(), out.ctypes.data)
        if n < 0:
            raise KeyError(name)
        return out[:n].copy()

    def set(self, name: str, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        if _ref_lib().capref_set(self._p, name.encode(), v.ctypes.data) < 0:
            raise KeyError(name)

    def forces(self) -> np.ndarray:
        return np.stack([self.get("fx"), self.get("fy"), self.get("fz")], 1)


def _ref_matvec(self, x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x)
    _ref_lib().capref_matvec(self._p, x.ctypes.data, y.ctypes.data)
    return y


def _ref_pair_fingerprint(self) -> tuple[int, int]:
    c, h = ctypes.c_long(0), ctypes.c_ulonglong(0)
    _ref_lib().capref_pair_fingerprint(self._p, ctypes.byref(c), ctypes.byref(h))
    return c.value, h.value


RefSim.matvec = _ref_matvec
RefSim.pair_fingerprint = _ref_pair_fingerprint


def open_reference(paths: dict, first_force: bool = True) -> RefSim:
    """RefSim without (optionally) the reference's first force call."""
    L = _ref_lib()
    L.capref_open_ex.restype = ctypes.c_void_p
    L.capref_open_ex.argtypes = [ctypes.c_char_p] * 3 + [ctypes.c_int]
    obj = RefSim.__new__(RefSim)
    obj._p = L.capref_open_ex(paths["gro"].encode(), paths["par"].encode(), paths["mds"].encode(),
                              1 if first_force else 0)
    if not obj._p:
        raise RuntimeError("reference failed to open the inputs")
    obj.n_atoms = L.capref_n_atoms(obj._p)
    obj.n_mat = L.capref_n_mat(obj._p)
    return obj


def time_sampled_force(ref: RefSim, pair_frac: float) -> tuple[float, np.ndarray]:
    """Wall seconds of one reference force call whose pair loop covers the
    last `pair_frac` of the pairs, and the per-phase seconds (time_used slots)."""
    L = _ref_lib()
    L.capref_time_sampled_force.restype = ctypes.c_double
    L.capref_time_sampled_force.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
    ph = np.zeros(15)
    t = L.capref_time_sampled_force(ref._p, float(pair_frac), ph.ctypes.data)
    return t, ph

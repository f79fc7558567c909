"""B200 (sm_100a) implementation of CapacMD's per-timestep force-and-solve path.

Python mirror of the C ABI in ``include/capacmd.h`` (ctypes; no torch types).
The names follow the reference driver: ``mpi_force`` evaluates one force call
(force.h:100-103), ``md_steps`` runs the reference MD loop (mpi-main.c:874-1013)
on the device, and the CPIM stages keep the reference's names (cpff.h,
bicg_stab.h).  Errors raise :class:`CapacError` carrying the C status code; the
reference prints and exits instead.

The CUDA library is required: importing works without it, but every call that
needs it raises if ``libcapacmd_gpu.so`` is missing or no sm_100 device is
present.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libcapacmd_gpu.so")

OK = 0
ERR_INVALID = -1
ERR_IO = -2
ERR_CUDA = -3
ERR_NOT_CONVERGED = -4
ERR_RATTLE = -5
ERR_UNSUPPORTED = -6
ERR_CAPACITY = -7
ERR_NO_DEVICE = -8

PREC_FP64 = 0
PREC_MIXED = 1

# thermostats (CAPAC_NVE / CAPAC_NVT / CAPAC_BERENDSEN of capacmd.h), as mdset.txt's ensemble selects
NVE, NVT, BERENDSEN = 0, 1, 2

# bonded term kinds (CAPAC_BT_* of capacmd.h)
BT_BOND_HARMONIC, BT_BOND_MORSE, BT_PAIR_14, BT_PAIR_USER = 1, 2, 3, 4
BT_ANGLE_HARMONIC, BT_ANGLE_UB, BT_DIHEDRAL_RB = 5, 6, 7

# Metal parameters of capac_param_get/set, in the order of capac_energy_param_grad.
PARAMS = ("cpff_capac", "cpff_polar", "cpim_rq", "cpim_rp", "qsc_eps", "qsc_c", "qsc_a", "qsc_n", "qsc_m")


class CapacError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("device", ctypes.c_int), ("skin", ctypes.c_double),
                ("list_every", ctypes.c_int), ("max_neighbors", ctypes.c_int),
                ("solver_tol", ctypes.c_double), ("refine_tol", ctypes.c_double),
                ("matrix_layout", ctypes.c_int), ("predictor", ctypes.c_int), ("solver_kernel", ctypes.c_int),
                ("inner_precond", ctypes.c_int), ("pair_list", ctypes.c_int), ("max_iter", ctypes.c_int),
                ("wait_polls", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("solver_iterations", ctypes.c_int), ("solver_outer", ctypes.c_int),
                ("solver_rel_residual", ctypes.c_double), ("list_builds", ctypes.c_long),
                ("list_entries", ctypes.c_long), ("max_neighbors", ctypes.c_long),
                ("list_capacity", ctypes.c_int), ("md_step", ctypes.c_long),
                ("solver_initial_rel_residual", ctypes.c_double)]


class Consts(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("r_cut2", "w_a2_sqrtpi", "w_const", "w_erfc_arcut",
                                               "inv_rc12", "inv_rc6", "inv_polar", "inv_capac",
                                               "inv_r_qq", "inv_r_pq", "inv_r_pp")] + [
        ("ndf", ctypes.c_int), ("kT", ctypes.c_double), ("q_mass", ctypes.c_double),
        ("dt_2", ctypes.c_double), ("n_mat", ctypes.c_int)]


_lib: Optional[ctypes.CDLL] = None


def lib() -> ctypes.CDLL:
    """The loaded CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CapacError(ERR_NO_DEVICE, f"{LIB_PATH} is missing: run `python -m capacmd_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp, cp, ip, dp = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    L.capac_last_error.restype = cp
    L.capac_desc_load.argtypes = [cp, cp, cp, ctypes.POINTER(vp)]
    L.capac_desc_free.argtypes = [vp]
    L.capac_desc_free.restype = None
    L.capac_desc_derive.argtypes = [vp, ctypes.POINTER(Consts)]
    L.capac_desc_get.argtypes = [vp, cp, vp]
    L.capac_desc_info.argtypes = [vp] + [ctypes.POINTER(ctypes.c_int)] * 5
    L.capac_options_default.argtypes = [ctypes.POINTER(Options)]
    L.capac_options_default.restype = None
    L.capac_create.argtypes = [vp, ctypes.POINTER(Options), ctypes.POINTER(vp)]
    L.capac_destroy.argtypes = [vp]
    for f in ("capac_force", "capac_qsc", "capac_cpff_vec_ext", "capac_cpff_force", "capac_md_init"):
        getattr(L, f).argtypes = [vp]
    L.capac_mpi_force.argtypes = [vp] + [vp] * 12
    L.capac_cpff_mat_relay.argtypes = [vp, ctypes.POINTER(ctypes.c_long)]
    L.capac_bicgstab.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.capac_md_steps.argtypes = [vp, ip]
    L.capac_get.argtypes = [vp, cp, vp]
    L.capac_set.argtypes = [vp, cp, vp]
    L.capac_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
    L.capac_pair_fingerprint.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_long),
                                         ctypes.POINTER(ctypes.c_ulonglong)]
    L.capac_phase_times.argtypes = [vp, dp]
    L.capac_kernel_launches.argtypes = [vp]
    L.capac_kernel_launches.restype = ctypes.c_long
    L.capac_param_get.argtypes = [vp, cp, dp]
    L.capac_param_set.argtypes = [vp, cp, ctypes.c_double]
    L.capac_energy_grad.argtypes = [vp, dp, dp, dp, dp]
    L.capac_force_match_grad.argtypes = [vp, dp, dp, dp, dp, dp, dp, dp, dp]
    _lib = L
    return L


def _check(rc: int) -> int:
    if rc < 0:
        raise CapacError(rc, lib().capac_last_error().decode(errors="replace"))
    return rc


class Desc:
    """A parsed system: the reference's mdset.txt, param.txt and .gro."""

    def __init__(self, gro: str, par: str, mds: str):
        self._p = ctypes.c_void_p()
        _check(lib().capac_desc_load(gro.encode(), par.encode(), mds.encode(), ctypes.byref(self._p)))
        probe = np.zeros(3)
        lib().capac_desc_get(self._p, b"box", probe.ctypes.data)
        self.box = probe.copy()
        c = Consts()
        _check(lib().capac_desc_derive(self._p, ctypes.byref(c)))
        self.consts = c
        info = [ctypes.c_int(0) for _ in range(5)]
        _check(lib().capac_desc_info(self._p, *[ctypes.byref(v) for v in info]))
        self.n_atoms, self.n_mols, self.n_metal, self.n_nps, self.n_mat = (v.value for v in info)

    @classmethod
    def from_paths(cls, paths: dict) -> "Desc":
        return cls(paths["gro"], paths["par"], paths["mds"])

    @property
    def ptr(self) -> ctypes.c_void_p:
        return self._p

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(max(self.n_atoms, 3))
        n = _check(lib().capac_desc_get(self._p, name.encode(), out.ctypes.data))
        return out[:n].copy()

    def __del__(self):
        try:
            if self._p:
                lib().capac_desc_free(self._p)
                self._p = ctypes.c_void_p()
        except Exception:
            pass


class Simulation:
    """Device-resident state of one system on one B200."""

    def __init__(self, desc: Desc, precision: int = PREC_FP64, device: int = 0, skin: float = 0.2,
                 solver_tol: float = 0.0, refine_tol: float = 1e-10, max_neighbors: int = 0,
                 matrix_layout: int = 0, predictor: int = 3, solver_kernel: int = 0, inner_precond: int = 3,
                 pair_list: int = 0, max_iter: int = 0, wait_polls: int = 0):
        self.desc = desc
        o = Options()
        lib().capac_options_default(ctypes.byref(o))
        o.precision, o.device, o.skin = precision, device, skin
        o.solver_tol, o.refine_tol, o.max_neighbors = solver_tol, refine_tol, max_neighbors
        o.matrix_layout, o.predictor, o.solver_kernel = matrix_layout, predictor, solver_kernel
        o.inner_precond = inner_precond
        o.pair_list = pair_list
        o.max_iter, o.wait_polls = max_iter, wait_polls
        self._p = ctypes.c_void_p()
        _check(lib().capac_create(desc.ptr, ctypes.byref(o), ctypes.byref(self._p)))
        self.n_atoms = desc.n_atoms
        self.n_mat = desc.n_mat

    def close(self):
        if getattr(self, "_p", None):
            lib().capac_destroy(self._p)
            self._p = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- the reference's entry points -------------------------------------
    def force(self) -> None:
        """mpi_force on the device-resident state (force.c:2097-2320)."""
        _check(lib().capac_force(self._p))

    def mpi_force(self, rx, ry, rz, vec_pq=None) -> dict:
        """mpi_force with host arrays in and out (drop-in mode)."""
        N = self.n_atoms
        rx, ry, rz = (np.ascontiguousarray(a, dtype=np.float64) for a in (rx, ry, rz))
        out = {k: np.zeros(N) for k in ("fx", "fy", "fz")}
        out["potential"] = np.zeros(15)
        out["virial"] = np.zeros(9)
        n = max(self.n_mat, 1)
        pq = np.zeros(n) if vec_pq is None else np.ascontiguousarray(vec_pq, dtype=np.float64).copy()
        ext, diag, isd = np.zeros(n), np.zeros(n), np.zeros(max(self.desc.n_metal, 1))
        _check(lib().capac_mpi_force(self._p, rx.ctypes.data, ry.ctypes.data, rz.ctypes.data,
                                     out["fx"].ctypes.data, out["fy"].ctypes.data, out["fz"].ctypes.data,
                                     out["potential"].ctypes.data, out["virial"].ctypes.data,
                                     pq.ctypes.data if vec_pq is not None else None,
                                     ext.ctypes.data, diag.ctypes.data, isd.ctypes.data))
        out.update(vec_pq=pq, vec_ext=ext, diag_relay=diag)
        return out

    def qsc(self) -> None:
        _check(lib().capac_qsc(self._p))

    def cpff_vec_ext(self) -> None:
        _check(lib().capac_cpff_vec_ext(self._p))

    def cpff_mat_relay(self) -> int:
        nnz = ctypes.c_long(0)
        _check(lib().capac_cpff_mat_relay(self._p, ctypes.byref(nnz)))
        return nnz.value

    def bicgstab(self) -> int:
        it = ctypes.c_int(0)
        _check(lib().capac_bicgstab(self._p, ctypes.byref(it)))
        return it.value

    def cpff_force(self) -> None:
        _check(lib().capac_cpff_force(self._p))

    def md_init(self) -> None:
        _check(lib().capac_md_init(self._p))

    def md_steps(self, n: int) -> None:
        _check(lib().capac_md_steps(self._p, int(n)))

    # --- state --------------------------------------------------------------
    def get(self, name: str) -> np.ndarray:
        out = np.zeros(max(self.n_atoms, self.n_mat, 16))
        n = _check(lib().capac_get(self._p, name.encode(), out.ctypes.data))
        return out[:n].copy()

    def set(self, name: str, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        _check(lib().capac_set(self._p, name.encode(), v.ctypes.data))

    def forces(self) -> np.ndarray:
        return np.stack([self.get("fx"), self.get("fy"), self.get("fz")], 1)

    def positions(self) -> np.ndarray:
        return np.stack([self.get("rx"), self.get("ry"), self.get("rz")], 1)

    def stats(self) -> Stats:
        s = Stats()
        _check(lib().capac_get_stats(self._p, ctypes.byref(s)))
        return s

    def pair_fingerprint(self, from_list: bool = True) -> tuple[int, int]:
        cnt, h = ctypes.c_long(0), ctypes.c_ulonglong(0)
        _check(lib().capac_pair_fingerprint(self._p, 1 if from_list else 0, ctypes.byref(cnt), ctypes.byref(h)))
        return cnt.value, h.value

    def phase_times(self) -> np.ndarray:
        out = np.zeros(15)
        _check(lib().capac_phase_times(self._p, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def kernel_launches(self) -> int:
        return int(lib().capac_kernel_launches(self._p))

    def param_get(self, name: str) -> float:
        """A metal parameter by its name in PARAMS (capac_param_get)."""
        v = ctypes.c_double(0.0)
        _check(lib().capac_param_get(self._p, name.encode(), ctypes.byref(v)))
        return v.value

    def param_set(self, name: str, value: float) -> None:
        """Set a metal parameter; the next force call uses it (capac_param_set)."""
        _check(lib().capac_param_set(self._p, name.encode(), float(value)))

    def energy_grad(self, positions: bool = True) -> tuple[dict, Optional[np.ndarray]]:
        """Total dE/dθ (dict over PARAMS, kJ/mol per unit) and dE/dr ((N, 3)
        kJ/mol/nm, or None) of the last force call (capac_energy_grad)."""
        g = np.zeros(len(PARAMS))
        n = self.desc.n_atoms
        xyz = [np.zeros(n) for _ in range(3)] if positions else [None] * 3
        ptr = [a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None for a in xyz]
        _check(lib().capac_energy_grad(self._p, g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), *ptr))
        return dict(zip(PARAMS, g.tolist())), (np.stack(xyz, 1) if positions else None)

    def force_match_grad(self, target: np.ndarray, positions: bool = False):
        """Force-matching loss mean((F - target)^2) over atoms and axes, its
        gradient over PARAMS and, with positions=True, dL/dr as (N, 3)
        (capac_force_match_grad); target is (N, 3)."""
        t = np.ascontiguousarray(np.asarray(target, dtype=np.float64).T)
        g = np.zeros(len(PARAMS))
        loss = ctypes.c_double(0.0)
        dpt = ctypes.POINTER(ctypes.c_double)
        n = self.desc.n_atoms
        xyz = [np.zeros(n) for _ in range(3)] if positions else [None] * 3
        ptr = [a.ctypes.data_as(dpt) if a is not None else None for a in xyz]
        _check(lib().capac_force_match_grad(self._p, t[0].ctypes.data_as(dpt), t[1].ctypes.data_as(dpt),
                                            t[2].ctypes.data_as(dpt), ctypes.byref(loss), g.ctypes.data_as(dpt),
                                            *ptr))
        if positions:
            return loss.value, dict(zip(PARAMS, g.tolist())), np.stack(xyz, 1)
        return loss.value, dict(zip(PARAMS, g.tolist()))


def load(paths: dict) -> Desc:
    return Desc.from_paths(paths)

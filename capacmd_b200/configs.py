"""Seeded synthetic inputs in CapacMD's own file formats.

The reference ships no benchmark inputs for the workloads this package is
measured on, so they are generated here: Mackay icosahedral gold nanoparticles
(optionally two, and optionally in a uniform external field), surrounded by
rigid 3-site water placed on a cubic lattice with random orientations, with
waters closer than 0.3 nm to any gold atom removed.  Velocities are
Maxwell-Boltzmann at the requested temperature with the water constraints
projected out.  Output: ``init.gro``, ``param.txt`` and ``mdset.txt`` in the
formats read by the reference (file.c:74-203, file.c:286-1023).

Units are the reference's (nm, ps, kJ/mol, e, amu).  Water charges, masses and
the Au-water erf-vdW and O-O LJ parameters are the reference example's
(example_01/param.txt:10-21); the Sutton-Chen and CPIM gold parameters are the
workload's (Sutton-Chen Au: eps 0.012793 eV, c 34.408, a 0.408 nm, n 10, m 8;
CPIM polarizability 39.5297 and capacitance 1.2159 a.u.).
"""
from __future__ import annotations

import dataclasses
import os
from typing import Sequence

import numpy as np

EV2KJMOL = 96.4853363969351
K_BOLTZ = 0.00831446214546895
AU_NN = 0.2884  # nm, Au nearest-neighbour distance
OH = 0.1  # nm
HOH_DEG = 109.47
M_AU, M_O, M_H = 196.97, 16.0, 1.008
Q_O, Q_H = -0.834, 0.417


@dataclasses.dataclass
class Workload:
    """One synthetic system: nanoparticles, water, box and run settings."""

    name: str
    shells: Sequence[int]  # Mackay shells per nanoparticle (3 -> Au147, 4 -> Au309, ...)
    n_waters: int
    box: float
    seed: int
    ensemble: str = "nvt"
    steps: int = 100
    dt: float = 0.001
    efield_vnm: tuple = (0.0, 0.0, 0.0)
    gap_z: float | None = None  # surface gap between two particles along z
    temperature: float = 300.0
    save_step: int = 10
    use_cpff: int = 1
    # NONBONDED lines replacing the default table, upper triangle of types
    # (Au, O, H): Au-Au, Au-O, Au-H, O-O, O-H, H-H
    nonbonded: tuple | None = None


# The five measured workloads plus small systems for tests.  Sizes: c1 147
# atoms; c2 ~9.3k; c3 ~91k (two Au561, 0.5 V/nm along z); c4 ~3.1k; c5 ~452k.
WORKLOADS = {
    "c1": Workload("c1", [3], 0, 6.0, seed=0, ensemble="nve", steps=1000),
    "c1_field": Workload("c1_field", [3], 0, 6.0, seed=0, ensemble="nve", steps=1000,
                         efield_vnm=(0.0, 0.0, 0.5)),
    "c2": Workload("c2", [4], 3000, 4.5, seed=1, steps=5000),
    # the same system under the Berendsen thermostat the workload's
    # description names (the reference has only the Nose-Hoover chain, so
    # "c2" keeps that for comparisons with it)
    "c2_berendsen": Workload("c2_berendsen", [4], 3000, 4.5, seed=1, ensemble="berendsen", steps=5000),
    # the same system without thermostat, for energy-drift measurements, with
    # two more seeds and, per seed, a variant without CPIM (the floor of the
    # integrator and RATTLE alone)
    "c2_nve": Workload("c2_nve", [4], 3000, 4.5, seed=1, ensemble="nve", steps=5000),
    **{f"c2_nve_s{k}": Workload(f"c2_nve_s{k}", [4], 3000, 4.5, seed=k, ensemble="nve", steps=5000)
       for k in (2, 3)},
    **{f"c2_nve_nocpim_s{k}": Workload(f"c2_nve_nocpim_s{k}", [4], 3000, 4.5, seed=k, ensemble="nve", steps=5000,
                                        use_cpff=0) for k in (1, 2, 3)},
    "c3": Workload("c3", [5, 5], 30000, 9.65, seed=2, steps=2000, efield_vnm=(0.0, 0.0, 0.5),
                   gap_z=1.5),
    "c4": Workload("c4", [3], 1000, 3.1, seed=3, steps=6400),
    "c5": Workload("c5", [8], 150000, 16.5, seed=4, steps=10000),
    # test systems
    "t_au13": Workload("t_au13", [1], 0, 4.0, seed=5, ensemble="nve", steps=20,
                       efield_vnm=(0.3, 0.0, 0.5)),
    "t_au55w": Workload("t_au55w", [2], 150, 2.9, seed=6, steps=20, efield_vnm=(0.0, 0.2, 0.0)),
    "t_2np": Workload("t_2np", [2, 2], 400, 4.2, seed=7, steps=20, efield_vnm=(0.0, 0.0, 0.5),
                      gap_z=0.8),
    "t_water": Workload("t_water", [], 120, 1.7, seed=8, steps=20, use_cpff=0),
    # Au-O as Buckingham (funct 2: A kJ/mol, B 1/nm, C6 kJ mol^-1 nm^6) and Au-H
    # as Morse (funct 3: D kJ/mol, a 1/nm, R nm), the two nonbonded forms no
    # other input uses (force.c:639-703); no CPIM, so a trace has no solver noise
    "t_morse_buck": Workload("t_morse_buck", [2], 150, 2.9, seed=9, steps=20, use_cpff=0,
                             nonbonded=(" 1    0.00000000e+00      0.00000000e+00",
                                        " 2    1.0e+05    30.0    2.0e-03",
                                        " 3    5.0    20.0    0.28",
                                        " 1    2.48970844e-03      2.43509761e-06",
                                        " 1    0.00000000e+00      0.00000000e+00",
                                        " 1    0.00000000e+00      0.00000000e+00")),
}


def icosahedron(shells: int, nn: float = AU_NN) -> np.ndarray:
    """Mackay icosahedron with `shells` shells around one centre atom.

    Shell k holds the 12 vertices of an icosahedron of edge k*nn, k-1 points on
    each of its 30 edges and (k-1)(k-2)/2 points inside each of its 20 faces:
    10k^2+2 atoms, so 1, 13, 55, 147, 309, 561, 923, 1415, 2057 in total.
    """
    g = (1.0 + 5.0 ** 0.5) / 2.0
    v = []
    for a in (-1.0, 1.0):
        for b in (-g, g):
            v += [(0.0, a, b), (a, b, 0.0), (b, 0.0, a)]
    v = np.array(v) / 2.0  # edge length 1
    d2 = ((v[:, None, :] - v[None, :, :]) ** 2).sum(-1)
    edges = [(i, j) for i in range(12) for j in range(i + 1, 12) if abs(d2[i, j] - 1.0) < 1e-9]
    faces = [(i, j, k) for (i, j) in edges for k in range(j + 1, 12)
             if abs(d2[i, k] - 1.0) < 1e-9 and abs(d2[j, k] - 1.0) < 1e-9]
    assert len(edges) == 30 and len(faces) == 20
    pts = [np.zeros(3)]
    for k in range(1, shells + 1):
        s = v * k * nn
        pts += list(s)
        for (i, j) in edges:
            for t in range(1, k):
                pts.append(s[i] + (s[j] - s[i]) * t / k)
        for (i, j, l) in faces:
            for a in range(1, k):
                for b in range(1, k - a):
                    pts.append(s[i] + (s[j] - s[i]) * a / k + (s[l] - s[i]) * b / k)
    out = np.array(pts)
    assert len(out) == 1 + sum(10 * k * k + 2 for k in range(1, shells + 1))
    return out


def _water_local() -> np.ndarray:
    half = np.deg2rad(HOH_DEG) / 2.0
    return np.array([[0.0, 0.0, 0.0],
                     [OH * np.sin(half), 0.0, OH * np.cos(half)],
                     [-OH * np.sin(half), 0.0, OH * np.cos(half)]])


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def _min_dist_to(points: np.ndarray, targets: np.ndarray, box: float) -> np.ndarray:
    """Minimum-image distance from each point to the nearest target."""
    out = np.full(len(points), np.inf)
    if len(targets) == 0:
        return out
    for s in range(0, len(points), 4096):
        p = points[s:s + 4096]
        d = p[:, None, :] - targets[None, :, :]
        d -= box * np.round(d / box)
        out[s:s + 4096] = np.sqrt((d * d).sum(-1)).min(1)
    return out


def build(w: Workload):
    """Positions, velocities and topology arrays of a workload (no files)."""
    rng = np.random.default_rng(w.seed)
    L = w.box
    centre = np.full(3, L / 2.0)
    nps = []
    if len(w.shells) == 1:
        nps.append(icosahedron(w.shells[0]) + centre)
    elif len(w.shells) == 2:
        a, b = icosahedron(w.shells[0]), icosahedron(w.shells[1])
        ra, rb = np.abs(a[:, 2]).max(), np.abs(b[:, 2]).max()
        gap = w.gap_z if w.gap_z is not None else 1.0
        nps.append(a + centre + [0.0, 0.0, -(gap / 2.0 + ra)])
        nps.append(b + centre + [0.0, 0.0, gap / 2.0 + rb])
    elif len(w.shells) > 2:
        raise ValueError("at most two nanoparticles")
    metal = np.concatenate(nps) if nps else np.zeros((0, 3))

    water = np.zeros((0, 3, 3))
    if w.n_waters > 0:
        n = int(np.ceil((w.n_waters * 1.25) ** (1.0 / 3.0)))
        while True:
            a = L / n
            g = (np.arange(n) + 0.5) * a
            sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
            rot = _random_rotations(rng, len(sites))
            mol = sites[:, None, :] + np.einsum("nij,kj->nki", rot, _water_local())
            dmin = np.full(len(mol), np.inf)
            for p in nps:  # only waters near a particle's bounding sphere need the full check
                c = p.mean(0)
                R = np.sqrt(((p - c) ** 2).sum(1)).max()
                d = sites - c
                d -= L * np.round(d / L)
                near = np.sqrt((d * d).sum(1)) < R + 0.3 + 2 * OH + 1e-6
                if near.any():
                    dn = _min_dist_to(mol[near].reshape(-1, 3), p, L).reshape(-1, 3).min(1)
                    dmin[near] = np.minimum(dmin[near], dn)
            ok = mol[dmin >= 0.3]
            if len(ok) >= w.n_waters:
                break
            n += 1
        keep = np.sort(rng.choice(len(ok), size=w.n_waters, replace=False))
        water = ok[keep]

    pos = np.concatenate([metal, water.reshape(-1, 3)])
    m = np.concatenate([np.full(len(metal), M_AU), np.tile([M_O, M_H, M_H], len(water))])
    vel = rng.normal(size=pos.shape) * np.sqrt(K_BOLTZ * w.temperature / m)[:, None]
    M = len(metal)
    nw = len(water)
    if nw:
        vw = vel[M:].reshape(nw, 3, 3)
        rw = water
        mw = np.array([M_O, M_H, M_H])
        cons = [(0, 1), (0, 2), (1, 2)]
        for _ in range(200):
            for (i, j) in cons:
                rij = rw[:, i] - rw[:, j]
                vij = vw[:, i] - vw[:, j]
                gij = -(rij * vij).sum(-1) / ((1 / mw[i] + 1 / mw[j]) * (rij * rij).sum(-1))
                vw[:, i] += (gij[:, None] * rij) / mw[i]
                vw[:, j] -= (gij[:, None] * rij) / mw[j]
        vel[M:] = vw.reshape(-1, 3)
    vel -= (vel * m[:, None]).sum(0) / m.sum()
    ndf = 3 * len(pos) - 3 - 3 * nw
    t_now = (m[:, None] * vel * vel).sum() / (K_BOLTZ * ndf)
    if t_now > 0:
        vel *= np.sqrt(w.temperature / t_now)
    return dict(pos=pos, vel=vel, n_metal=M, n_waters=nw,
                np_ranges=[(sum(len(x) for x in nps[:k]), sum(len(x) for x in nps[:k + 1]) - 1)
                           for k in range(len(nps))])


def param_text(n_metal: int, n_waters: int, np_ranges, use_cpff: int = 1, nonbonded=None) -> str:
    eps = 0.012793 * EV2KJMOL
    lines = ["SCALE_LJ_QQ    0.50000000     0.83333333", ""]
    mols = []
    if n_metal:
        mols.append(("gold", n_metal))
    if n_waters:
        mols.append(("SOL", n_waters))
    lines.append(f"MOLECULES      {len(mols)}")
    for nm, cnt in mols:
        lines.append(f"{nm}           {cnt}")
    lines.append("")
    for nm, _ in mols:
        if nm == "gold":
            lines += ["gold_ATOMS          1", f"     0.000000   {M_AU:.6f}       0", ""]
        else:
            lines += ["SOL_ATOMS           3", f"    {Q_O:.6f}    {M_O:.6f}       1",
                      f"     {Q_H:.6f}     {M_H:.6f}       2", f"     {Q_H:.6f}     {M_H:.6f}       2", ""]
    lines += ["NONBONDED      3         6"] + list(nonbonded or (
        " 1    0.00000000e+00      0.00000000e+00",
        " 4  0.002522219544  3.624859037184e-06  2.25",
        " 4  0.001028707002  1.45541995368e-06   2.25",
        " 1    2.48970844e-03      2.43509761e-06",
        " 1    0.00000000e+00      0.00000000e+00",
        " 1    0.00000000e+00      0.00000000e+00")) + [""]
    hh = 2.0 * OH * np.sin(np.deg2rad(HOH_DEG) / 2.0)
    for nm, _ in mols:
        for sec in ("BONDS", "PAIRS", "ANGLES", "DIHEDRALS", "VSITES"):
            lines.append(f"{nm}_{sec:<14s} 0")
        if nm == "SOL":
            lines += ["SOL_CSTRS           3", f"0 1   {OH:.6f}", f"0 2   {OH:.6f}", f"1 2   {hh:.6f}"]
        else:
            lines.append(f"{nm}_CSTRS          0")
        lines.append("")
    if n_metal:
        lines.append(f"MM_METAL  0  {n_metal - 1}")
    else:
        lines.append("MM_METAL  -1  -1")
    lines.append(f"QSC_METAL  10  8  {eps:.9f}  34.408000  0.408000")
    lines.append("CPFF_METAL  39.529700  1.215900   ;  Note: atomic unit")
    lines.append("")
    lines.append(f"NANOPARTICLES   {len(np_ranges)}")
    for (s, e) in np_ranges:
        lines.append(f"START_END_CHG   {s}  {e}   0.0")
    return "\n".join(lines) + "\n"


def mdset_text(w: Workload, steps: int | None = None) -> str:
    ex, ey, ez = w.efield_vnm
    return "\n".join([
        "run_type          md",
        f"ensemble          {w.ensemble}",
        "",
        "em_steps          100",
        "em_length_in_nm   0.0001",
        "em_tolerance      1000.0",
        "",
        f"number_of_steps   {w.steps if steps is None else steps}",
        f"time_step_in_ps   {w.dt}",
        f"save_step         {w.save_step}",
        "",
        "vdw_type          shifted",
        "coulomb_type      wolf_sum",
        "cut_off_radius    1.2",
        "coulomb_alpha     2.0",
        "",
        "heating_steps     0",
        f"ref_T_in_K        {w.temperature}",
        "tau_T_in_ps       0.1",
        "",
        "fix_metal         0",
        f"use_cpff          {w.use_cpff}",
        "",
        f"external_Ex       {ex}",
        f"external_Ey       {ey}",
        f"external_Ez       {ez}",
    ]) + "\n"


def gro_text(pos: np.ndarray, vel: np.ndarray, n_metal: int, box: float) -> str:
    """.gro with the reference's fixed columns; numbers at full precision.

    read_gro takes residue id/name and atom name from columns 0-14 and reads
    the numbers free-format from column 20 (file.c:168-190), so writing them
    with more decimals than write_gro (file.c:221) loses nothing and keeps both
    parsers on identical doubles.
    """
    out = ["step  0  vQ  0.000000  vP  0.000000", f"{len(pos):5d}"]
    names = ["OW", "HW1", "HW2"]
    for i in range(len(pos)):
        if i < n_metal:
            res, rn, an = i + 1, "AU", "Au"
        else:
            k = i - n_metal
            res, rn, an = n_metal + k // 3 + 1, "SOL", names[k % 3]
        x, y, z = pos[i]
        vx, vy, vz = vel[i]
        out.append(f"{res % 100000:5d}{rn:<5s}{an:>5s}{(i + 1) % 100000:5d}"
                   f" {x:.12f} {y:.12f} {z:.12f} {vx:.12f} {vy:.12f} {vz:.12f}")
    out.append(f"{box:10.5f}{box:10.5f}{box:10.5f}")
    return "\n".join(out) + "\n"


# ------------------------------------------------------------------------------
# A test system with every bonded term and a virtual site: Au13 (CPIM on),
# 5-atom chains (harmonic and Morse bonds, 1-4 pairs of
# both kinds, harmonic and Urey-Bradley angles, RB and periodic dihedrals of
# multiplicity 1 to 4), rigid 4-site waters whose charge site is a funct-4
# virtual site with an out-of-plane part, and flexible 3-site waters.

BONDED_BOX = 3.5
_CHAIN = dict(n=20, q=[0.2, -0.1, 0.0, -0.1, 0.0], m=12.011, t=3)
_T4P = dict(n=30, q=[0.0, 0.52, 0.52, -1.04], m=[16.0, 1.008, 1.008, 0.0], t=[1, 2, 2, 4])
_FLW = dict(n=10, q=[-0.82, 0.41, 0.41], m=[16.0, 1.008, 1.008], t=[1, 2, 2])
_VS = (0.128, 0.128, 1.5)


def _chain_local() -> np.ndarray:
    """Zig-zag chain, bonds 0.153 nm, angles 111 degrees, torsions +-60 degrees."""
    b, ang = 0.153, np.deg2rad(111.0)
    pts = [np.zeros(3), np.array([b, 0.0, 0.0])]
    pts.append(pts[1] + b * np.array([-np.cos(ang), np.sin(ang), 0.0]))
    for tors in (np.deg2rad(60.0), np.deg2rad(-65.0)):
        a, b_, c = pts[-3], pts[-2], pts[-1]
        bc = (c - b_) / np.linalg.norm(c - b_)
        n = np.cross(b_ - a, bc)
        n /= np.linalg.norm(n)
        m = np.cross(n, bc)
        d = np.array([-b * np.cos(ang), b * np.sin(ang) * np.cos(tors), b * np.sin(ang) * np.sin(tors)])
        pts.append(c + d[0] * bc + d[1] * m + d[2] * n)
    return np.array(pts)


def _t4p_local() -> np.ndarray:
    half = np.deg2rad(104.52) / 2.0
    oh = 0.09572
    o, h1, h2 = np.zeros(3), np.array([oh * np.sin(half), 0.0, oh * np.cos(half)]), \
        np.array([-oh * np.sin(half), 0.0, oh * np.cos(half)])
    a, b, c = _VS
    s = o + a * (h1 - o) + b * (h2 - o) + c * np.cross(h1 - o, h2 - o)
    return np.array([o, h1, h2, s])


def _flw_local() -> np.ndarray:
    half = np.deg2rad(107.0) / 2.0
    return np.array([[0.0, 0.0, 0.0], [0.101 * np.sin(half), 0.0, 0.101 * np.cos(half)],
                     [-0.099 * np.sin(half), 0.0, 0.099 * np.cos(half)]])


def build_bonded(seed: int = 11):
    rng = np.random.default_rng(seed)
    L = BONDED_BOX
    metal = icosahedron(1) + L / 2
    placed = [metal]
    mols = []
    for spec, local in ((_CHAIN, _chain_local()), (_T4P, _t4p_local()), (_FLW, _flw_local())):
        for _ in range(spec["n"]):
            for _attempt in range(10000):
                rot = _random_rotations(rng, 1)[0]
                x = (local - local.mean(0)) @ rot.T + rng.uniform(0.0, L, 3)
                allp = np.concatenate(placed)
                if _min_dist_to(x, allp, L).min() > 0.28:
                    break
            placed.append(x)
            mols.append(x)
    pos = np.concatenate(placed)
    masses = np.concatenate([np.full(13, M_AU), np.full(_CHAIN["n"] * 5, _CHAIN["m"]),
                             np.tile(_T4P["m"], _T4P["n"]), np.tile(_FLW["m"], _FLW["n"])])
    vel = rng.normal(size=pos.shape) * np.sqrt(K_BOLTZ * 300.0 / np.where(masses > 0, masses, 1.0))[:, None]
    vel[masses == 0] = 0.0
    # rigid 4-site waters: remove the velocity components along their constraints
    s0 = 13 + _CHAIN["n"] * 5
    mw = np.array(_T4P["m"][:3])
    for k in range(_T4P["n"]):
        r = pos[s0 + 4 * k:s0 + 4 * k + 3]
        v = vel[s0 + 4 * k:s0 + 4 * k + 3]
        for _ in range(200):
            for (i, j) in ((0, 1), (0, 2), (1, 2)):
                rij, vij = r[i] - r[j], v[i] - v[j]
                g = -(rij @ vij) / ((1 / mw[i] + 1 / mw[j]) * (rij @ rij))
                v[i] += g * rij / mw[i]
                v[j] -= g * rij / mw[j]
    real = masses > 0
    vel[real] -= (vel[real] * masses[real, None]).sum(0) / masses[real].sum()
    return pos, vel


def bonded_param_text() -> str:
    eps = 0.012793 * EV2KJMOL
    hh = 0.15139
    L = ["SCALE_LJ_QQ    0.50000000     0.83333333", "", "MOLECULES      4",
         "gold           13", f"CHN            {_CHAIN['n']}", f"T4P            {_T4P['n']}",
         f"FLW            {_FLW['n']}", "",
         "gold_ATOMS          1", f"     0.000000   {M_AU:.6f}       0", "",
         "CHN_ATOMS           5"]
    L += [f"    {q:.6f}    {_CHAIN['m']:.6f}       {_CHAIN['t']}" for q in _CHAIN["q"]]
    L += ["", "T4P_ATOMS           4"]
    L += [f"    {q:.6f}    {m:.6f}       {t}" for q, m, t in zip(_T4P["q"], _T4P["m"], _T4P["t"])]
    L += ["", "FLW_ATOMS           3"]
    L += [f"    {q:.6f}    {m:.6f}       {t}" for q, m, t in zip(_FLW["q"], _FLW["m"], _FLW["t"])]
    L += ["", "NONBONDED      5         15",
          " 1    0.00000000e+00      0.00000000e+00",   # Au Au
          " 4  0.002522219544  3.624859037184e-06  2.25",  # Au O
          " 4  0.001028707002  1.45541995368e-06   2.25",  # Au H
          " 1    3.00000000e-03      5.00000000e-06",   # Au C
          " 1    0.00000000e+00      0.00000000e+00",   # Au M
          " 1    2.48970844e-03      2.43509761e-06",   # O O
          " 1    0.00000000e+00      0.00000000e+00",   # O H
          " 1    2.00000000e-03      3.00000000e-06",   # O C
          " 1    0.00000000e+00      0.00000000e+00",   # O M
          " 1    0.00000000e+00      0.00000000e+00",   # H H
          " 1    5.00000000e-04      5.00000000e-07",   # H C
          " 1    0.00000000e+00      0.00000000e+00",   # H M
          " 1    4.00000000e-03      8.00000000e-06",   # C C
          " 1    0.00000000e+00      0.00000000e+00",   # C M
          " 1    0.00000000e+00      0.00000000e+00",   # M M
          ""]
    L += ["gold_BONDS          0", "gold_PAIRS          0", "gold_ANGLES         0", "gold_DIHEDRALS      0",
          "gold_VSITES         0", "gold_CSTRS          0", ""]
    # no funct-5 (exclusion-only) bond: the reference leaves its BondParam
    # unset and mpi_bonded still applies it (undefined behaviour)
    L += ["CHN_BONDS           3",
          "0 1 1   0.153  250000.0",
          "1 2 3   0.153  350.0  20.0",
          "2 3 1   0.153  250000.0",
          "CHN_PAIRS           2",
          "0 3 1",
          "1 4 2   0.5  0.1  -0.1  3.0e-01  4.0e-01",
          "CHN_ANGLES          3",
          "0 1 2 1   111.0  400.0",
          "1 2 3 5   112.0  450.0  0.25  5000.0",
          "2 3 4 1   110.0  420.0",
          "CHN_DIHEDRALS       5",
          "0 1 2 3 3   9.28  12.16  -13.12  -3.06  26.24  -31.5",
          "1 2 3 4 9   0.0  5.92  3",
          "1 2 3 4 1   180.0  2.0  1",
          "0 1 2 3 4   0.0  1.0  2",
          "0 1 2 3 9   180.0  0.5  4",
          "CHN_VSITES          0",
          "CHN_CSTRS           0", ""]
    a, b, c = _VS
    L += ["T4P_BONDS           0", "T4P_PAIRS           0", "T4P_ANGLES          0", "T4P_DIHEDRALS       0",
          "T4P_VSITES          1", f"0 1 2 3 4   {a}  {b}  {c}",
          "T4P_CSTRS           3", "0 1   0.09572", "0 2   0.09572", f"1 2   {hh}", ""]
    L += ["FLW_BONDS           2", "0 1 1   0.1  345000.0", "0 2 1   0.1  345000.0",
          "FLW_PAIRS           0", "FLW_ANGLES          1", "1 0 2 5   109.47  383.0  0.1633  2000.0",
          "FLW_DIHEDRALS       0", "FLW_VSITES          0", "FLW_CSTRS           0", ""]
    L += ["MM_METAL  0  12", f"QSC_METAL  10  8  {eps:.9f}  34.408000  0.408000",
          "CPFF_METAL  39.529700  1.215900   ;  Note: atomic unit", "", "NANOPARTICLES   1",
          "START_END_CHG   0  12   0.0"]
    return "\n".join(L) + "\n"


def bonded_gro_text(pos: np.ndarray, vel: np.ndarray) -> str:
    out = ["step  0  vQ  0.000000  vP  0.000000", f"{len(pos):5d}"]
    rows = [(k + 1, "AU", "Au") for k in range(13)]
    res = 14
    for _ in range(_CHAIN["n"]):
        rows += [(res, "CHN", f"C{a + 1}") for a in range(5)]
        res += 1
    for _ in range(_T4P["n"]):
        rows += [(res, "T4P", n) for n in ("OW", "HW1", "HW2", "MW")]
        res += 1
    for _ in range(_FLW["n"]):
        rows += [(res, "FLW", n) for n in ("OW", "HW1", "HW2")]
        res += 1
    for i, ((r, rn, an), x, v) in enumerate(zip(rows, pos, vel)):
        out.append(f"{r % 100000:5d}{rn:<5s}{an:>5s}{(i + 1) % 100000:5d}"
                   f" {x[0]:.12f} {x[1]:.12f} {x[2]:.12f} {v[0]:.12f} {v[1]:.12f} {v[2]:.12f}")
    out.append(f"{BONDED_BOX:10.5f}{BONDED_BOX:10.5f}{BONDED_BOX:10.5f}")
    return "\n".join(out) + "\n"


def write_bonded(out_dir: str, steps: int | None = None) -> dict:
    os.makedirs(out_dir, exist_ok=True)
    pos, vel = build_bonded()
    w = Workload("t_bonded", [1], 0, BONDED_BOX, seed=11, ensemble="nvt", steps=steps or 20)
    paths = {k: os.path.join(out_dir, f) for k, f in
             (("gro", "init.gro"), ("par", "param.txt"), ("mds", "mdset.txt"))}
    with open(paths["gro"], "w") as f:
        f.write(bonded_gro_text(pos, vel))
    with open(paths["par"], "w") as f:
        f.write(bonded_param_text())
    with open(paths["mds"], "w") as f:
        f.write(mdset_text(w, steps))
    paths["n_atoms"] = len(pos)
    paths["n_metal"] = 13
    return paths


def write(name: str, out_dir: str, steps: int | None = None) -> dict:
    """Write one workload's three input files; returns their paths."""
    if name == "t_bonded":
        return write_bonded(out_dir, steps)
    w = WORKLOADS[name]
    os.makedirs(out_dir, exist_ok=True)
    s = build(w)
    paths = {k: os.path.join(out_dir, f) for k, f in
             (("gro", "init.gro"), ("par", "param.txt"), ("mds", "mdset.txt"))}
    with open(paths["gro"], "w") as f:
        f.write(gro_text(s["pos"], s["vel"], s["n_metal"], w.box))
    with open(paths["par"], "w") as f:
        f.write(param_text(s["n_metal"], s["n_waters"], s["np_ranges"], w.use_cpff, w.nonbonded))
    with open(paths["mds"], "w") as f:
        f.write(mdset_text(w, steps))
    paths["n_atoms"] = len(s["pos"])
    paths["n_metal"] = s["n_metal"]
    return paths


def cached(name: str, root: str | None = None, steps: int | None = None) -> dict:
    """Write a workload under a cache folder once and reuse it afterwards."""
    root = root or os.environ.get("CAPAC_CONFIG_DIR") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "build", "configs")
    d = os.path.join(root, name if steps is None else f"{name}_s{steps}")
    paths = {k: os.path.join(d, f) for k, f in
             (("gro", "init.gro"), ("par", "param.txt"), ("mds", "mdset.txt"))}
    if not all(os.path.exists(p) for p in paths.values()):
        return write(name, d, steps)
    return paths

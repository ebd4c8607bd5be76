"""Atomic data in the layout the reference's loader produces.

`AtomSpec` holds the raw per-element data of an old-style atomic data file
(ions with ionisation energies and ground levels, levels with ion stage,
statistical weight and excitation energy, level-to-level lines with
Einstein A) plus a fuzz line list (nu, gf, El, ion).  `AtomicModel.to_struct`
applies the loader's own post-processing (AtomicData::read_atomic_data_oldstyle,
src/opacity/AtomicData.cpp:459-760; read_fuzzfile_data_for_atom :783-868):
E_ion = chi - E, g = 0 -> 1, ic = ground level of the next stage, line
frequency and oscillator strength, hydrogenic photoionisation tables, and
the fuzz-line selection nu_min < nu < nu_max, ion < n_ions.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import abi
from .grids import LocGrid, PI

EV_TO_ERGS = 1.60217646e-12
H = 6.6260755e-27
C_LIGHT = 2.99792458e10
SIGMA_TOT = 0.0265400193567
CM_TO_ANGS = 1.0e8
ANGS_TO_CM = 1.0e-8


@dataclass
class AtomSpec:
    Z: int
    ion_chi: np.ndarray          # [n_ions] eV (last entry: fully ionised stage)
    ion_ground: np.ndarray       # [n_ions] first level of each stage
    lev_ion: np.ndarray          # [n_levels]
    lev_g: np.ndarray
    lev_E: np.ndarray            # eV
    line_l: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    line_u: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    line_A: np.ndarray = field(default_factory=lambda: np.zeros(0))
    fuzz_nu: np.ndarray = field(default_factory=lambda: np.zeros(0))
    fuzz_gf: np.ndarray = field(default_factory=lambda: np.zeros(0))
    fuzz_El: np.ndarray = field(default_factory=lambda: np.zeros(0))
    fuzz_ion: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))

    @property
    def n_ions(self) -> int:
        return int(self.ion_chi.size)


def _photo_table(E_ion: float, ion: int, chi_ground: float):
    """hydrogenic photoionisation cross-section table (AtomicData.cpp:713-756),
    on xy_array::init(start, stop, delta) abscissae (xy_array.cpp:25-35)"""
    npts, fmax = 100, 10
    E_max = E_ion * fmax
    dE = (E_max - E_ion) / npts
    n = int((E_max - E_ion) / dE) + 1
    delta = dE
    if n <= 1:
        n = 1
        delta = E_max - E_ion
    if delta < 0:
        delta = 0.0
    x = np.array([E_ion + i * delta for i in range(n)], dtype=np.float64)
    y = np.zeros(n)
    n_eff = (1 - (chi_ground - E_ion) / chi_ground) ** -0.5
    s_fac = n_eff / (ion + 1) / (ion + 1)
    for j in range(min(npts, n)):
        y[j] = 6.3e-18 * s_fac * (x[j] / E_ion) ** -3.0
    return x, y


@dataclass
class AtomicModel:
    atoms: list

    def n_fuzz(self) -> int:
        return int(sum(a.fuzz_nu.size for a in self.atoms))

    def selected_fuzz(self, a: AtomSpec, nu_grid: LocGrid):
        keep = (a.fuzz_ion < a.n_ions) & (a.fuzz_nu > nu_grid.min) & (a.fuzz_nu < nu_grid.right[-1])
        return keep

    def to_struct(self, keep: abi.Keep, nu_grid: LocGrid) -> abi.AtomicData:
        ion_off, lev_off, line_off, fuzz_off, photo_off = [0], [0], [0], [0], [0]
        ion_chi, lev_ion, lev_g, lev_ic, lev_E, lev_Eion = [], [], [], [], [], []
        photo_E, photo_s = [], []
        line_l, line_u, line_nu, line_f = [], [], [], []
        fnu, fgf, fEl, fion = [], [], [], []
        for a in self.atoms:
            ion_chi.extend(a.ion_chi.tolist())
            nl = a.lev_ion.size
            for i in range(nl):
                ion = int(a.lev_ion[i])
                g = int(a.lev_g[i]) or 1
                E = float(a.lev_E[i])
                E_ion = float(a.ion_chi[ion]) - E
                ic = -1
                for j in range(a.n_ions):   # stage j == index j
                    if j == ion + 1:
                        ic = int(a.ion_ground[j])
                lev_ion.append(ion); lev_g.append(g); lev_ic.append(ic)
                lev_E.append(E); lev_Eion.append(E_ion)
                x, y = _photo_table(E_ion, ion, float(a.ion_chi[ion]))
                photo_E.extend(x.tolist()); photo_s.extend(y.tolist())
                photo_off.append(photo_off[-1] + x.size)
            for k in range(a.line_l.size):
                ll, lu = int(a.line_l[k]), int(a.line_u[k])
                dE = float(a.lev_E[lu]) - float(a.lev_E[ll])
                if dE == 0:
                    raise ValueError("zero-energy line in synthetic data")
                nu = dE * EV_TO_ERGS / H
                lam = C_LIGHT / nu * CM_TO_ANGS
                gl = int(a.lev_g[ll]) or 1
                gu = int(a.lev_g[lu]) or 1
                lam_cm = lam * ANGS_TO_CM
                f = lam_cm * lam_cm * float(a.line_A[k]) * gu / gl / (8 * PI * SIGMA_TOT)
                line_l.append(ll); line_u.append(lu); line_nu.append(nu); line_f.append(f)
            sel = self.selected_fuzz(a, nu_grid)
            fnu.extend(a.fuzz_nu[sel].tolist()); fgf.extend(a.fuzz_gf[sel].tolist())
            fEl.extend(a.fuzz_El[sel].tolist()); fion.extend(a.fuzz_ion[sel].tolist())
            ion_off.append(len(ion_chi)); lev_off.append(len(lev_ion))
            line_off.append(len(line_l)); fuzz_off.append(len(fnu))
        s = abi.AtomicData()
        s.n_atoms = len(self.atoms)
        s.ion_off = keep.i(ion_off); s.ion_chi = keep.d(ion_chi)
        s.lev_off = keep.i(lev_off); s.lev_ion = keep.i(lev_ion); s.lev_g = keep.i(lev_g)
        s.lev_ic = keep.i(lev_ic); s.lev_E = keep.d(lev_E); s.lev_Eion = keep.d(lev_Eion)
        s.photo_off = keep.i(photo_off); s.photo_E = keep.d(photo_E); s.photo_s = keep.d(photo_s)
        s.line_off = keep.i(line_off); s.line_l = keep.i(line_l); s.line_u = keep.i(line_u)
        s.line_nu = keep.d(line_nu); s.line_f = keep.d(line_f)
        s.fuzz_off = keep.i(fuzz_off); s.fuzz_nu = keep.d(fnu); s.fuzz_gf = keep.d(fgf)
        s.fuzz_El = keep.d(fEl); s.fuzz_ion = keep.i(fion)
        return s


# approximate first five ionisation energies (eV) of the ejecta elements
_CHI = {
    6: [11.26, 24.38, 47.89, 64.49, 392.1],
    8: [13.62, 35.12, 54.94, 77.41, 113.9],
    14: [8.15, 16.35, 33.49, 45.14, 166.8],
    16: [10.36, 23.34, 34.79, 47.22, 72.59],
    20: [6.11, 11.87, 50.91, 67.27, 84.5],
    26: [7.90, 16.19, 30.65, 54.8, 75.0],
    27: [7.88, 17.08, 33.50, 51.3, 79.5],
    28: [7.64, 18.17, 35.19, 54.9, 76.06],
}


def synthetic_atoms(elements, n_levels_per_ion: int, n_lines_per_ion: int,
                    rng: np.random.Generator, E_max_eV: Optional[float] = None) -> AtomicModel:
    """Seeded synthetic ion/level model: five real stages per element (the
    ionisation energies above) plus the bare stage, `n_levels_per_ion`
    levels per stage with E in [0, 0.8 chi) (ground level at 0; the bound is
    min(0.8 chi, E_max_eV) when E_max_eV is given) and odd g, and optional
    level-to-level lines with A log-uniform in 1e4..1e8 s^-1."""
    atoms = []
    for Z in elements:
        chi = list(_CHI[Z]) + [99999.0]
        lev_ion, lev_g, lev_E, ground = [], [], [], []
        for s in range(len(chi)):
            ground.append(len(lev_ion))
            nl = 1 if s == len(chi) - 1 else n_levels_per_ion
            top = 0.8 * chi[s] if E_max_eV is None else min(0.8 * chi[s], E_max_eV)
            Es = np.sort(rng.uniform(0.0, top, nl - 1)) if nl > 1 else np.zeros(0)
            Es = np.concatenate([[0.0], Es])
            gs = 2 * rng.integers(0, 5, nl) + 1
            if s == len(chi) - 1:
                gs[:] = 1
            lev_ion.extend([s] * nl); lev_g.extend(gs.tolist()); lev_E.extend(Es.tolist())
        ll, lu, A = [], [], []
        for s in range(len(chi) - 1):
            base = ground[s]
            for _ in range(n_lines_per_ion):
                a, b = sorted(rng.choice(n_levels_per_ion, 2, replace=False))
                ll.append(base + a); lu.append(base + b)
                A.append(10 ** rng.uniform(4, 8))
        atoms.append(AtomSpec(Z=Z, ion_chi=np.array(chi), ion_ground=np.array(ground, np.int32),
                              lev_ion=np.array(lev_ion, np.int32), lev_g=np.array(lev_g, np.int32),
                              lev_E=np.array(lev_E), line_l=np.array(ll, np.int32),
                              line_u=np.array(lu, np.int32), line_A=np.array(A)))
    return AtomicModel(atoms)


def add_level_lines(model: AtomicModel, n_lines: int, nu_min: float, nu_max: float,
                    rng: np.random.Generator, A_min: float = 1e4, A_max: float = 1e8) -> AtomicModel:
    """Synthetic level-to-level line list for the Sobolev line-expansion
    opacity: each line's (element, ion stage) uniform over the real stages
    of the elements present, its lower/upper level a uniform pair of distinct
    levels of that stage whose transition frequency lies strictly inside
    (nu_min, nu_max) (pairs outside are redrawn), Einstein A log-uniform in
    [A_min, A_max].  Exactly n_lines lines; each atom keeps its lines in
    draw order."""
    species = [(ai, s) for ai, a in enumerate(model.atoms) for s in range(a.n_ions - 1)]
    out = {ai: ([], [], []) for ai in range(len(model.atoms))}
    made = 0
    while made < n_lines:
        m = 2 * (n_lines - made) + 64
        pick = rng.integers(0, len(species), m)
        r1 = rng.random(m)
        r2 = rng.random(m)
        lgA = rng.uniform(np.log10(A_min), np.log10(A_max), m)
        for k in range(m):
            if made == n_lines:
                break
            ai, s = species[pick[k]]
            a = model.atoms[ai]
            g0 = int(a.ion_ground[s])
            nlev = int(a.ion_ground[s + 1]) - g0
            l = g0 + int(r1[k] * nlev)
            u = g0 + int(r2[k] * nlev)
            if l == u:
                continue
            if a.lev_E[l] > a.lev_E[u]:
                l, u = u, l
            nu = (float(a.lev_E[u]) - float(a.lev_E[l])) * EV_TO_ERGS / H
            if not (nu_min < nu < nu_max):
                continue
            out[ai][0].append(l)
            out[ai][1].append(u)
            out[ai][2].append(10.0 ** lgA[k])
            made += 1
    for ai, a in enumerate(model.atoms):
        ll, lu, A = out[ai]
        a.line_l = np.array(ll, np.int32)
        a.line_u = np.array(lu, np.int32)
        a.line_A = np.array(A, np.float64)
    return model


def add_fuzz_lines(model: AtomicModel, n_lines: int, lam_min_A: float, lam_max_A: float,
                   gf_min: float, gf_max: float, El_max: float, rng: np.random.Generator):
    """Synthetic fuzz line list: wavelength log-uniform in [lam_min, lam_max] A,
    gf log-uniform in [gf_min, gf_max], lower-level energy uniform in
    [0, El_max] eV; each line's (element, ion stage) drawn uniformly among
    the real (non-bare) stages of the elements present."""
    lam = 10 ** rng.uniform(np.log10(lam_min_A), np.log10(lam_max_A), n_lines)
    nu = C_LIGHT / (lam * ANGS_TO_CM)
    gf = 10 ** rng.uniform(np.log10(gf_min), np.log10(gf_max), n_lines)
    El = rng.uniform(0.0, El_max, n_lines)
    species = [(ai, s) for ai, a in enumerate(model.atoms) for s in range(a.n_ions - 1)]
    pick = rng.integers(0, len(species), n_lines)
    for ai, a in enumerate(model.atoms):
        idx = [k for k, (aa, s) in enumerate(species) if aa == ai]
        m = np.isin(pick, idx)
        a.fuzz_nu = nu[m]
        a.fuzz_gf = gf[m]
        a.fuzz_El = El[m]
        a.fuzz_ion = np.array([species[p][1] for p in pick[m]], dtype=np.int32)
    return model

"""Text outputs in the reference's formats, written from the arrays the C ABI
returns, so files read by the reference's own scripts (np.loadtxt of
spectrum_<it>.dat and plt_<iw>.dat) come out byte for byte as the reference
writes them for the same values.

  write_spectrum_dat   spectrum_array::print, text part
                       (src/transport/spectrum_array.cpp:253-310)
  write_plotfile_1d    grid_1D_sphere::write_plotfile, text part
                       (src/grid/grid_1D_sphere.cpp:598-633)

The reference also writes HDF5 versions of both; there is no HDF5 library in
this build, so those are not written.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from .grids import LocGrid

A_RAD = 7.5657e-15  # physical_constants::a


def spectrum_unitized(flux: np.ndarray, click: np.ndarray, t_grid: LocGrid, nu_grid: LocGrid, mu_grid: LocGrid,
                      phi_grid: LocGrid, n_procs: int = 1):
    """flux per unit frequency (and time) and per angle bin, and clicks times
    the number of ranks, as spectrum_array::print forms them (:268-284)."""
    nt, nw, nm, npf = t_grid.n, nu_grid.n, mu_grid.n, phi_grid.n
    d = np.empty(flux.size)
    cb = np.empty(flux.size)
    for k in range(nm):
        for m in range(npf):
            for i in range(nt):
                for j in range(nw):
                    idx = ((i * nw + j) * nm + k) * npf + m
                    norm = 1.0 / (nm * npf)
                    if nw > 1:
                        norm *= nu_grid.delta_at(j)
                    if nt > 1:
                        norm *= t_grid.delta_at(i)
                    d[idx] = flux[idx] / norm
                    cb[idx] = click[idx] * n_procs
    return d, cb


def write_spectrum_dat(name: str, flux: np.ndarray, click: np.ndarray, t_grid: LocGrid, nu_grid: LocGrid,
                       mu_grid: LocGrid, phi_grid: LocGrid, n_procs: int = 1) -> str:
    """Writes `<name>.dat` as spectrum_array::print does; returns the path."""
    nt, nw, nm, npf = t_grid.n, nu_grid.n, mu_grid.n, phi_grid.n
    d, cb = spectrum_unitized(flux, click, t_grid, nu_grid, mu_grid, phi_grid, n_procs)
    lines = ["# %d %d %d %d\n" % (nt, nw, nm, npf)]
    for k in range(nm):
        for m in range(npf):
            for i in range(nt):
                for j in range(nw):
                    idx = ((i * nw + j) * nm + k) * npf + m
                    s = ""
                    if nt > 1:
                        s += "%12.4e " % t_grid.center_at(i)
                    if nw > 1:
                        s += "%12.4e " % nu_grid.center_at(j)
                    if nm > 1:
                        s += "%12.4f " % mu_grid.center_at(k)
                    if npf > 1:
                        s += "%12.4f " % phi_grid.center_at(m)
                    s += "%12.5e %12.5e\n" % (d[idx], cb[idx])
                    lines.append(s)
    path = name + ".dat"
    with open(path, "w") as f:
        f.write("".join(lines))
    return path


def write_plotfile_1d(path: str, t: float, r_min: float, r_out: np.ndarray, rho: np.ndarray, v: np.ndarray,
                      T_gas: np.ndarray, e_rad: np.ndarray, n_elec: np.ndarray,
                      L_dep: Optional[np.ndarray] = None, L_emit: Optional[np.ndarray] = None,
                      X: Optional[np.ndarray] = None, elems: Optional[Sequence[tuple]] = None) -> str:
    """Writes the text plot file of a 1D sphere (plt_%05d.dat) as
    grid_1D_sphere::write_plotfile does; X / elems add the mass fractions
    (write_mass_fracs).  T_rad = (e_rad / a)^(1/4)."""
    n = r_out.size
    L_dep = np.zeros(n) if L_dep is None else L_dep
    L_emit = np.zeros(n) if L_emit is None else L_emit
    out = ["# t = %8.4e ; rmin = %8.4e\n" % (t, r_min)]
    h = "#  %-12.12s %-15.15s %-15.15s %-15.15s %-15.15s %-15.15s %-15.15s %-15.15s" % (
        "r", "rho", "v", "T_gas", "T_rad", "n_elec", "L_dep_nuc", "L_emit_nuc")
    if X is not None:
        for z, a in elems:
            h += " %-15.15s" % ("%d.%d" % (z, a))
    out.append(h + "\n")
    for i in range(n):
        T_rad = (e_rad[i] / A_RAD) ** 0.25
        s = "%12.8e  %12.8e  %12.8e  %12.8e  %12.8e  %12.8e  %12.8e  %12.8e" % (
            r_out[i], rho[i], v[i], T_gas[i], T_rad, n_elec[i], L_dep[i], L_emit[i])
        if X is not None:
            for k in range(X.shape[1]):
                s += "  %12.8e" % X[i, k]
        out.append(s + "\n")
    with open(path, "w") as f:
        f.write("".join(out))
    return path


def plotfile_name(iw: int) -> str:
    return "plt_%05d.dat" % iw

"""Host-side mirror of the reference's `transport` class
(src/transport/transport.h:45-320) for the hot path: a `Transport` owns one
context of the CUDA library and runs `step(dt)` as transport::step does
(src/transport/transport.cpp:26-140): opacity build, emission, propagation,
tally normalisation, then the radiative-equilibrium temperature solve when
the parameters ask for it.  `output_spectrum(it)` and `write_plotfile(iw)`
write the reference's text outputs; `run_steady` iterates like the
reference's driver does for steady-state runs
(src/main/SedonaClass.cpp:349-390).
"""
from __future__ import annotations

import os
from typing import Optional

import numpy as np

from . import abi, output
from .engine import Engine


class Transport:
    def __init__(self, workload, precision: int = abi.PREC_FP64, device: int = 0):
        self.w = workload
        self.P = workload.P
        self.eng = Engine(workload, precision=precision, device=device)
        self.radiative_eq = self.P.scalar("transport_radiative_equilibrium", int)
        self.steady_state = int(self.P.scalar("transport_steady_iterate", int) > 0)
        self.fix_Tgas = self.P.scalar("transport_fix_Tgas_during_transport", int)
        self.solve_Tgas_updated = self.P.scalar("transport_solve_Tgas_with_updated_opacities", int)
        self.set_Tgas_to_Trad = self.P.scalar("transport_set_Tgas_to_Trad", int)
        self.tallies = None
        self.n_unsolved = 0
        self.last_stats = None

    def step(self, dt: float = 1.0) -> dict:
        """transport::step: the zone state of the workload is copied in, the
        step runs on the device, tallies come back, and with radiative
        equilibrium the new gas temperatures replace the workload's."""
        if self.steady_state:
            dt = 1.0
        self.eng.upload_grid()
        st = self.eng.step(dt)
        if self.radiative_eq and not self.fix_Tgas and not self.solve_Tgas_updated:
            T, self.n_unsolved = self.eng.solve_temperature(self.set_Tgas_to_Trad)
            self.w.zones.T = T
        self.tallies = self.eng.tallies()
        self.last_stats = st
        return st

    def n_particles(self) -> int:
        return 0  # every packet of a step finishes within the step (steady state or escape/absorption)

    def output_spectrum(self, it: int, outdir: str = ".") -> Optional[str]:
        """transport::output_spectrum(it) (src/transport/transport_output.cpp:
        17-60): spectrum_name + "_" + it (or "_final" for it < 0), text part."""
        name = self.P.get("spectrum_name")
        if not name or self.P.scalar("spectrum_suppress_txt", int):
            return None
        base = "_final" if it < 0 else "_%d" % it
        flux, click = self.eng.spectrum()
        tg, ng, mg, pg = self.w.spectrum_grids()
        return output.write_spectrum_dat(os.path.join(outdir, name + base), flux, click, tg, ng, mg, pg)

    def write_plotfile(self, iw: int, t: float, outdir: str = ".") -> str:
        """grid_1D_sphere::write_plotfile(iw, t) (src/grid/grid_1D_sphere.cpp:
        598-633), text part, from the last step's tallies."""
        z = self.w.zones
        if z.type != abi.GRID_1D_SPHERE:
            raise ValueError("the text plot file is written for 1D spheres")
        n_elec = self.eng.opacity()["n_elec"]
        fr = bool(self.P.scalar("output_write_mass_fractions", int))
        elems = list(zip(z.elem_Z.tolist(), z.elem_A.tolist()))
        v = z.v if z.v is not None else np.zeros(z.n_zones)
        return output.write_plotfile_1d(os.path.join(outdir, output.plotfile_name(iw)), t, z.r_min, z.r_out, z.rho,
                                        v, z.T, self.tallies["e_rad"], n_elec,
                                        X=z.X if fr else None, elems=elems if fr else None)

    def close(self):
        self.eng.close()


def run_steady(workload, outdir: str = ".", precision: int = abi.PREC_FP64, device: int = 0) -> Transport:
    """Steady-state iterations as the reference's driver runs them
    (SedonaClass::evolve_system with transport_steady_iterate = n): each
    iteration steps the transport and writes spectrum_<it>.dat and
    plt_<it>.dat at the grid time."""
    n_iter = max(1, workload.P.scalar("transport_steady_iterate", int))
    tr = Transport(workload, precision=precision, device=device)
    for it in range(1, n_iter + 1):
        tr.step(1.0)
        tr.output_spectrum(it, outdir)
        tr.write_plotfile(it, workload.zones.t_now, outdir)
    return tr

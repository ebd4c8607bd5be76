"""Host-side mirror of the reference's `transport` class
(src/transport/transport.h:45-320) for the hot path: a `Transport` owns one
context of the CUDA library and runs `step(dt)` as transport::step does
(src/transport/transport.cpp:26-140): opacity build, emission, propagation,
tally normalisation, then the radiative-equilibrium temperature solve when
the parameters ask for it.  With particles_n_emit_radioactive > 0 the step
also emits and transports the decay packets and keeps L_radio_emit /
L_radio_dep and the gamma-ray spectrum.  `output_spectrum(it)` and
`write_plotfile(iw)` write the reference's text outputs; `run_steady` iterates like the
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
        self.n_radio = self.P.scalar("particles_n_emit_radioactive", int)
        self.tallies = None
        self.radio = None
        self.n_unsolved = 0
        self.last_stats = None
        # transport::init ends with initialize_particles (transport_init.cpp:376-379)
        n_init = int(self.P.scalar("particles_n_initialize", int))
        if n_init > 0:
            from .workloads import initial_e_rad
            self.eng.initialize_particles(n_init, initial_e_rad(workload.zones))

    def emission_counts(self, dt: float, last_iteration: bool) -> tuple:
        """Packet counts of a step: emit_radioactive scales its count by
        dt / tstep_max_dt when multiply_particles_n_emit_by_dt_over_dtmax is
        set (an int times a double, truncated: emission.cpp:170-173), and on
        the last iteration both it and emit_inner_source multiply theirs by
        particles_last_iter_pump when that is not 0 (:180-184, :377-382)."""
        n_core = int(self.P.scalar("core_n_emit", int))
        n_radio = int(self.n_radio)
        if n_radio and self.P.scalar("multiply_particles_n_emit_by_dt_over_dtmax", int):
            n_radio = int(n_radio * (dt / self.P.scalar("tstep_max_dt")))
        if last_iteration:
            pump = self.P.scalar("particles_last_iter_pump", int)
            if pump != 0:
                n_core *= pump
                n_radio *= pump
        return n_core, n_radio

    def step(self, dt: float = 1.0, last_iteration: bool = False) -> dict:
        """transport::step: the zone state of the workload is copied in, the
        step runs on the device, tallies come back, and with radiative
        equilibrium the new gas temperatures replace the workload's."""
        if self.steady_state:
            dt = 1.0
        n_core, n_radio = self.emission_counts(dt, last_iteration)
        if (n_core, n_radio) != (int(self.eng.tp.core_n_emit), int(self.eng.tp.n_emit_radioactive)):
            self.eng.set_emission(n_core, n_radio)
        # emit_inner_source takes core_luminosity at the transport clock when
        # it is not 0 (emission.cpp:386-388)
        L_now = self.P.function("core_luminosity", self.eng.time())
        if L_now != 0 and L_now != self.eng.tp.core_luminosity:
            self.eng.set_core_luminosity(L_now)
        self.eng.upload_grid()
        st = self.eng.step(dt)
        if self.radiative_eq and not self.fix_Tgas and not self.solve_Tgas_updated:
            T, self.n_unsolved = self.eng.solve_temperature(self.set_Tgas_to_Trad)
            self.w.zones.T = T
        self.tallies = self.eng.tallies()
        self.radio = self.eng.radioactive() if n_radio > 0 else None
        self.last_stats = st
        return st

    def n_particles(self) -> int:
        """transport::n_particles: packets carried to the next step."""
        return self.eng.n_particles()

    def output_spectrum(self, it: int, outdir: str = ".") -> Optional[str]:
        """transport::output_spectrum(it) (src/transport/transport_output.cpp:
        17-60): spectrum_name + "_" + it (or "_final" for it < 0), text part;
        with gamma_name set, the gamma-ray spectrum too (on the same grids,
        as the reference builds it).  Returns the optical spectrum's path."""
        if self.P.scalar("spectrum_suppress_txt", int):
            return None
        base = "_final" if it < 0 else "_%d" % it
        tg, ng, mg, pg = self.w.spectrum_grids()
        gname = self.P.get("gamma_name")
        if gname and self.radio is not None:
            output.write_spectrum_dat(os.path.join(outdir, gname + base), self.radio["gamma_flux"],
                                      self.radio["gamma_click"], tg, ng, mg, pg)
        name = self.P.get("spectrum_name")
        if not name:
            return None
        flux, click = self.eng.spectrum()
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
        R = self.radio or {}
        return output.write_plotfile_1d(os.path.join(outdir, output.plotfile_name(iw)), t, z.r_min, z.r_out, z.rho,
                                        v, z.T, self.tallies["e_rad"], n_elec,
                                        L_dep=R.get("L_radio_dep"), L_emit=R.get("L_radio_emit"),
                                        X=z.X if fr else None, elems=elems if fr else None)

    def close(self):
        self.eng.close()


def run_steady(workload, outdir: str = ".", precision: int = abi.PREC_FP64, device: int = 0) -> Transport:
    """Steady-state iterations as the reference's driver runs them
    (SedonaClass::evolve_system with transport_steady_iterate = n): each
    iteration steps the transport and writes spectrum_<it>.dat and
    plt_<it>.dat at the grid time; the last iteration is flagged
    (SedonaClass.cpp:333), which pumps its emission."""
    n_iter = max(1, workload.P.scalar("transport_steady_iterate", int))
    tr = Transport(workload, precision=precision, device=device)
    for it in range(1, n_iter + 1):
        tr.step(1.0, last_iteration=(it == n_iter))
        tr.output_spectrum(it, outdir)
        tr.write_plotfile(it, workload.zones.t_now, outdir)
    return tr


def step_size(t: float, dt_max: float, dt_min: float, dt_del: float) -> float:
    """The driver's time step (SedonaClass.cpp:318-328, no hydro limit):
    tstep_max_dt, at most tstep_max_delta of the time once t > 0, at least
    tstep_min_dt."""
    dt = dt_max
    if dt_del > 0 and t > 0 and dt > t * dt_del:
        dt = t * dt_del
    if dt < dt_min:
        dt = dt_min
    return dt


def run_time_dependent(workload, outdir: Optional[str] = ".", precision: int = abi.PREC_FP64, device: int = 0,
                       on_write=None) -> Transport:
    """The reference driver's time loop (SedonaClass::evolve_system,
    src/main/SedonaClass.cpp:300-414) for a time-dependent run: per step the
    step size (tstep_max_dt, at most tstep_max_delta of the time once t > 0,
    at least tstep_min_dt), the homologous hydro step when hydro_module is
    "homologous", the transport step, and every output_write_plt_file_time a
    plot file and spectrum (with outdir) at t + dt; the loop ends after the
    step that starts beyond tstep_time_stop or after tstep_max_steps steps.
    on_write(i_write, t_write, transport) is called at each write."""
    from . import workloads as wl
    P = workload.P
    n_steps = int(P.scalar("tstep_max_steps", int))
    t_stop = P.scalar("tstep_time_stop")
    dt_max, dt_min, dt_del = P.scalar("tstep_max_dt"), P.scalar("tstep_min_dt"), P.scalar("tstep_max_delta")
    write_step = P.scalar("output_write_plt_file_time")
    write_log = P.scalar("output_write_plt_log_space")
    hydro = P.get("hydro_module") == "homologous"
    tr = Transport(workload, precision=precision, device=device)
    t = workload.zones.t_now
    next_write = t
    i_write = 0
    for _ in range(n_steps):
        dt = step_size(t, dt_max, dt_min, dt_del)
        if hydro:
            wl.homologous_step(workload.zones, dt)
        tr.step(dt)
        if t >= next_write:
            t_write = t + dt
            if outdir is not None:
                if workload.zones.type == abi.GRID_1D_SPHERE:
                    tr.write_plotfile(i_write + 1, t_write, outdir)
                tr.output_spectrum(i_write + 1, outdir)
            if on_write is not None:
                on_write(i_write + 1, t_write, tr)
            next_write = next_write * (1.0 + write_log) if (write_log > 0 and i_write > 0) else next_write + write_step
            i_write += 1
        if t > t_stop:
            break
        t += dt
    return tr

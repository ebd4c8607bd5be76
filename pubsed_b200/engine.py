"""Thin Python driver of the CUDA library (one sed_ctx) for a Workload.

Used by the benchmark and by pubsed_b200.transport; every call goes through
the C ABI of include/sedona_gpu.h.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import abi
from ._lib import lib as _load


class Engine:
    def __init__(self, workload, precision: int = abi.PREC_FP64, device: int = 0,
                 n_packets: Optional[int] = None, seed_offset: int = 0):
        self.L = _load()
        self.w = workload
        self.keep = abi.Keep()
        self.tp = workload.transport_params(self.keep, precision, n_packets)
        self.tp.rng_seed = (self.tp.rng_seed + seed_offset) & 0xFFFFFFFF
        self.ctx = C.c_void_p()
        self._check(self.L.sed_ctx_create(C.byref(self.tp), device, C.byref(self.ctx)), "sed_ctx_create")
        _, L_core, weights = workload.core_source()
        if weights is not None:  # core_spectrum_file in place of the blackbody
            w = np.ascontiguousarray(weights, dtype=np.float64)
            self._check(self.L.sed_set_core_source(self.ctx, L_core, w.ctypes.data_as(abi._dp)), "sed_set_core_source")
        self.nz = workload.zones.n_zones
        self.nn = self.tp.nu_grid.n
        self.nspec = self.tp.spec_time.n * self.tp.spec_nu.n * self.tp.spec_mu.n * self.tp.spec_phi.n
        self.upload_grid()
        op = workload.opacity_params(self.keep)
        self._check(self.L.sed_set_opacity_params(self.ctx, C.byref(op)), "sed_set_opacity_params")
        at = workload.atomic_struct(self.keep)
        if at is not None:
            self._check(self.L.sed_set_atomic_data(self.ctx, C.byref(at)), "sed_set_atomic_data")

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self.L.sed_last_error(self.ctx) if self.ctx else b""
            raise RuntimeError("%s failed (%d): %s" % (what, rc, (msg or b"").decode()))

    def upload_grid(self) -> int:
        """sed_set_grid from host arrays; returns the bytes copied host->device."""
        k = abi.Keep()
        g = self.w.grid_struct(k)
        self._check(self.L.sed_set_grid(self.ctx, C.byref(g)), "sed_set_grid")
        return int(sum(a.nbytes for a in k.arrays))

    def set_opacity(self, dt: float = 1.0):
        self._check(self.L.sed_set_opacity(self.ctx, dt), "sed_set_opacity")

    def transport(self, dt: float = 1.0) -> dict:
        st = abi.StepStats()
        self._check(self.L.sed_transport(self.ctx, dt, C.byref(st)), "sed_transport")
        return st.as_dict()

    def step(self, dt: float = 1.0) -> dict:
        st = abi.StepStats()
        self._check(self.L.sed_step(self.ctx, dt, C.byref(st)), "sed_step")
        return st.as_dict()

    def solve_temperature(self, set_Tgas_to_Trad: int = 0):
        """sed_solve_temperature: new zone temperatures (also kept on the
        device for the next opacity build) and the number of zones Brent left
        unsolved."""
        T = np.zeros(self.nz)
        bad = C.c_int32(0)
        self._check(self.L.sed_solve_temperature(self.ctx, int(set_Tgas_to_Trad), T.ctypes.data_as(abi._dp),
                                                 C.byref(bad)), "sed_solve_temperature")
        return T, int(bad.value)

    def spectrum(self):
        flux = np.zeros(self.nspec)
        click = np.zeros(self.nspec)
        self._check(self.L.sed_get_spectrum(self.ctx, flux.ctypes.data_as(abi._dp), click.ctypes.data_as(abi._dp)),
                    "sed_get_spectrum")
        return flux, click

    def tallies(self, J: bool = True) -> dict:
        """Zone tallies; J=False skips the [n_zones x n_bins] J_nu array."""
        nj = self.nn if self.tp.store_Jnu else 1
        out = {"J_nu": np.zeros(self.nz * nj)} if J else {}
        out.update({k: np.zeros(self.nz) for k in ("e_abs", "e_rad", "fx", "fy", "fz", "fr")})
        P = lambda a: a.ctypes.data_as(abi._dp)
        self._check(self.L.sed_get_zone_tallies(self.ctx, P(out["J_nu"]) if J else None, P(out["e_abs"]), P(out["e_rad"]),
                                                P(out["fx"]), P(out["fy"]), P(out["fz"]), P(out["fr"])),
                    "sed_get_zone_tallies")
        return out

    def set_core_luminosity(self, L: float) -> None:
        """sed_set_core_source with the spectrum kept."""
        self._check(self.L.sed_set_core_source(self.ctx, float(L), None), "sed_set_core_source")
        self.tp.core_luminosity = float(L)

    def time(self) -> float:
        return float(self.L.sed_get_time(self.ctx))

    def initialize_particles(self, n: int, e_rad) -> None:
        """sed_initialize_particles: n packets of the radiation field e_rad."""
        e = np.ascontiguousarray(e_rad, dtype=np.float64)
        self._check(self.L.sed_initialize_particles(self.ctx, int(n), e.ctypes.data_as(abi._dp)),
                    "sed_initialize_particles")

    def n_particles(self) -> int:
        return int(self.L.sed_n_particles(self.ctx))

    def set_emission(self, core_n_emit: float, n_emit_radioactive: int):
        """sed_set_emission: packet counts of the following steps."""
        self._check(self.L.sed_set_emission(self.ctx, float(core_n_emit), int(n_emit_radioactive)), "sed_set_emission")
        self.tp.core_n_emit = float(core_n_emit)
        self.tp.n_emit_radioactive = int(n_emit_radioactive)

    def radioactive(self) -> dict:
        """Radioactive source results of the last step: L_radio_emit and
        L_radio_dep per zone (per volume) and the gamma-ray spectrum."""
        le, ld = np.zeros(self.nz), np.zeros(self.nz)
        ng = self.tp.spec_time.n * max(self.tp.gamma_nu.n, 1) * self.tp.spec_mu.n * self.tp.spec_phi.n
        gf, gc = np.zeros(ng), np.zeros(ng)
        P = lambda a: a.ctypes.data_as(abi._dp)
        self._check(self.L.sed_get_radioactive_tallies(self.ctx, P(le), P(ld)), "sed_get_radioactive_tallies")
        self._check(self.L.sed_get_gamma_spectrum(self.ctx, P(gf), P(gc)), "sed_get_gamma_spectrum")
        return {"L_radio_emit": le, "L_radio_dep": ld, "gamma_flux": gf, "gamma_click": gc}

    def opacity(self) -> dict:
        n = self.nz * self.nn
        out = {k: np.zeros(n) for k in ("abs", "scat", "emis_cdf")}
        out.update({k: np.zeros(self.nz) for k in ("n_elec", "eps_imc", "planck_mean", "rosseland_mean", "L_thermal")})
        P = lambda a: a.ctypes.data_as(abi._dp)
        self._check(self.L.sed_get_opacity(self.ctx, P(out["abs"]), P(out["scat"]), P(out["emis_cdf"]),
                                           P(out["n_elec"]), P(out["eps_imc"]), P(out["planck_mean"]),
                                           P(out["rosseland_mean"]), P(out["L_thermal"])), "sed_get_opacity")
        return out

    def close(self):
        if self.ctx:
            self.L.sed_ctx_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""Python driver of a batch of independent 1D models (sed_batch_* in
include/sedona_gpu.h) built from a workloads.BatchWorkload.

Every model of the batch keeps its own Sedona parameters; the parameters a
batch shares (grids, switches, opacity parameters, atomic data, element
list, grid time) are taken from the first model and must be equal in all.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._lib import lib as _load

# parameters that may differ between the models of one batch: the model
# itself and its core source / packet stream
PER_MODEL = {"core_n_emit", "core_radius", "core_luminosity", "core_temperature", "transport_rng_seed",
             "particles_max_total", "model_file"}


class BatchEngine:
    def __init__(self, bw, precision: int = abi.PREC_MIXED, device: int = 0, graph: bool = True):
        self.L = _load()
        self.bw = bw
        self.keep = abi.Keep()
        first = bw.models[0]
        for m in bw.models[1:]:
            for k, v in first.params.items():
                if k not in PER_MODEL and m.params.get(k) != v:
                    raise ValueError("batch models differ in shared parameter %s" % k)
            if m.zones.t_now != first.zones.t_now or m.atoms is not first.atoms:
                raise ValueError("batch models must share t_now and atomic data")
            if not np.array_equal(m.zones.elem_Z, first.zones.elem_Z):
                raise ValueError("batch models must share the element list")
        self.tp = first.transport_params(self.keep, precision)
        self.tp.max_particles = max(int(m.P.scalar("particles_max_total", int)) for m in bw.models)
        n = len(bw.models)
        arr = (abi.BatchModel * n)()
        for i, w in enumerate(bw.models):
            z, P, d = w.zones, w.P, arr[i]
            d.n_zones = z.n_zones
            d.r_min = z.r_min
            d.r_out = self.keep.d(z.r_out)
            d.vol = self.keep.d(z.vol)
            d.rho = self.keep.d(z.rho)
            d.T_gas = self.keep.d(z.T)
            d.e_gas = None
            d.total_grey_opacity = self.keep.d(w.total_grey())
            d.X = self.keep.d(z.X.reshape(-1))
            d.core_n_emit = w.n_packets
            d.core_radius = P.scalar("core_radius")
            d.core_luminosity = P.function("core_luminosity", z.t_now)
            d.core_temperature = P.scalar("core_temperature")
            d.rng_seed = P.scalar("transport_rng_seed", int) & 0xFFFFFFFF
            d.first_packet_id = 0
        self.models = arr
        self.b = C.c_void_p()
        zs = first.zones
        rc = self.L.sed_batch_create(C.byref(self.tp), zs.t_now, zs.n_elems, self.keep.i(zs.elem_Z),
                                     self.keep.i(zs.elem_A), n, arr, device, C.byref(self.b))
        if rc != 0:
            raise RuntimeError("sed_batch_create failed (%d)" % rc)
        op = first.opacity_params(self.keep)
        self._check(self.L.sed_batch_set_opacity_params(self.b, C.byref(op)), "sed_batch_set_opacity_params")
        at = first.atomic_struct(self.keep)
        if at is not None:
            self._check(self.L.sed_batch_set_atomic_data(self.b, C.byref(at)), "sed_batch_set_atomic_data")
        self._check(self.L.sed_batch_use_graph(self.b, int(graph)), "sed_batch_use_graph")
        self.nn = self.tp.nu_grid.n
        self.nspec = self.tp.spec_time.n * self.tp.spec_nu.n * self.tp.spec_mu.n * self.tp.spec_phi.n

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self.L.sed_batch_last_error(self.b) if self.b else b""
            raise RuntimeError("%s failed (%d): %s" % (what, rc, (msg or b"").decode()))

    def autotune(self, sample_fraction: float = 0.05) -> dict:
        t = abi.BatchTuning()
        self._check(self.L.sed_batch_autotune(self.b, sample_fraction, C.byref(t)), "sed_batch_autotune")
        return t.as_dict()

    def set_tuning(self, variant: int, queue_chunk: int = 1, blocks_per_sm: int = 0):
        t = abi.BatchTuning(variant=variant, threads=0, blocks_per_sm=blocks_per_sm, queue_chunk=queue_chunk)
        self._check(self.L.sed_batch_set_tuning(self.b, C.byref(t)), "sed_batch_set_tuning")

    def record(self, on: bool = True):
        self._check(self.L.sed_batch_record_packets(self.b, int(on)), "sed_batch_record_packets")

    def step(self, dt: float = 1.0) -> dict:
        st = abi.StepStats()
        self._check(self.L.sed_batch_step(self.b, dt, C.byref(st)), "sed_batch_step")
        return st.as_dict()

    def set_zone_state(self, m: int, rho=None, T=None) -> int:
        """Copies model m's density / temperature to the device; returns the bytes copied."""
        k = abi.Keep()
        self._check(self.L.sed_batch_set_zone_state(self.b, m, k.d(rho), k.d(T)), "sed_batch_set_zone_state")
        return int(sum(a.nbytes for a in k.arrays))

    def escaped(self) -> np.ndarray:
        out = np.zeros(len(self.bw.models), np.int64)
        self._check(self.L.sed_batch_get_escaped(self.b, out.ctypes.data_as(C.POINTER(C.c_int64))),
                    "sed_batch_get_escaped")
        return out

    def spectrum(self, m: int):
        flux = np.zeros(self.nspec)
        click = np.zeros(self.nspec)
        self._check(self.L.sed_batch_get_spectrum(self.b, m, flux.ctypes.data_as(abi._dp),
                                                  click.ctypes.data_as(abi._dp)), "sed_batch_get_spectrum")
        return flux, click

    def tallies(self, m: int, J: bool = True) -> dict:
        nz = self.bw.models[m].zones.n_zones
        nj = self.nn if self.tp.store_Jnu else 1
        out = {"J_nu": np.zeros(nz * nj)} if J else {}
        out.update({k: np.zeros(nz) for k in ("e_abs", "e_rad", "fx", "fy", "fz", "fr")})
        P = lambda a: a.ctypes.data_as(abi._dp)
        self._check(self.L.sed_batch_get_zone_tallies(self.b, m, P(out["J_nu"]) if J else None, P(out["e_abs"]),
                                                      P(out["e_rad"]), P(out["fx"]), P(out["fy"]), P(out["fz"]),
                                                      P(out["fr"])), "sed_batch_get_zone_tallies")
        return out

    def opacity(self, m: int) -> dict:
        nz = self.bw.models[m].zones.n_zones
        out = {k: np.zeros(nz * self.nn) for k in ("abs", "scat", "emis_cdf")}
        out.update({k: np.zeros(nz) for k in ("n_elec", "eps_imc")})
        P = lambda a: a.ctypes.data_as(abi._dp)
        self._check(self.L.sed_batch_get_opacity(self.b, m, P(out["abs"]), P(out["scat"]), P(out["emis_cdf"]),
                                                 P(out["n_elec"]), P(out["eps_imc"])), "sed_batch_get_opacity")
        return out

    def records(self, m: int, n: int) -> dict:
        fate = np.zeros(n, np.int32); ind = np.zeros(n, np.int32); draws = np.zeros(n, np.int32)
        st = np.zeros(n * 9)
        self._check(self.L.sed_batch_get_packet_records(self.b, m, n, fate.ctypes.data_as(abi._ip),
                                                        ind.ctypes.data_as(abi._ip), draws.ctypes.data_as(abi._ip),
                                                        st.ctypes.data_as(abi._dp)), "sed_batch_get_packet_records")
        return {"fate": fate, "ind": ind, "draws": draws, "state": st.reshape(n, 9)}

    def close(self):
        if self.b:
            self.L.sed_batch_destroy(self.b)
            self.b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

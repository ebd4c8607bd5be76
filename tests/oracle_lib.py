"""Loads the C oracle (oracle/liboracle.so) and drives it, or the CUDA
library, through the same ABI calls.  Test infrastructure."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

from pubsed_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
_lib = None


def build_oracle(force: bool = False) -> str:
    src = os.path.join(ROOT, "oracle", "sed_oracle.c")
    if force or not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True)
    return ORACLE_SO


def oracle_lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = abi.declare(C.CDLL(build_oracle()), "oracle_")
    return _lib


class Engine:
    """One context of either library, fed from a Workload."""

    def __init__(self, lib: C.CDLL, prefix: str, workload, precision: int = abi.PREC_FP64,
                 n_packets: Optional[int] = None, device: int = 0):
        self.lib, self.p, self.w = lib, prefix, workload
        self.keep = abi.Keep()
        self.tp = workload.transport_params(self.keep, precision, n_packets)
        self.ctx = C.c_void_p()
        f = getattr(lib, prefix + "ctx_create")
        rc = f(C.byref(self.tp), device, C.byref(self.ctx)) if prefix == "sed_" else f(C.byref(self.tp), C.byref(self.ctx))
        self.check(rc, "ctx_create")
        self.nz = workload.zones.n_zones
        self.nn = self.tp.nu_grid.n
        self.nspec = self.tp.spec_time.n * self.tp.spec_nu.n * self.tp.spec_mu.n * self.tp.spec_phi.n
        self.set_grid()
        op = workload.opacity_params(self.keep)
        self.check(self.fn("set_opacity_params")(self.ctx, C.byref(op)), "set_opacity_params")
        at = workload.atomic_struct(self.keep)
        if at is not None:
            self.check(self.fn("set_atomic_data")(self.ctx, C.byref(at)), "set_atomic_data")

    def fn(self, name):
        return getattr(self.lib, self.p + name)

    def check(self, rc, what):
        if rc != 0:
            msg = self.fn("last_error")(self.ctx) if getattr(self, "ctx", None) else b""
            raise RuntimeError("%s%s failed (%d): %s" % (self.p, what, rc, (msg or b"").decode()))

    def set_grid(self):
        g = self.w.grid_struct(self.keep)
        self.check(self.fn("set_grid")(self.ctx, C.byref(g)), "set_grid")

    def set_opacity(self, dt: float = 1.0):
        self.check(self.fn("set_opacity")(self.ctx, dt), "set_opacity")

    def load_opacity(self, abs_, scat, cdf, eps_imc):
        k = abi.Keep()
        self.check(self.fn("load_opacity")(self.ctx, k.d(abs_), k.d(scat), k.d(cdf), k.d(eps_imc)), "load_opacity")

    def record(self, on: bool = True):
        self.check(self.fn("record_packets")(self.ctx, int(on)), "record_packets")

    def transport(self, dt: float = 1.0) -> dict:
        st = abi.StepStats()
        self.check(self.fn("transport")(self.ctx, dt, C.byref(st)), "transport")
        return st.as_dict()

    def transport_range(self, first: int, count: int, finish: bool, dt: float = 1.0) -> dict:
        st = abi.StepStats()
        self.check(self.fn("transport_range")(self.ctx, dt, first, count, int(finish), C.byref(st)), "transport_range")
        return st.as_dict()

    def spectrum(self):
        flux = np.zeros(self.nspec); click = np.zeros(self.nspec)
        k = abi.Keep()
        self.check(self.fn("get_spectrum")(self.ctx, flux.ctypes.data_as(abi._dp), click.ctypes.data_as(abi._dp)), "get_spectrum")
        return flux, click

    def tallies(self) -> dict:
        nj = self.nn if self.tp.store_Jnu else 1
        J = np.zeros(self.nz * nj)
        arrs = {n: np.zeros(self.nz) for n in ("e_abs", "e_rad", "fx", "fy", "fz", "fr")}
        P = lambda a: a.ctypes.data_as(abi._dp)
        self.check(self.fn("get_zone_tallies")(self.ctx, P(J), P(arrs["e_abs"]), P(arrs["e_rad"]), P(arrs["fx"]),
                                               P(arrs["fy"]), P(arrs["fz"]), P(arrs["fr"])), "get_zone_tallies")
        arrs["J_nu"] = J
        return arrs

    def opacity(self) -> dict:
        n = self.nz * self.nn
        out = {k: np.zeros(n) for k in ("abs", "scat", "emis_cdf")}
        out.update({k: np.zeros(self.nz) for k in ("n_elec", "eps_imc", "planck_mean", "rosseland_mean", "L_thermal")})
        P = lambda a: a.ctypes.data_as(abi._dp)
        self.check(self.fn("get_opacity")(self.ctx, P(out["abs"]), P(out["scat"]), P(out["emis_cdf"]), P(out["n_elec"]),
                                          P(out["eps_imc"]), P(out["planck_mean"]), P(out["rosseland_mean"]),
                                          P(out["L_thermal"])), "get_opacity")
        return out

    def records(self, n: int) -> dict:
        fate = np.zeros(n, np.int32); ind = np.zeros(n, np.int32); draws = np.zeros(n, np.int32)
        st = np.zeros(n * 9)
        self.check(self.fn("get_packet_records")(self.ctx, n, fate.ctypes.data_as(abi._ip), ind.ctypes.data_as(abi._ip),
                                                  draws.ctypes.data_as(abi._ip), st.ctypes.data_as(abi._dp)), "get_packet_records")
        return {"fate": fate, "ind": ind, "draws": draws, "state": st.reshape(n, 9)}

    def close(self):
        if self.ctx:
            self.fn("ctx_destroy")(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

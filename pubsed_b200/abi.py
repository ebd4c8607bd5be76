"""ctypes mirror of the C ABI in include/sedona_gpu.h.

Struct layouts here must match the header field for field.  `Bound` turns
a Workload (numpy arrays) into the C structs and keeps every array alive for
as long as the structs are in use.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any

import numpy as np

SED_OK = 0
SED_ERR_ARG = 1
SED_ERR_CUDA = 2
SED_ERR_CAPACITY = 3
SED_WARN_NO_PARTICLE_SPACE = 1
SED_ERR_STATE = 4
SED_ERR_LIMIT = 5
SED_ERR_NOMEM = 6

LOC_FLEX, LOC_LIN, LOC_LOG, LOC_NONE = 0, 1, 2, 3
GRID_1D_SPHERE, GRID_3D_CART = 0, 1
PREC_FP64, PREC_MIXED = 0, 1

# ParticleFate (src/transport/particle.h:9)
FATE_MOVING, FATE_STOPPED, FATE_ESCAPED, FATE_ABSORBED = 0, 1, 2, 3

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class LocateGrid(C.Structure):
    _fields_ = [("n", C.c_int32), ("type", C.c_int32), ("min", C.c_double),
                ("del_", C.c_double), ("right", _dp)]


class TransportParams(C.Structure):
    _fields_ = [
        ("steady_state", C.c_int32), ("radiative_eq", C.c_int32),
        ("boundary_in_reflect", C.c_int32), ("boundary_out_reflect", C.c_int32),
        ("store_Jnu", C.c_int32), ("omit_scattering", C.c_int32),
        ("core_fix_luminosity", C.c_int32), ("tally_forces", C.c_int32),
        ("precision", C.c_int32), ("rng_seed", C.c_uint32),
        ("max_particles", C.c_int64), ("core_n_emit", C.c_int64),
        ("core_radius", C.c_double), ("core_luminosity", C.c_double),
        ("core_temperature", C.c_double), ("core_photon_frequency", C.c_double),
        ("fleck_alpha", C.c_double), ("max_segments", C.c_int32), ("reserved", C.c_int32),
        ("first_packet_id", C.c_int64),
        ("nu_grid", LocateGrid), ("spec_time", LocateGrid), ("spec_nu", LocateGrid),
        ("spec_mu", LocateGrid), ("spec_phi", LocateGrid),
        ("n_emit_radioactive", C.c_int64), ("force_rprocess_heating", C.c_int32), ("reserved3", C.c_int32),
        ("gamma_nu", LocateGrid),
        ("use_ddmc", C.c_int32), ("reserved4", C.c_int32), ("ddmc_tau", C.c_double),
    ]


class Grid(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("n_zones", C.c_int32), ("homologous", C.c_int32),
        ("n_elems", C.c_int32), ("t_now", C.c_double), ("r_min", C.c_double),
        ("r_out", _dp), ("v_r", _dp),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("x_axis", LocateGrid), ("y_axis", LocateGrid), ("z_axis", LocateGrid),
        ("vol", _dp), ("rho", _dp), ("T_gas", _dp), ("e_gas", _dp),
        ("total_grey_opacity", _dp), ("X", _dp), ("elem_Z", _ip), ("elem_A", _ip),
    ]


class OpacityParams(C.Structure):
    _fields_ = [
        ("use_electron_scattering", C.c_int32), ("use_free_free", C.c_int32),
        ("use_bound_free", C.c_int32), ("use_line_expansion", C.c_int32),
        ("use_fuzz_expansion", C.c_int32), ("n_atom_zero_epsilon", C.c_int32),
        ("atom_zero_epsilon", _ip), ("epsilon", C.c_double),
        ("maximum_opacity", C.c_double), ("temp_min", C.c_double), ("temp_max", C.c_double),
        ("line_velocity_width", C.c_double),
    ]


class AtomicData(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32), ("ion_off", _ip), ("ion_chi", _dp),
        ("lev_off", _ip), ("lev_ion", _ip), ("lev_g", _ip), ("lev_ic", _ip),
        ("lev_E", _dp), ("lev_Eion", _dp), ("photo_off", _ip), ("photo_E", _dp),
        ("photo_s", _dp), ("line_off", _ip), ("line_l", _ip), ("line_u", _ip),
        ("line_nu", _dp), ("line_f", _dp), ("fuzz_off", _ip), ("fuzz_nu", _dp),
        ("fuzz_gf", _dp), ("fuzz_El", _dp), ("fuzz_ion", _ip),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("n_packets", C.c_int64), ("n_escaped", C.c_int64), ("n_absorbed", C.c_int64),
        ("n_stopped", C.c_int64), ("n_segments", C.c_int64), ("n_scatters", C.c_int64),
        ("n_limit", C.c_int64), ("kernel_launches", C.c_int32), ("warnings", C.c_int32),
        ("ms_opacity", C.c_float), ("ms_transport", C.c_float), ("ms_total", C.c_float),
        ("ms_propagate_kernel", C.c_float),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchModel(C.Structure):
    _fields_ = [
        ("n_zones", C.c_int32), ("reserved", C.c_int32), ("r_min", C.c_double),
        ("r_out", _dp), ("vol", _dp), ("rho", _dp), ("T_gas", _dp), ("e_gas", _dp),
        ("total_grey_opacity", _dp), ("X", _dp),
        ("core_n_emit", C.c_int64), ("core_radius", C.c_double), ("core_luminosity", C.c_double),
        ("core_temperature", C.c_double), ("rng_seed", C.c_uint32), ("reserved2", C.c_int32),
        ("first_packet_id", C.c_int64),
    ]


class BatchTuning(C.Structure):
    _fields_ = [("variant", C.c_int32), ("threads", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("queue_chunk", C.c_int32), ("ms", C.c_float), ("n_tried", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


@dataclass
class Keep:
    """Holds numpy buffers referenced by C structs."""
    arrays: list = field(default_factory=list)

    def d(self, a) -> Any:
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.arrays.append(a)
        return a.ctypes.data_as(_dp)

    def i(self, a) -> Any:
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.int32)
        self.arrays.append(a)
        return a.ctypes.data_as(_ip)


def locate_grid(keep: Keep, g) -> LocateGrid:
    """g: pubsed_b200.grids.LocGrid"""
    return LocateGrid(int(g.n), int(g.type), float(g.min), float(g.delta), keep.d(g.right))


def declare(lib: C.CDLL, prefix: str) -> C.CDLL:
    """Attach argtypes/restype for the ABI functions under `prefix` ("sed_")."""
    vp = C.c_void_p
    sig = {
        "ctx_create": ([C.POINTER(TransportParams), C.c_int, C.POINTER(vp)], C.c_int),
        "set_grid": ([vp, C.POINTER(Grid)], C.c_int),
        "set_atomic_data": ([vp, C.POINTER(AtomicData)], C.c_int),
        "set_opacity_params": ([vp, C.POINTER(OpacityParams)], C.c_int),
        "set_opacity": ([vp, C.c_double], C.c_int),
        "load_opacity": ([vp, _dp, _dp, _dp, _dp], C.c_int),
        "transport": ([vp, C.c_double, C.POINTER(StepStats)], C.c_int),
        "get_spectrum": ([vp, _dp, _dp], C.c_int),
        "get_zone_tallies": ([vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp], C.c_int),
        "get_opacity": ([vp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp], C.c_int),
        "record_packets": ([vp, C.c_int32], C.c_int),
        "get_packet_records": ([vp, C.c_int64, _ip, _ip, _ip, _dp], C.c_int),
        "last_error": ([vp], C.c_char_p),
        "ctx_destroy": ([vp], None),
    }
    if prefix == "sed_":
        sig["step"] = ([vp, C.c_double, C.POINTER(StepStats)], C.c_int)
        sig["version"] = ([], C.c_char_p)
    else:
        sig["ctx_create"] = ([C.POINTER(TransportParams), C.POINTER(vp)], C.c_int)
        sig["transport_range"] = ([vp, C.c_double, C.c_int64, C.c_int64, C.c_int, C.POINTER(StepStats)], C.c_int)
        sig["get_fuzz_bins"] = ([vp, _ip], C.c_int)
        sig["locate"] = ([C.POINTER(LocateGrid), C.c_double], C.c_int)
    sig.update({
        "set_rng_step": ([vp, C.c_uint32], C.c_int),
        "diff_forward": ([vp, C.c_double, _dp, C.c_int32, C.POINTER(StepStats)], C.c_int),
        "diff_vjp": ([vp, _dp, _dp, C.POINTER(StepStats)], C.c_int),
        "diff_jacobian": ([vp, _dp, C.POINTER(StepStats)], C.c_int),
        "diff_vjp_density": ([vp, _dp, _dp, C.POINTER(StepStats)], C.c_int),
        "solve_temperature": ([vp, C.c_int32, _dp, _ip], C.c_int),
        "get_gamma_spectrum": ([vp, _dp, _dp], C.c_int),
        "get_radioactive_tallies": ([vp, _dp, _dp], C.c_int),
        "set_emission": ([vp, C.c_double, C.c_int64], C.c_int),
        "get_particles": ([vp, C.c_int64, _ip, _ip, _dp], C.c_int),
        "set_time": ([vp, C.c_double], C.c_int),
        "get_time": ([vp], C.c_double),
        "initialize_particles": ([vp, C.c_int64, _dp], C.c_int),
        "n_particles": ([vp], C.c_int64),
        "wipe_spectra": ([vp], C.c_int),
        "set_core_source": ([vp, C.c_double, _dp], C.c_int),
    })
    if prefix == "sed_":
        i64p = C.POINTER(C.c_int64)
        sig.update({
            "batch_create": ([C.POINTER(TransportParams), C.c_double, C.c_int32, _ip, _ip, C.c_int32,
                              C.POINTER(BatchModel), C.c_int, C.POINTER(vp)], C.c_int),
            "batch_set_opacity_params": ([vp, C.POINTER(OpacityParams)], C.c_int),
            "batch_set_atomic_data": ([vp, C.POINTER(AtomicData)], C.c_int),
            "batch_autotune": ([vp, C.c_double, C.POINTER(BatchTuning)], C.c_int),
            "batch_set_tuning": ([vp, C.POINTER(BatchTuning)], C.c_int),
            "batch_use_graph": ([vp, C.c_int32], C.c_int),
            "batch_step": ([vp, C.c_double, C.POINTER(StepStats)], C.c_int),
            "batch_set_zone_state": ([vp, C.c_int32, _dp, _dp], C.c_int),
            "batch_get_escaped": ([vp, i64p], C.c_int),
            "batch_get_spectrum": ([vp, C.c_int32, _dp, _dp], C.c_int),
            "batch_get_zone_tallies": ([vp, C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp, _dp], C.c_int),
            "batch_get_opacity": ([vp, C.c_int32, _dp, _dp, _dp, _dp, _dp], C.c_int),
            "batch_record_packets": ([vp, C.c_int32], C.c_int),
            "batch_get_packet_records": ([vp, C.c_int32, C.c_int64, _ip, _ip, _ip, _dp], C.c_int),
            "batch_last_error": ([vp], C.c_char_p),
            "batch_destroy": ([vp], None),
            # device-pointer forms of the differentiable transport (pointers as integers)
            "diff_forward_dev": ([vp, C.c_double, vp, C.c_int32, vp, C.POINTER(StepStats)], C.c_int),
            "diff_vjp_dev": ([vp, vp, vp, C.POINTER(StepStats)], C.c_int),
            "diff_vjp_density_dev": ([vp, vp, vp, C.POINTER(StepStats)], C.c_int),
            "diff_scale_extinction": ([vp, _dp], C.c_int),
            "diff_scale_extinction_dev": ([vp, vp], C.c_int),
        })
    for name, (args, res) in sig.items():
        fn = getattr(lib, prefix + name)
        fn.argtypes = args
        fn.restype = res
    return lib

"""Loads the CUDA library (pubsed_b200/libsedona_gpu.so) through ctypes.

There is no CPU fallback: if the library is missing or no CUDA device is
visible, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsedona_gpu.so")
CSRC = os.path.join(HERE, "csrc")
_lib = None


def build(force: bool = False) -> str:
    """Compiles the CUDA sources for sm_100a with nvcc (works without a GPU)."""
    args = ["make", "-s", "-C", CSRC]
    if force:
        subprocess.run(["make", "-s", "-C", CSRC, "clean"], check=True)
    subprocess.run(args, check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("CUDA library %s is not built; run pubsed_b200._lib.build()" % LIB_PATH)
        _lib = abi.declare(C.CDLL(LIB_PATH), "sed_")
    return _lib


EXPORTED = [
    "sed_ctx_create", "sed_set_grid", "sed_set_atomic_data", "sed_set_opacity_params",
    "sed_set_opacity", "sed_load_opacity", "sed_transport", "sed_step", "sed_get_spectrum",
    "sed_get_zone_tallies", "sed_get_opacity", "sed_record_packets", "sed_get_packet_records",
    "sed_n_particles", "sed_last_error", "sed_ctx_destroy", "sed_version",
    "sed_set_rng_step", "sed_diff_forward", "sed_diff_vjp", "sed_diff_vjp_density", "sed_diff_jacobian", "sed_solve_temperature",
    "sed_diff_forward_dev", "sed_diff_vjp_dev", "sed_diff_vjp_density_dev", "sed_diff_scale_extinction",
    "sed_diff_scale_extinction_dev",
    "sed_get_gamma_spectrum", "sed_get_radioactive_tallies", "sed_set_emission",
    "sed_get_particles", "sed_set_time", "sed_get_time", "sed_initialize_particles", "sed_wipe_spectra", "sed_set_core_source",
    "sed_batch_create", "sed_batch_set_opacity_params", "sed_batch_set_atomic_data", "sed_batch_autotune",
    "sed_batch_set_tuning", "sed_batch_use_graph", "sed_batch_step", "sed_batch_set_zone_state", "sed_batch_get_escaped",
    "sed_batch_get_spectrum", "sed_batch_get_zone_tallies", "sed_batch_get_opacity", "sed_batch_record_packets",
    "sed_batch_get_packet_records", "sed_batch_last_error", "sed_batch_destroy",
]

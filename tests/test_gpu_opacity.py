"""Parity of the CUDA opacity build (LTE solve + line binning + continuum)
with the oracle, and of a full step (opacity -> emission -> propagation).

FP64 tables: 1e-12 relative.  Mixed precision (FP32 line sums with Kahan
compensation, FP32 packed tables): 1e-5 relative against the FP64 oracle,
the tolerance the mixed-precision form is specified to meet.
"""
import numpy as np
import pytest

from pubsed_b200 import abi, workloads
import oracle_lib

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12
MIXED_RTOL = 1e-5


def _engines(sed_lib, w, precision):
    o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    g = oracle_lib.Engine(sed_lib, "sed_", w, precision=precision)
    o.set_opacity(1.0)
    g.set_opacity(1.0)
    return o, g


def _maxrel(a, b, floor=0.0):
    s = np.maximum(np.abs(b), floor)
    s[s == 0] = 1e-300
    return float(np.max(np.abs(a - b) / s))


@pytest.mark.parametrize("bf,ff", [(0, 1), (1, 1)])
def test_lte_opacity_fp64(sed_lib, bf, ff):
    w = workloads.type_ia(n_packets=10, n_zones=24, n_lines=20000, n_bins=512, bound_free=bf, free_free=ff,
                          n_levels_per_ion=8)
    o, g = _engines(sed_lib, w, abi.PREC_FP64)
    Oo, Og = o.opacity(), g.opacity()
    for k in ("n_elec", "abs", "scat", "emis_cdf", "planck_mean", "rosseland_mean", "L_thermal", "eps_imc"):
        assert _maxrel(Og[k], Oo[k]) <= FP64_RTOL, k


def test_lte_opacity_mixed(sed_lib):
    w = workloads.type_ia(n_packets=10, n_zones=32, n_lines=50000, n_bins=1024)
    o, g = _engines(sed_lib, w, abi.PREC_MIXED)
    Oo, Og = o.opacity(), g.opacity()
    assert _maxrel(Og["n_elec"], Oo["n_elec"]) <= FP64_RTOL
    for k in ("abs", "scat"):
        assert _maxrel(Og[k], Oo[k]) <= MIXED_RTOL, k


def test_full_step_replay_fp64(sed_lib):
    n = 3000
    w = workloads.type_ia(n_packets=n, n_zones=48, n_lines=30000, n_bins=1024)
    o, g = _engines(sed_lib, w, abi.PREC_FP64)
    o.record(True)
    g.record(True)
    so, sg = o.transport(1.0), g.transport(1.0)
    ro, rg = o.records(n), g.records(n)
    assert np.array_equal(ro["fate"], rg["fate"])
    assert np.array_equal(ro["ind"], rg["ind"])
    assert np.array_equal(ro["draws"], rg["draws"])
    oracle_lib.check_states(rg["state"], ro["state"])
    assert so["n_segments"] == sg["n_segments"]
    fo, co = o.spectrum()
    fg, cg = g.spectrum()
    assert np.array_equal(co, cg)
    assert _maxrel(fg, fo) <= oracle_lib.TALLY_RTOL
    To, Tg = o.tallies(), g.tallies()
    oracle_lib.zone_tally_close(Tg["J_nu"], To["J_nu"])
    oracle_lib.zone_tally_close(Tg["e_abs"], To["e_abs"])

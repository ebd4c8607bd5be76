"""Parity of the CUDA packet kernel with the oracle, through the C ABI.

Replay: the oracle and the GPU draw identical Philox deviates per packet,
so per-packet integer outcomes (fate, final zone, number of deviates drawn)
must be identical and the final FP64 state must agree to 1e-12 relative
(oracle_lib.check_states spells out the criterion).
Tallies are sums of the same terms in a different order (FP64 atomics),
compared within oracle_lib.TALLY_RTOL; final packet states with
oracle_lib.check_states.
"""
import numpy as np
import pytest

from pubsed_b200 import abi, workloads
import oracle_lib

pytestmark = pytest.mark.gpu

TALLY_RTOL = oracle_lib.TALLY_RTOL


def _pair(sed_lib, w, precision=abi.PREC_FP64, record=True):
    o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    g = oracle_lib.Engine(sed_lib, "sed_", w, precision=precision)
    o.set_opacity(1.0)
    g.set_opacity(1.0)
    if record:
        o.record(True)
        g.record(True)
    so = o.transport(1.0)
    sg = g.transport(1.0)
    return o, g, so, sg


def _rel(a, b):
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin), "non-finite pattern differs"
    d = np.abs(a[fin] - b[fin])
    s = np.maximum(np.abs(b[fin]), 1e-300)
    return float(np.max(d / s)) if d.size else 0.0


@pytest.mark.parametrize("radiative_eq", [0, 1])
def test_replay_lightbulb_grey(sed_lib, radiative_eq):
    n = 4000
    w = workloads.lightbulb_grey(n_packets=n, radiative_eq=radiative_eq)
    o, g, so, sg = _pair(sed_lib, w)
    ro, rg = o.records(n), g.records(n)
    assert np.array_equal(ro["fate"], rg["fate"])
    assert np.array_equal(ro["ind"], rg["ind"])
    assert np.array_equal(ro["draws"], rg["draws"])
    oracle_lib.check_states(rg["state"], ro["state"])
    for k in ("n_escaped", "n_absorbed", "n_segments", "n_scatters"):
        assert so[k] == sg[k], k
    To, Tg = o.tallies(), g.tallies()
    # path-length tallies, compared against their largest entry
    for k in ("J_nu", "e_abs", "e_rad", "fx", "fy", "fz", "fr"):
        oracle_lib.zone_tally_close(Tg[k], To[k])
    fo, co = o.spectrum()
    fg, cg = g.spectrum()
    assert np.array_equal(co, cg)
    assert _rel(fg, fo) <= TALLY_RTOL


def test_grey_opacity_tables_match(sed_lib):
    w = workloads.lightbulb_grey(n_packets=10)
    o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    g = oracle_lib.Engine(sed_lib, "sed_", w)
    o.set_opacity(1.0)
    g.set_opacity(1.0)
    Oo, Og = o.opacity(), g.opacity()
    for k in ("abs", "scat", "eps_imc"):
        assert _rel(Og[k], Oo[k]) <= 1e-15, k
    # the CDF prefix sum, L_thermal and the means are sums of the same
    # non-negative terms in a blocked / tree order: within n * 2^-53 of the
    # sequential sum (1024 bins)
    for k in ("emis_cdf", "L_thermal", "planck_mean", "rosseland_mean"):
        assert _rel(Og[k], Oo[k]) <= 1e-13, k


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_loaded_tables_replay(sed_lib, precision):
    """sed_load_opacity: tables computed elsewhere (here the oracle's) drive the
    packet kernel; the coarse and guide tables of the emissivity CDF are built
    from them on the host.  FP64: every packet as in the oracle; mixed: the
    same tables in FP32, spectrum within Monte Carlo noise of the FP64 run
    (the mixed form draws its own deviates)."""
    n = 4000
    w = workloads.type_ia(n_packets=n, n_zones=32, n_lines=5000, n_bins=512, spectrum_bins=64, seed=23)
    o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    o.set_opacity(1.0)
    T = o.opacity()
    g = oracle_lib.Engine(sed_lib, "sed_", w, precision=precision)
    g.load_opacity(T["abs"], T["scat"], T["emis_cdf"], T["eps_imc"])
    g.record(True)
    o.record(True)
    so = o.transport(1.0)
    sg = g.transport(1.0)
    if precision == abi.PREC_FP64:
        ro, rg = o.records(n), g.records(n)
        assert np.array_equal(ro["fate"], rg["fate"])
        assert np.array_equal(ro["draws"], rg["draws"])
        oracle_lib.check_states(rg["state"], ro["state"])
    else:
        assert abs(sg["n_escaped"] - so["n_escaped"]) <= 5 * np.sqrt(so["n_escaped"]) + 5
    o.close()
    g.close()


@pytest.mark.parametrize("case", ["grey", "ia"])
def test_temperature_solve_matches_oracle(sed_lib, case):
    """sed_solve_temperature after a replayed step: Brent on the same emission
    sums gives the oracle's temperatures (the oracle's are the reference's,
    tests/test_oracle_golden.py); the next opacity build runs at them; and
    set_Tgas_to_Trad gives (e_rad / a)^(1/4)."""
    if case == "grey":
        w = workloads.lightbulb_grey(n_packets=20000, n_zones=64, n_bins=256, radiative_eq=1, seed=4)
    else:
        w = workloads.type_ia(n_packets=4000, n_zones=32, n_lines=5000, n_bins=512, spectrum_bins=64, seed=24)
    o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    g = oracle_lib.Engine(sed_lib, "sed_", w)
    for e in (o, g):
        e.set_opacity(1.0)
        e.transport(1.0)
    To, bo = oracle_lib.solve_temperature(o)
    Tg, bg = oracle_lib.solve_temperature(g)
    assert bo == bg == 0
    # e_abs agrees to the summation order (1e-12); the root to far below
    # Brent's 1e-2 K tolerance
    assert np.max(np.abs(Tg - To) / To) <= 1e-9, np.max(np.abs(Tg - To) / To)
    for e in (o, g):
        e.set_opacity(1.0)
    Oo, Og = o.opacity(), g.opacity()
    for k in ("abs", "scat", "eps_imc"):
        assert _rel(Og[k], Oo[k]) <= 1e-8, k
    Ro, _ = oracle_lib.solve_temperature(o, set_Tgas_to_Trad=1)
    Rg, _ = oracle_lib.solve_temperature(g, set_Tgas_to_Trad=1)
    assert _rel(Rg, Ro) <= 1e-10
    o.close()
    g.close()


@pytest.mark.parametrize("name", ["replay_core_file", "replay_core_derived"])
def test_core_source_rules_match_reference_replay(sed_lib, name):
    """The inner source as transport::setup_core_emission sets it up: a
    spectrum read from core_spectrum_file with its luminosity the file's
    integral, and a core temperature derived from L and r_core; every packet
    against the reference's replayed step."""
    import json
    import os
    from pubsed_b200 import workloads
    ref = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name + ".npz"))
    w = getattr(workloads, str(ref["generator"]))(**json.loads(str(ref["kwargs"])))
    g = oracle_lib.Engine(sed_lib, "sed_", w)
    g.set_opacity(1.0)
    g.record(True)
    st = g.transport(1.0)
    n = int(ref["pkt_fate"].size)
    rec = g.records(n)
    for k in ("fate", "ind", "draws"):
        assert np.array_equal(rec[k], ref["pkt_" + k]), k
    oracle_lib.check_states(rec["state"], ref["pkt_state"].reshape(-1, 9))
    assert st["n_escaped"] == int(ref["n_escaped"])
    f, c = g.spectrum()
    assert np.array_equal(c, ref["spec_click"])
    g.close()

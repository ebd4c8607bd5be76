"""The radioactive source on the GPU: 56Ni/56Co decay luminosity per zone,
gamma-ray emission and transport (Klein-Nishina Compton scattering and
photo-electric absorption, both depositing into L_radio_dep), positrons
deposited on the spot, and the optical photons all of these hand to the packet
kernel (transport::emit_radioactive, src/transport/emission.cpp:165-243;
do_scatter / compton_scatter, src/transport/scatter.cpp:45-133).

FP64 form: every packet against the reference's own replayed step (golden
fixtures) and, at larger sizes, against the oracle -- fate, final zone and
deviates drawn exactly, final states within oracle_lib's criterion; zone and
spectrum tallies are sums of the same terms in another order.  Mixed form:
the gamma-ray phase reads no FP32 table, so packets that end as gamma-rays
are identical to the FP64 form's.
"""
import json
import os

import numpy as np
import pytest

from pubsed_b200 import abi, workloads
import oracle_lib

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rel(a, b):
    d = np.abs(a - b)
    s = np.maximum(np.abs(b), 1e-300)
    return float(np.max(d / s)) if d.size else 0.0


def _load(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    w = getattr(workloads, str(d["generator"]))(**json.loads(str(d["kwargs"])))
    return d, w


def _step(lib, w, precision=abi.PREC_FP64):
    prefix = "oracle_" if lib is oracle_lib.oracle_lib() else "sed_"
    e = oracle_lib.Engine(lib, prefix, w, precision=precision)
    e.set_opacity(1.0)
    e.record(True)
    st = e.transport(1.0)
    return e, st


@pytest.mark.parametrize("name", ["replay_ia_radio", "replay_ia_radio_late"])
def test_radioactive_step_matches_reference_replay(sed_lib, name):
    ref, w = _load(name)
    g, st = _step(sed_lib, w)
    n = int(ref["pkt_fate"].size)
    assert st["n_packets"] == n
    rec = g.records(n)
    assert np.array_equal(rec["fate"], ref["pkt_fate"])
    assert np.array_equal(rec["ind"], ref["pkt_ind"])
    assert np.array_equal(rec["draws"], ref["pkt_draws"])
    oracle_lib.check_states(rec["state"], ref["pkt_state"].reshape(-1, 9))
    assert st["n_escaped"] == int(ref["n_escaped"])
    R = g.radioactive()
    assert _rel(R["L_radio_emit"], ref["L_radio_emit"]) <= 1e-12
    oracle_lib.zone_tally_close(R["L_radio_dep"], ref["L_radio_dep"])
    assert np.array_equal(R["gamma_click"], ref["gamma_click"])
    assert _rel(R["gamma_flux"], ref["gamma_flux"]) <= oracle_lib.TALLY_RTOL
    f, c = g.spectrum()
    assert np.array_equal(c, ref["spec_click"])
    assert _rel(f, ref["spec_flux"]) <= oracle_lib.TALLY_RTOL
    T = g.tallies()
    for k, rk in (("e_abs", "e_abs"), ("e_rad", "e_rad"), ("fr", "fr_rad")):
        oracle_lib.zone_tally_close(T[k], ref[rk])
    g.close()


@pytest.mark.parametrize("t_days", [20.0, 120.0])
def test_radioactive_step_matches_oracle(sed_lib, t_days):
    """40000 decay packets and 4000 core packets on 64 zones."""
    w = workloads.type_ia(n_packets=4000, n_zones=64, n_lines=20000, n_bins=512, n_levels_per_ion=8, v_core=1e8,
                          n_radioactive=40000, t_days=t_days, seed=31)
    g, sg = _step(sed_lib, w)
    o, so = _step(oracle_lib.oracle_lib(), w)
    n = 44000
    rg, ro = g.records(n), o.records(n)
    for k in ("fate", "ind", "draws"):
        assert np.array_equal(rg[k], ro[k]), k
    oracle_lib.check_states(rg["state"], ro["state"])
    for k in ("n_packets", "n_escaped", "n_absorbed", "n_stopped", "n_segments", "n_scatters"):
        assert sg[k] == so[k], k
    Rg, Ro = g.radioactive(), o.radioactive()
    assert _rel(Rg["L_radio_emit"], Ro["L_radio_emit"]) <= 1e-12
    oracle_lib.zone_tally_close(Rg["L_radio_dep"], Ro["L_radio_dep"])
    assert np.array_equal(Rg["gamma_click"], Ro["gamma_click"])
    assert _rel(Rg["gamma_flux"], Ro["gamma_flux"]) <= oracle_lib.TALLY_RTOL
    fg, cg = g.spectrum()
    fo, co = o.spectrum()
    assert np.array_equal(cg, co)
    assert _rel(fg, fo) <= oracle_lib.TALLY_RTOL
    Tg, To = g.tallies(), o.tallies()
    for k in ("J_nu", "e_abs", "e_rad", "fx", "fy", "fz", "fr"):
        oracle_lib.zone_tally_close(Tg[k], To[k])
    # energy bookkeeping: positrons deposit their energy on the spot, and a
    # gamma-ray that stays one ends escaped or absorbed, so the deposited
    # energy is at most the decay energy (lab-frame shifts are ~v/c)
    vol = w.zones.vol
    E_dep = float(np.sum(Rg["L_radio_dep"] * vol))
    E_tot = float(np.sum(Rg["L_radio_emit"] * vol))
    assert 0 < E_dep <= 1.2 * E_tot
    g.close()
    o.close()


def test_mixed_form_keeps_the_gamma_ray_phase(sed_lib):
    w = workloads.type_ia(n_packets=2000, n_zones=64, n_lines=20000, n_bins=512, n_levels_per_ion=8, v_core=1e8,
                          n_radioactive=30000, t_days=120.0, seed=37)
    g64, s64 = _step(sed_lib, w, abi.PREC_FP64)
    g32, s32 = _step(sed_lib, w, abi.PREC_MIXED)
    n = 32000
    r64, r32 = g64.records(n), g32.records(n)
    radio = np.arange(n) >= 2000
    gamma_end = radio & (r64["state"][:, 8] < 1e3)  # MeV: still a gamma-ray
    assert gamma_end.sum() > 1000
    for k in ("fate", "ind", "draws"):
        assert np.array_equal(r64[k][gamma_end], r32[k][gamma_end]), k
    assert np.array_equal(r64["state"][gamma_end], r32["state"][gamma_end])
    R64, R32 = g64.radioactive(), g32.radioactive()
    assert np.array_equal(R64["gamma_click"], R32["gamma_click"])
    assert np.array_equal(R64["L_radio_emit"], R32["L_radio_emit"])
    # deposition: the same terms (gamma-ray phase only), summed in another order
    oracle_lib.zone_tally_close(R32["L_radio_dep"], R64["L_radio_dep"])
    assert s32["n_packets"] == s64["n_packets"] == n
    g64.close()
    g32.close()


def test_no_radioactive_material_emits_nothing(sed_lib):
    """L_tot = 0: the reference returns before emitting (emission.cpp:211)."""
    w = workloads.type_ia(n_packets=500, n_zones=16, n_lines=2000, n_bins=128, n_levels_per_ion=6,
                          n_radioactive=300, seed=41)
    w.zones.X[:, 2] += w.zones.X[:, -1]  # the 56Ni layer becomes silicon
    w.zones.X[:, -1] = 0.0
    g, sg = _step(sed_lib, w)
    o, so = _step(oracle_lib.oracle_lib(), w)
    rg, ro = g.records(800), o.records(800)
    assert np.all(rg["fate"][500:] == -1) and np.all(ro["fate"][500:] == -1)
    for k in ("fate", "ind", "draws"):
        assert np.array_equal(rg[k], ro[k]), k
    Rg = g.radioactive()
    assert np.all(Rg["L_radio_emit"] == 0) and np.all(Rg["L_radio_dep"] == 0)
    assert sg["n_escaped"] + sg["n_absorbed"] + sg["n_stopped"] == 500
    g.close()
    o.close()


def test_capacity_rules(sed_lib):
    """Core packets that do not fit next to the radioactive ones are not
    emitted and the step runs with the decay packets alone, flagged in its
    warnings (emit_inner_source, emission.cpp:391-392); radioactive packets
    that alone exceed particles_max_total are not emitted
    (emission.cpp:215-218)."""
    w = workloads.type_ia(n_packets=500, n_zones=16, n_lines=2000, n_bins=128, n_levels_per_ion=6, v_core=1e8,
                          n_radioactive=300, seed=43)
    w.params["particles_max_total"] = 700
    out = []
    for lib in (sed_lib, oracle_lib.oracle_lib()):
        e, st = _step(lib, w)
        assert st["n_packets"] == 300
        assert st["warnings"] & abi.SED_WARN_NO_PARTICLE_SPACE
        out.append(e.records(300))
        e.close()
    assert np.array_equal(out[0]["fate"], out[1]["fate"])
    assert np.array_equal(out[0]["draws"], out[1]["draws"])
    w.params["particles_max_total"] = 200
    w.params["core_n_emit"] = 100
    for lib in (sed_lib, oracle_lib.oracle_lib()):
        e, st = _step(lib, w)
        assert st["n_packets"] == 100
        e.close()


def test_forced_rprocess_heating(sed_lib):
    """force_rprocess_heating: the Lippuner-Roberts heating rate with no
    gamma-rays, so every decay packet deposits where it is emitted and the
    deposited luminosity equals the decay luminosity."""
    w = workloads.type_ia(n_packets=1000, n_zones=32, n_lines=5000, n_bins=256, n_levels_per_ion=6, v_core=1e8,
                          n_radioactive=20000, seed=47)
    w.params["force_rprocess_heating"] = 1
    g, sg = _step(sed_lib, w)
    o, so = _step(oracle_lib.oracle_lib(), w)
    rg, ro = g.records(21000), o.records(21000)
    for k in ("fate", "ind", "draws"):
        assert np.array_equal(rg[k], ro[k]), k
    oracle_lib.check_states(rg["state"], ro["state"])
    Rg, Ro = g.radioactive(), o.radioactive()
    assert _rel(Rg["L_radio_emit"], Ro["L_radio_emit"]) <= 1e-12
    oracle_lib.zone_tally_close(Rg["L_radio_dep"], Ro["L_radio_dep"])
    vol = w.zones.vol
    assert abs(np.sum(Rg["L_radio_dep"] * vol) / np.sum(Rg["L_radio_emit"] * vol) - 1) < 1e-9
    assert np.all(Rg["gamma_click"] == 0)
    g.close()
    o.close()


def test_transport_driver_writes_the_reference_outputs(sed_lib, tmp_path):
    """Transport.step through the public host API, then the plot file
    (L_dep_nuc / L_emit_nuc columns) and the gamma-ray spectrum text, read
    back as numbers against the reference's own files of the replayed step."""
    from pubsed_b200.transport import Transport
    ref, w = _load("replay_ia_radio_late")
    w.params["gamma_name"] = "gamma"
    w.params["spectrum_name"] = "spectrum"
    tr = Transport(w)
    st = tr.step(1.0)
    assert st["n_packets"] == int(ref["pkt_fate"].size)
    tr.output_spectrum(1, str(tmp_path))
    p = tr.write_plotfile(1, w.zones.t_now, str(tmp_path))
    mine = np.loadtxt(p)
    theirs = np.loadtxt(str(ref["plt_dat"]).splitlines())
    assert mine.shape == theirs.shape
    # r, rho, v exact; T_gas from the solve (Brent on tallies equal to ~1e-14);
    # T_rad, L_dep and L_emit from tallies
    assert np.array_equal(mine[:, :3], theirs[:, :3])
    assert np.allclose(mine[:, 3:], theirs[:, 3:], rtol=1e-7, atol=0)
    g = np.loadtxt(str(tmp_path / "gamma_1.dat"))
    gr = np.loadtxt(str(ref["gamma_dat"]).splitlines())
    assert np.array_equal(g[:, 0], gr[:, 0]) and np.array_equal(g[:, 2], gr[:, 2])
    assert np.allclose(g[:, 1], gr[:, 1], rtol=1e-7, atol=0)
    tr.close()


def test_set_emission_matches_oracle(sed_lib):
    """A context made without a radioactive source takes one for its second
    step (sed_set_emission); that step matches the oracle's packet for packet."""
    w = workloads.type_ia(n_packets=1000, n_zones=32, n_lines=5000, n_bins=256, n_levels_per_ion=6, v_core=1e8,
                          n_radioactive=0, t_days=60.0, seed=53)
    engines = []
    for lib, prefix in ((sed_lib, "sed_"), (oracle_lib.oracle_lib(), "oracle_")):
        e = oracle_lib.Engine(lib, prefix, w)
        e.set_opacity(1.0)
        e.transport(1.0)
        e.check(e.fn("set_emission")(e.ctx, 500.0, 6000), "set_emission")
        e.tp.n_emit_radioactive = 6000
        e.record(True)
        e.set_opacity(1.0)
        engines.append((e, e.transport(1.0)))
    (g, sg), (o, so) = engines
    assert sg["n_packets"] == so["n_packets"] == 6500
    rg, ro = g.records(6500), o.records(6500)
    for k in ("fate", "ind", "draws"):
        assert np.array_equal(rg[k], ro[k]), k
    oracle_lib.check_states(rg["state"], ro["state"])
    assert np.array_equal(g.radioactive()["gamma_click"], o.radioactive()["gamma_click"])
    g.close()
    o.close()

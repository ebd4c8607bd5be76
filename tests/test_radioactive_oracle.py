"""The oracle's radioactive source on the CPU: the edge cases and the
energy bookkeeping that the reference's emission rules give
(transport::emit_radioactive, src/transport/emission.cpp:165-243)."""
import numpy as np
import pytest

from pubsed_b200 import abi, workloads
import oracle_lib


def _step(w):
    e = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    e.set_opacity(1.0)
    e.record(True)
    return e, e.transport(1.0)


def _small(**over):
    kw = dict(n_packets=200, n_zones=16, n_lines=2000, n_bins=128, n_levels_per_ion=6, v_core=1e8,
              n_radioactive=400, seed=51)
    kw.update(over)
    return workloads.type_ia(**kw)


def test_every_emitted_packet_ends_once():
    w = _small(t_days=60.0)
    e, st = _step(w)
    assert st["n_packets"] == 600
    assert st["n_escaped"] + st["n_absorbed"] + st["n_stopped"] == 600
    rec = e.records(600)
    assert np.all(rec["fate"] >= 1)
    # radioactive packets record every deviate of their stream: at least the
    # eight of a gamma-ray's emission
    assert np.all(rec["draws"][200:] >= 8)
    e.close()


def test_no_radioactive_material():
    w = _small()
    w.zones.X[:, 2] += w.zones.X[:, -1]
    w.zones.X[:, -1] = 0.0
    e, st = _step(w)
    assert st["n_packets"] == 600
    assert st["n_escaped"] + st["n_absorbed"] + st["n_stopped"] == 200
    rec = e.records(600)
    assert np.all(rec["fate"][200:] == -1)
    R = e.radioactive()
    assert np.all(R["L_radio_emit"] == 0) and np.all(R["L_radio_dep"] == 0)
    e.close()


def test_forced_rprocess_deposits_everything():
    w = _small()
    w.params["force_rprocess_heating"] = 1
    e, st = _step(w)
    R = e.radioactive()
    vol = w.zones.vol
    assert abs(np.sum(R["L_radio_dep"] * vol) / np.sum(R["L_radio_emit"] * vol) - 1) < 1e-12
    assert np.all(R["gamma_click"] == 0)
    e.close()


def test_capacity():
    w = _small()
    w.params["particles_max_total"] = 500
    # the 200 core packets do not fit next to the 400 decay packets: the step
    # runs without them ("# Not enough particle space", emission.cpp:391-392)
    e, st = _step(w)
    assert st["n_packets"] == 400
    assert st["warnings"] & abi.SED_WARN_NO_PARTICLE_SPACE
    e.close()
    w.params["particles_max_total"] = 300  # the 400 decay packets alone do not fit
    e, st = _step(w)
    assert st["n_packets"] == 200
    e.close()


def test_decay_luminosity_follows_the_56ni_chain():
    """L_radio_emit per unit mass of 56Ni at two epochs against the two-step
    decay chain written out here (tau_Ni = 8.8 d, tau_Co = 111.4 d, 1.725 and
    3.730 MeV per decay)."""
    for t_days in (5.0, 80.0):
        w = _small(t_days=t_days)
        e, _ = _step(w)
        R = e.radioactive()
        z = w.zones
        ni = z.X[:, -1] > 0
        t = t_days * 86400.0
        tn, tc = 757241.8, 9627379.0
        mev = 1.60217646e-6
        rate = (np.exp(-t / tn) / tn * 1.725 + (np.exp(-t / tn) - np.exp(-t / tc)) / (tn - tc) * 3.730) * mev
        expect = z.rho[ni] * z.X[ni, -1] / (56 * 1.67262158e-24) * rate
        assert np.allclose(R["L_radio_emit"][ni], expect, rtol=1e-12)
        assert np.all(R["L_radio_emit"][~ni] == 0)
        e.close()


def test_set_emission_changes_the_next_step():
    """sed_/oracle_set_emission: a context made without a radioactive source
    can take one later (the gamma-ray spectrum is allocated then)."""
    w = _small(n_radioactive=0)
    e = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    e.set_opacity(1.0)
    assert e.transport(1.0)["n_packets"] == 200
    e.check(e.fn("set_emission")(e.ctx, 300.0, 500), "set_emission")
    e.tp.n_emit_radioactive = 500
    st = e.transport(1.0)
    assert st["n_packets"] == 800
    R = e.radioactive()
    assert np.sum(R["L_radio_emit"]) > 0
    with pytest.raises(RuntimeError, match=r"\(1\)"):
        e.check(e.fn("set_emission")(e.ctx, -1.0, 0), "set_emission")
    e.close()


def test_emission_count_rules():
    """Transport.emission_counts: dt scaling of the radioactive count
    (truncated), then the last-iteration pump of both counts."""
    from types import SimpleNamespace
    from pubsed_b200.params import Params
    from pubsed_b200.transport import Transport
    P = Params({"core_n_emit": 1000, "multiply_particles_n_emit_by_dt_over_dtmax": 1, "tstep_max_dt": 3.0,
                "particles_last_iter_pump": 10})
    t = SimpleNamespace(P=P, n_radio=100)
    assert Transport.emission_counts(t, 1.0, False) == (1000, 33)
    assert Transport.emission_counts(t, 1.0, True) == (10000, 330)
    P2 = Params({"core_n_emit": 1000, "particles_last_iter_pump": 0})
    t2 = SimpleNamespace(P=P2, n_radio=100)
    assert Transport.emission_counts(t2, 0.5, True) == (1000, 100)

"""Time-dependent steps of the oracle against the reference's own replayed
steps (CPU): packets that reach the end of a step are carried to the next in
the order transport::clean_up_particle_vector leaves them
(src/transport/transport.cpp:164-194), the grid expands homologously before
each step (hydro_homologous::step), the transport clock advances by dt, the
spectrum accumulates over the steps, and the initial radiation field's
packets (transport::initialize_particles) start in the census."""
import json
import os

import numpy as np
import pytest

from pubsed_b200 import workloads
import oracle_lib

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_td(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    kw = json.loads(str(d["kwargs"]))
    w = workloads.time_dependent(**kw)
    return d, w, kw


def _rel(a, b):
    fin = np.isfinite(b)  # fr is NaN in a zone whose packets pass r = 0, in both codes
    assert np.array_equal(np.isfinite(a), fin)
    s = np.maximum(np.abs(b[fin]), 1e-300)
    return float(np.max(np.abs(a[fin] - b[fin]) / s)) if s.size else 0.0


@pytest.mark.parametrize("name", ["replay_td_grey", "replay_td_ia_radio", "replay_td_ddmc_ia", "replay_td_ddmc_grey",
                                  "replay_td_full", "replay_td_imd_grey", "replay_td_imd_ia"])
def test_oracle_matches_reference_time_dependent_replay(name):
    ref, w, kw = load_td(name)
    steps = int(ref["steps"])
    e = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    radio = bool(kw.get("n_radioactive"))
    if kw.get("n_initialize"):
        e.initialize_particles(kw["n_initialize"], workloads.initial_e_rad(w.zones))
        c = e.census()
        assert np.array_equal(c["ind"], ref["init_ind"])
        assert oracle_lib.state_rel(c["state"], ref["init_state"].reshape(-1, 9)) <= 1e-14
        e2 = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", load_td(name)[1])
        res = oracle_lib.td_steps(e2, e2.w, steps, kw["n_initialize"], radio)
    else:
        res = oracle_lib.td_steps(e, w, steps, 0, radio)
    for s, r in enumerate(res):
        sf = "_s%d" % s
        rec = r["records"]
        # a step whose core packets found no room emitted none and carried on
        # with the census (emission.cpp:391-392)
        full = bool(r["stats"]["warnings"] & 1)
        assert rec["fate"].size == ref["pkt_fate" + sf].size
        if name == "replay_td_full":
            assert full == (s % 2 == 0), s
        assert np.array_equal(rec["fate"], ref["pkt_fate" + sf]), s
        assert np.array_equal(rec["ind"], ref["pkt_ind" + sf]), s
        assert np.array_equal(rec["draws"], ref["pkt_draws" + sf]), s
        assert oracle_lib.state_rel(rec["state"], ref["pkt_state" + sf].reshape(-1, 9)) <= 1e-13
        c = r["census"]
        assert np.array_equal(c["ind"], ref["census_ind" + sf])
        assert np.array_equal(c["type"], ref["census_type" + sf])
        assert oracle_lib.state_rel(c["state"], ref["census_state" + sf].reshape(-1, 9)) <= 1e-13
        f, cl = r["spectrum"]
        assert np.array_equal(cl, ref["spec_click" + sf])
        assert _rel(f, ref["spec_flux" + sf]) <= 1e-12
        T = r["tallies"]
        for k, rk in (("e_abs", "e_abs"), ("e_rad", "e_rad"), ("fr", "fr_rad")):
            assert _rel(T[k], ref[rk + sf]) <= 1e-12, (s, k)
        if radio:
            R = r["radio"]
            assert _rel(R["L_radio_emit"], ref["L_radio_emit" + sf]) <= 1e-14
            assert _rel(R["L_radio_dep"], ref["L_radio_dep" + sf]) <= 1e-12
            assert np.array_equal(R["gamma_click"], ref["gamma_click" + sf])
        if "T_gas" in r:
            assert _rel(r["T_gas"], ref["T_gas" + sf]) <= 1e-10
    # the carried packets end the last step at its end time, which is also
    # the grid's time after the last hydro step (not after an IMD call: it
    # advances the photon's time by the step's end time, as the reference does)
    last = res[-1]["census"]["state"]
    if last.size and kw.get("params", {}).get("transport_use_ddmc") != 1:
        ww = e2.w if kw.get("n_initialize") else w
        assert np.allclose(last[:, 6], ww.zones.t_now, rtol=1e-12)


def test_clock_and_spectrum_accumulate():
    w = workloads.time_dependent("lightbulb_grey", n_initialize=0, dt_days=0.1, n_packets=100, n_zones=16,
                                 n_bins=64, seed=5)
    e = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    t0 = e.fn("get_time")(e.ctx)
    res = oracle_lib.td_steps(e, w, 2)
    assert e.fn("get_time")(e.ctx) == t0 + w.notes["dt"] + w.notes["dt"]
    c1 = res[0]["spectrum"][1].sum()
    c2 = res[1]["spectrum"][1].sum()
    assert c2 >= c1  # the second step adds to the first step's spectrum
    e.check(e.fn("wipe_spectra")(e.ctx), "wipe_spectra")
    assert e.spectrum()[1].sum() == 0
    e.close()


def test_driver_step_sizes():
    """The driver's step rule on the diffusing pulse's settings: the first
    step is tstep_max_dt (t = 0), then at most 10% of the time until that
    exceeds tstep_max_dt; tstep_min_dt is a floor."""
    from pubsed_b200.transport import step_size
    t, seq = 0.0, []
    for _ in range(40):
        dt = step_size(t, 5e-10, 0.0, 0.1)
        seq.append(dt)
        t += dt
    assert seq[0] == 5e-10 and seq[1] == 5e-10 * 0.1
    assert all(b >= a for a, b in zip(seq[1:], seq[2:]))
    assert seq[-1] == 5e-10
    assert step_size(1.0, 5e-10, 1e-9, 0.1) == 1e-9

"""Device-side bounds that end a loop the reference leaves unbounded: each
stops the loop, finishes the step with the results it has, and makes the
call return SED_ERR_LIMIT with the count in the step's statistics.

* The per-packet segment limit (gpu_max_segments; propagate_monte_carlo,
  src/transport/transport.cpp:260-484, has none): a packet that reaches it
  ends the step as stopped, where it was.  FP64 form: which packets stop,
  and their states, are the oracle's; mixed form: the count is consistent.
* The effective-scattering loop of a diffusion event
  (src/transport/discrete_diffusion.cpp:270-277) repeats until the
  re-emitted photon leaves its frequency bin; with one bin, eps_imc = 1 and
  no radiative equilibrium every pass absorbs and none ever leaves, so the
  reference never ends.  Here it gives up after 65 536 passes.

Every loop involved is bounded by construction, so nothing here can hang.
"""
import ctypes as C

import numpy as np
import pytest

from pubsed_b200 import abi, workloads
import oracle_lib

pytestmark = pytest.mark.gpu


def _transport(e, dt=1.0):
    st = abi.StepStats()
    rc = e.fn("transport")(e.ctx, dt, C.byref(st))
    return rc, st.as_dict()


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_segment_limit_stops_packets(sed_lib, precision):
    n, limit = 3000, 8
    w = workloads.lightbulb_grey(n_packets=n, n_zones=32, n_bins=64, radiative_eq=1, seed=13)
    w.params["gpu_max_segments"] = limit
    g = oracle_lib.Engine(sed_lib, "sed_", w, precision=precision)
    g.set_opacity(1.0)
    g.record(True)
    rc, st = _transport(g)
    assert rc == abi.SED_ERR_LIMIT
    assert b"segment limit" in g.fn("last_error")(g.ctx)
    rg = g.records(n)
    stopped = rg["fate"] == 1
    # a steady-state step stops packets only at the limit; each of them ran
    # exactly `limit` segments
    assert st["n_limit"] == st["n_stopped"] == int(stopped.sum()) > 0
    assert st["n_escaped"] + st["n_absorbed"] + st["n_stopped"] == n
    assert st["n_segments"] <= n * limit
    if precision == abi.PREC_FP64:
        o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
        o.set_opacity(1.0)
        o.record(True)
        ro_rc, so = _transport(o)
        assert ro_rc == abi.SED_ERR_LIMIT
        assert so["n_limit"] == st["n_limit"]
        ro = o.records(n)
        for k in ("fate", "ind", "draws"):
            assert np.array_equal(rg[k], ro[k]), k
        oracle_lib.check_states(rg["state"], ro["state"])
        o.close()
    # without the limit the same packets run to the end
    w.params["gpu_max_segments"] = 0
    g2 = oracle_lib.Engine(sed_lib, "sed_", w, precision=precision)
    g2.set_opacity(1.0)
    st2 = g2.transport(1.0)
    assert st2["n_limit"] == 0 and st2["n_stopped"] == 0
    g.close()
    g2.close()


def test_diffusion_effective_scattering_bound(sed_lib):
    """DDMC (method 2) on the diffusing pulse's grey sphere with four
    frequency bins, absorption (epsilon 0.5), Fleck factor 1 (no Fleck
    factor) and no radiative equilibrium: an effective-scattering event
    (there are some: the zone's emission is spread over the bins, so the
    inelastic fraction is not 0) absorbs on every pass and never changes bin,
    so each one ends at the 65 536-pass bound; the step returns
    SED_ERR_LIMIT and the oracle, bounded the same way, agrees packet for
    packet."""
    n = 200
    w = workloads.diffusing_pulse(n_initialize=n, seed=3)
    w.params["opacity_epsilon"] = 0.5
    w.params["transport_radiative_equilibrium"] = 0
    w.params["transport_fleck_alpha"] = 0
    w.params["transport_nu_grid"] = [1e14, 1e16, 10 ** 0.5 - 1, 1]  # four log bins
    dt = 5e-10
    out = []
    for lib, prefix in ((sed_lib, "sed_"), (oracle_lib.oracle_lib(), "oracle_")):
        e = oracle_lib.Engine(lib, prefix, w)
        e.initialize_particles(n, workloads.initial_e_rad(w.zones))
        e.set_opacity(dt)
        e.record(True)
        rc, st = _transport(e, dt)
        out.append((rc, st, e.records(st["n_packets"]), e))
    (rg, sg, recg, eg), (ro, so, reco, eo) = out
    assert rg == abi.SED_ERR_LIMIT and ro == abi.SED_ERR_LIMIT
    assert b"diffusion" in eg.fn("last_error")(eg.ctx)
    assert sg["n_scatters"] > 0
    for k in ("fate", "ind", "draws"):
        assert np.array_equal(recg[k], reco[k]), k
    eg.close()
    eo.close()

"""Batches of independent 1D models (sed_batch_*) against the same models run
one by one: through the oracle, and through separate CUDA contexts.

A model's packets keep that model's Philox key and stream ids inside the
batch, so every packet must have the integer history it has alone (fate,
final zone, deviates drawn) and the same final state (oracle_lib's
criterion); spectra and zone tallies are sums of the same terms in another
order (oracle_lib tolerances).  Steps after the first replay a captured CUDA
graph; the autotuned launch shape must not change any result.
"""
import numpy as np
import pytest

from pubsed_b200 import abi, workloads
from pubsed_b200.batch import BatchEngine
import oracle_lib

pytestmark = pytest.mark.gpu


def small_batch(**over):
    kw = dict(n_models=5, zones=(40, 120), packets=(500, 3000), n_lines=2000, n_bins=256, seed=3, data_seed=1)
    kw.update(over)
    return workloads.batch64(**kw)


def _rel(a, b):
    d = np.abs(a - b)
    s = np.maximum(np.abs(b), 1e-300)
    return float(np.max(d / s)) if d.size else 0.0


def _same_packets(rb, rs):
    assert np.array_equal(rb["fate"], rs["fate"])
    assert np.array_equal(rb["ind"], rs["ind"])
    assert np.array_equal(rb["draws"], rs["draws"])
    oracle_lib.check_states(rb["state"], rs["state"])


def _same_tallies(Tb, Ts):
    for k in ("J_nu", "e_abs", "e_rad", "fx", "fy", "fz", "fr"):
        oracle_lib.zone_tally_close(Tb[k], Ts[k])


def test_batch_matches_oracle_model_by_model(sed_lib):
    bw = small_batch()
    be = BatchEngine(bw, precision=abi.PREC_FP64, graph=False)
    be.record(True)
    st = be.step(1.0)
    assert st["n_packets"] == bw.n_packets
    esc = be.escaped()
    n_esc = 0
    for m, w in enumerate(bw.models):
        n = w.n_packets
        o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
        o.set_opacity(1.0)
        o.record(True)
        so = o.transport(1.0)
        _same_packets(be.records(m, n), o.records(n))
        assert esc[m] == so["n_escaped"]
        n_esc += so["n_escaped"]
        fo, co = o.spectrum()
        fb, cb = be.spectrum(m)
        assert np.array_equal(cb, co)
        assert _rel(fb, fo) <= oracle_lib.TALLY_RTOL
        _same_tallies(be.tallies(m), o.tallies())
        Oo, Ob = o.opacity(), be.opacity(m)
        for k in ("abs", "scat"):
            assert _rel(Ob[k], Oo[k]) <= 1e-12, k
        o.close()
    assert st["n_escaped"] == n_esc


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_graph_steps_match_separate_contexts(sed_lib, precision):
    bw = small_batch(seed=11)
    if precision == abi.PREC_MIXED:  # steady-state luminosity rescale per model
        for w in bw.models:
            w.params["core_fix_luminosity"] = 1
    be = BatchEngine(bw, precision=precision, graph=True)
    be.record(True)
    singles = []
    for w in bw.models:
        g = oracle_lib.Engine(sed_lib, "sed_", w, precision=precision)
        g.record(True)
        singles.append(g)
    for step in range(3):  # step 0 eager, steps 1 and 2 graph replays
        sb = be.step(1.0)
        assert sb["ms_propagate_kernel"] > 0 and sb["ms_total"] >= sb["ms_propagate_kernel"]
        esc = be.escaped()
        for m, (w, g) in enumerate(zip(bw.models, singles)):
            g.set_opacity(1.0)
            sg = g.transport(1.0)
            n = w.n_packets
            _same_packets(be.records(m, n), g.records(n))
            assert esc[m] == sg["n_escaped"], (step, m)
            fs, cs = g.spectrum()
            fb, cb = be.spectrum(m)
            assert np.array_equal(cb, cs)
            assert _rel(fb, fs) <= oracle_lib.TALLY_RTOL
            _same_tallies(be.tallies(m), g.tallies())
            if step == 0:
                Os, Ob = g.opacity(), be.opacity(m)
                for k in ("abs", "scat", "emis_cdf", "n_elec", "eps_imc"):
                    assert np.array_equal(Ob[k], Os[k]), k
    for g in singles:
        g.close()


def test_autotuned_shapes_keep_every_packet(sed_lib):
    bw = small_batch(seed=5)
    ref = BatchEngine(bw, precision=abi.PREC_MIXED, graph=False)
    ref.record(True)
    ref.step(1.0)
    tuned = BatchEngine(bw, precision=abi.PREC_MIXED, graph=True)
    t = tuned.autotune(0.25)
    assert t["n_tried"] == 12 and t["threads"] in (128, 256) and t["queue_chunk"] in (1, 4, 16)
    tuned.record(True)
    tuned.step(1.0)
    forced = BatchEngine(bw, precision=abi.PREC_MIXED, graph=False)
    forced.set_tuning(variant=3, queue_chunk=16, blocks_per_sm=1)
    forced.record(True)
    forced.step(1.0)
    for m, w in enumerate(bw.models):
        r0 = ref.records(m, w.n_packets)
        for other in (tuned, forced):
            r1 = other.records(m, w.n_packets)
            for k in ("fate", "ind", "draws", "state"):
                assert np.array_equal(r0[k], r1[k]), (m, k)


def test_many_zone_batch_matches_separate_contexts(sed_lib):
    """More zones than the per-block shared-memory tallies hold (24 models,
    ~2600 zones): the zone-scalar tallies go to global copies that the finish
    kernel sums; every model still matches its own context."""
    bw = small_batch(n_models=24, zones=(90, 130), packets=(300, 800), seed=17)
    assert bw.n_zones * 5 * 8 > 64 * 1024
    be = BatchEngine(bw, precision=abi.PREC_FP64, graph=True)
    be.record(True)
    be.step(1.0)
    for m, w in enumerate(bw.models):
        g = oracle_lib.Engine(sed_lib, "sed_", w)
        g.set_opacity(1.0)
        g.record(True)
        g.transport(1.0)
        _same_packets(be.records(m, w.n_packets), g.records(w.n_packets))
        _same_tallies(be.tallies(m), g.tallies())
        fs, cs = g.spectrum()
        fb, cb = be.spectrum(m)
        assert np.array_equal(cb, cs)
        g.close()

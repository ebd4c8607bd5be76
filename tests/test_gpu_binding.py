"""The compiled C++ binding of the reference's transport class.

oracle/_ref/sedona_ref_gpu is the reference harness built (here, by
oracle/ref/build_ref.sh) from the reference's own sources together with
pubsed_b200/binding/transport_gpu.cpp and pubsed_b200/libsedona_gpu.so: it
runs transport::init on the workload's parameter and model files, then the
binding fills the C ABI's structs from that live transport (parameters,
grids, opacity switches, the atomic data the reference loaded), steps on the
device and copies the results back into the transport's own vectors, which
the harness dumps.  The same workload through the Python ctypes path must
give the same results: the same library on the same inputs, so a field the
binding fills differently from the reference's meaning shows up here.
"""
import os
import sys

import numpy as np
import pytest

from pubsed_b200 import abi, workloads
import oracle_lib

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
import run_ref  # noqa: E402


def _cases():
    return {
        "grey_radeq": workloads.lightbulb_grey(n_packets=20000, n_zones=32, n_bins=128, radiative_eq=1, seed=5),
        "ia_lte": workloads.type_ia(n_packets=4000, n_zones=16, n_lines=5000, n_bins=256, n_levels_per_ion=6,
                                    bound_free=1, free_free=1, seed=7),
    }


@pytest.mark.parametrize("case", ["grey_radeq", "ia_lte"])
@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_binding_step_matches_the_abi_path(sed_lib, case, precision):
    if not os.path.exists(run_ref.REF_GPU_BIN):
        pytest.fail("oracle/_ref/sedona_ref_gpu is not built (oracle/ref/build_ref.sh)")
    w = _cases()[case]
    out = run_ref.run(w, "gpu", precision=precision, steps=1)
    g = oracle_lib.Engine(sed_lib, "sed_", w, precision=precision)
    g.set_opacity(1.0)
    st = g.transport(1.0)
    f, c = g.spectrum()
    T = g.tallies()
    O = g.opacity()
    # the tables: within the FP64 parity tolerance (the binding passes the
    # atomic data the reference loaded, whose photoionisation tables its C++
    # loader computed, where the ctypes path passes the Python restatement of
    # that loader: the two round differently in the last bit); packets take
    # the same paths: equal counts; tallies are sums of FP64 atomics, whose
    # order varies from run to run: oracle_lib's tally tolerances
    for k in ("abs", "scat", "emis_cdf", "eps_imc", "planck_mean", "rosseland_mean"):
        a, b = out[k], O[k]
        assert np.all(np.abs(a - b) <= 1e-12 * np.maximum(np.abs(b), 1e-300)), k
    assert int(out["n_escaped_steps"][0]) == st["n_escaped"]
    assert np.array_equal(out["spec_click"], c)
    fin = c > 0
    assert np.all(np.abs(out["spec_flux"][fin] - f[fin]) <= oracle_lib.TALLY_RTOL * np.abs(f[fin]))
    for k, rk in (("J_nu", "J_nu"), ("e_abs", "e_abs"), ("e_rad", "e_rad"), ("fr", "fr_rad")):
        oracle_lib.zone_tally_close(out[rk], T[k])
    if int(w.params.get("transport_radiative_equilibrium", 0)):
        # Brent on tallies equal to ~1e-12 stops within its tolerance
        T_gpu, _ = oracle_lib.solve_temperature(g)
        assert np.allclose(out["T_gas"], T_gpu, rtol=1e-6, atol=0)
    g.close()

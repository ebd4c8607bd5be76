"""The text outputs against the reference's own (CPU): the oracle replays
the step of each golden case (its arrays equal the reference's to 1e-12,
tests/test_oracle_golden.py), pubsed_b200.output formats them, and the files
must be the reference's spectrum_array::print / grid_1D_sphere::
write_plotfile text byte for byte (the n_elec column of grey models excepted:
the reference never sets it there and prints whatever the memory held)."""
import json
import os

import numpy as np
import pytest

from pubsed_b200 import abi, output, workloads
import oracle_lib

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["replay_grey_absorb", "replay_grey_radeq", "replay_ia_lte", "replay_cart3d", "replay_ia_radio",
         "replay_ia_radio_late", "replay_core_file", "replay_core_derived"]


@pytest.mark.parametrize("name", CASES)
def test_text_outputs_match_reference(name, tmp_path):
    ref = np.load(os.path.join(GOLDEN, name + ".npz"))
    w = getattr(workloads, str(ref["generator"]))(**json.loads(str(ref["kwargs"])))
    e = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    e.set_opacity(1.0)
    e.transport(1.0)
    T = w.zones.T
    if int(w.params.get("transport_radiative_equilibrium", 0)):
        T, _ = oracle_lib.solve_temperature(e)
    flux, click = e.spectrum()
    tg, ng, mg, pg = w.spectrum_grids()
    path = output.write_spectrum_dat(str(tmp_path / "spec"), flux, click, tg, ng, mg, pg)
    assert open(path).read() == str(ref["spectrum_dat"])
    R = {}
    if "gamma_dat" in ref.files:  # binned on the optical spectrum's grids, as the reference does
        R = e.radioactive()
        path = output.write_spectrum_dat(str(tmp_path / "gamma"), R["gamma_flux"], R["gamma_click"], tg, ng, mg, pg)
        assert open(path).read() == str(ref["gamma_dat"])
    if "plt_dat" in ref.files:
        z = w.zones
        tal = e.tallies()
        n_elec = e.opacity()["n_elec"]
        p = output.write_plotfile_1d(str(tmp_path / "plt_00001.dat"), z.t_now, z.r_min, z.r_out, z.rho, z.v, T,
                                     tal["e_rad"], n_elec, L_dep=R.get("L_radio_dep"), L_emit=R.get("L_radio_emit"))
        mine = open(p).read().splitlines()
        theirs = str(ref["plt_dat"]).splitlines()
        assert len(mine) == len(theirs)
        assert mine[:2] == theirs[:2]
        grey = float(w.params.get("opacity_grey_opacity", 0)) != 0
        for a, b in zip(mine[2:], theirs[2:]):
            ca, cb = a.split("  "), b.split("  ")
            if grey:
                ca[5] = cb[5] = ""
            assert ca == cb, (a, b)
    e.close()


def test_mod_file_reader_round_trip(tmp_path):
    """read_mod_1d reads the SNR model files the reference harness is given."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "ref"))
    import run_ref
    w = workloads.type_ia(n_packets=10, n_zones=16, n_lines=100, n_bins=64)
    p = str(tmp_path / "m.mod")
    run_ref.write_mod_file(p, w.zones)
    z = workloads.read_mod_1d(p)
    for k in ("rho", "T", "vol"):
        assert np.array_equal(getattr(z, k), getattr(w.zones, k)), k
    # the reader normalises the mass fractions again, as the reference does
    assert np.allclose(z.X, w.zones.X, rtol=1e-15, atol=1e-16)
    assert np.allclose(z.r_out, w.zones.r_out, rtol=1e-15, atol=0)

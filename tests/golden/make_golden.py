"""Generates the golden fixtures in tests/golden/ from the reference itself.

Needs the reference harness built from the reference sources
(oracle/ref/build_ref.sh -> oracle/_ref/sedona_ref and
oracle/_ref/locate_array_test).  Each fixture records the workload that made
it (generator name and arguments) so tests can rebuild the same seeded
inputs, plus the reference's outputs:

  replay_*.npz   one transport step in replay mode (per-packet fate, final
                 zone, number of deviates drawn, final state; J_nu, e_abs,
                 e_rad, forces, spectrum; with a radioactive source the
                 gamma-ray spectrum and L_radio_emit / L_radio_dep; opacity
                 tables; the zone
                 temperatures after the step's radiative-equilibrium solve;
                 the reference's own spectrum .dat and, for 1D, plt .dat text)
  replay_td_*.npz  several time-dependent steps in replay mode: the initial
                 packets, and per step (suffix _s<k>) the per-packet results,
                 the census carried on, tallies and the accumulated spectrum
  locate_kat.json  value/index pairs printed by the reference's own
                 src/utils/locate_array_test.cpp

usage: python tests/golden/make_golden.py [fixture names ...]   (default: all)
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))

from pubsed_b200 import workloads  # noqa: E402
import run_ref  # noqa: E402

CASES = {
    "replay_grey_absorb": ("lightbulb_grey", dict(n_packets=1000, n_zones=32, n_bins=128, radiative_eq=0, seed=3)),
    "replay_grey_radeq": ("lightbulb_grey", dict(n_packets=600, n_zones=32, n_bins=128, radiative_eq=1, seed=5)),
    "replay_ia_lte": ("type_ia", dict(n_packets=300, n_zones=16, n_lines=5000, n_bins=256, n_levels_per_ion=6,
                                      bound_free=1, free_free=1, seed=7)),
    # 56Ni/56Co decay packets (gamma-rays and positrons) next to the core
    # packets; a small core so that most of the 56Ni sits outside it
    "replay_ia_radio": ("type_ia", dict(n_packets=200, n_zones=16, n_lines=5000, n_bins=256, n_levels_per_ion=6,
                                        v_core=1e8, n_radioactive=600, seed=19)),
    # the same ejecta at 150 days: thin enough that gamma-rays escape
    "replay_ia_radio_late": ("type_ia", dict(n_packets=100, n_zones=16, n_lines=5000, n_bins=256,
                                             n_levels_per_ion=6, v_core=1e8, n_radioactive=800, t_days=150.0,
                                             seed=23)),
    # the inner source's spectrum read from core_spectrum_file, its
    # luminosity the file's integral (core_luminosity = 0)
    "replay_core_file": ("with_params", dict(base="lightbulb_grey",
                                             params={"core_spectrum_file": "tests/golden/core_spectrum.txt",
                                                     "core_luminosity": 0.0},
                                             n_packets=800, n_zones=32, n_bins=128, seed=9)),
    # a core of radius 1e14 cm with core_temperature 0: T from L and r
    "replay_core_derived": ("with_params", dict(base="lightbulb_grey",
                                                params={"core_radius": 1e14, "core_temperature": 0.0,
                                                        "core_luminosity": 1e42},
                                                n_packets=800, n_zones=32, n_bins=128, seed=10)),
    "replay_cart3d": ("cart3d", dict(n_packets=300, n_cells=6, n_lines=1500, n_bins=128, spectrum_bins=64, n_mu=4,
                                     seed=13)),
}

# time-dependent replays: several steps with the census carried between them,
# the grid expanding homologously before each step, initial packets from the
# radiation field; every per-step array carries the suffix _s<step>
TD_CASES = {
    "replay_td_grey": ("time_dependent", dict(base="lightbulb_grey", n_initialize=300, dt_days=0.1, n_packets=200,
                                              n_zones=32, n_bins=128, radiative_eq=0, seed=3), 3),
    # gamma-rays and photons in flight at the end of each step
    "replay_td_ia_radio": ("time_dependent", dict(base="type_ia", n_initialize=200, dt_days=0.5, n_packets=100,
                                                  n_zones=16, n_lines=5000, n_bins=256, n_levels_per_ion=6,
                                                  v_core=1e8, n_radioactive=300, t_days=60.0, seed=29), 3),
    # discrete diffusion (transport_use_ddmc = 2) in the optically thick
    # zones and frequencies, Monte Carlo elsewhere, interfaces both ways
    "replay_td_ddmc_ia": ("time_dependent", dict(base="type_ia", n_initialize=200, dt_days=0.5,
                                                 params={"transport_use_ddmc": 2,
                                                         "transport_ddmc_tau_threshold": 3.0},
                                                 n_packets=100, n_zones=16, n_lines=5000, n_bins=256,
                                                 n_levels_per_ion=6, v_core=1e8, t_days=40.0, seed=31), 3),
    # grey, every zone diffusive; the initial radiation field only (a central
    # point source would put photons at r = 0, where the reference's
    # diffusion step divides by r)
    "replay_td_ddmc_grey": ("time_dependent", dict(base="lightbulb_grey", n_initialize=400, dt_days=0.1,
                                                   params={"transport_use_ddmc": 2,
                                                           "transport_ddmc_tau_threshold": 0.1},
                                                   n_packets=0, n_zones=32, n_bins=64, radiative_eq=1, seed=7), 3),
    # IMD (transport_use_ddmc = 1) on the same two configurations as DDMC:
    # every zone diffusive, and line opacity with diffusive and Monte Carlo
    # zones and frequencies
    "replay_td_imd_grey": ("time_dependent", dict(base="lightbulb_grey", n_initialize=400, dt_days=0.1,
                                                  params={"transport_use_ddmc": 1,
                                                          "transport_ddmc_tau_threshold": 0.1},
                                                  n_packets=0, n_zones=32, n_bins=64, radiative_eq=1, seed=41), 3),
    "replay_td_imd_ia": ("time_dependent", dict(base="type_ia", n_initialize=200, dt_days=0.5,
                                                params={"transport_use_ddmc": 1,
                                                        "transport_ddmc_tau_threshold": 3.0},
                                                n_packets=100, n_zones=16, n_lines=5000, n_bins=256,
                                                n_levels_per_ion=6, v_core=1e8, t_days=40.0, seed=43), 3),
    # particles_max_total below census + core packets on every other step:
    # those steps emit no core packets ("# Not enough particle space") and
    # propagate the census alone
    "replay_td_full": ("time_dependent", dict(base="lightbulb_grey", n_initialize=300, dt_days=0.1, n_packets=200,
                                              n_zones=32, n_bins=128, radiative_eq=0, seed=37,
                                              params={"particles_max_total": 450}), 4),
}
TD_KEYS = ["pkt_fate", "pkt_ind", "pkt_draws", "pkt_state", "pkt_type", "census_ind", "census_type", "census_state",
           "J_nu", "e_abs", "e_rad", "fr_rad", "spec_flux", "spec_click", "T_gas"]
TD_RADIO_KEYS = ["L_radio_emit", "L_radio_dep", "gamma_flux", "gamma_click"]

FREE_CASES = {
    "free_grey_radeq": ("lightbulb_grey", dict(n_packets=200000, n_zones=128, n_bins=256, radiative_eq=1, seed=101)),
    "free_ia": ("type_ia", dict(n_packets=60000, n_zones=64, n_lines=50000, n_bins=1024, seed=103)),
    "free_cart3d": ("cart3d", dict(n_packets=100000, n_cells=16, n_lines=10000, n_bins=512, spectrum_bins=128,
                                   n_mu=16, seed=109)),
    # absorption final, lines almost pure scattering: the configuration of the
    # differentiable (weighted) transport
    "free_ia_absorb": ("type_ia", dict(n_packets=150000, n_zones=64, n_lines=50000, n_bins=1024, spectrum_bins=256,
                                       epsilon=1e-4, radiative_eq=0, seed=107)),
}

KEYS = ["pkt_fate", "pkt_ind", "pkt_draws", "pkt_state", "J_nu", "e_abs", "e_rad", "fx_rad", "fy_rad", "fz_rad",
        "fr_rad", "spec_flux", "spec_click", "abs", "scat", "emis_cdf", "n_elec", "eps_imc", "planck_mean",
        "rosseland_mean", "L_thermal", "nu_right", "nu_left", "T_gas"]


def make_workload(gen: str, kw: dict):
    return getattr(workloads, gen)(**kw)


def write_core_spectrum():
    """A synthetic inner-source spectrum for replay_core_file: L_nu of a
    broken power law on 60 log-spaced frequencies inside the grid, one pair
    per line, the file ending in a newline (the reference then reads the last
    pair twice)."""
    nu = np.logspace(14.05, 15.9, 60)
    L = np.where(nu < 6e14, 1e28 * (nu / 6e14) ** 2, 1e28 * (nu / 6e14) ** -3)
    with open(os.path.join(HERE, "core_spectrum.txt"), "w") as f:
        for a, b in zip(nu, L):
            f.write("%.6e %.6e\n" % (a, b))


def main():
    if not run_ref.available():
        raise SystemExit("build the reference harness first: oracle/ref/build_ref.sh")
    only = set(sys.argv[1:])
    if not only or "replay_core_file" in only:
        write_core_spectrum()
    for name, (gen, kw) in CASES.items():
        if only and name not in only:
            continue
        w = make_workload(gen, kw)
        out = run_ref.run(w, "replay", threads=1, seed=kw.get("seed", 0))
        arrays = {k: out[k] for k in KEYS}
        for k in ("L_radio_emit", "L_radio_dep", "gamma_flux", "gamma_click"):
            if k in out:
                arrays[k] = out[k]
        # with grey opacity the reference never sets zone n_elec: its dump is
        # whatever the memory held; the restatement has zeros there
        if float(w.params.get("opacity_grey_opacity", 0)) != 0:
            arrays["n_elec"] = np.zeros_like(arrays["n_elec"])
        # the reference's own text outputs of the step
        with open(os.path.join(out["_dir"], "out_spectrum.dat")) as f:
            arrays["spectrum_dat"] = np.array(f.read())
        gam = os.path.join(out["_dir"], "out_gamma.dat")
        if os.path.exists(gam):
            with open(gam) as f:
                arrays["gamma_dat"] = np.array(f.read())
        plt = os.path.join(out["_dir"], "plt_00001.dat")
        if os.path.exists(plt):
            with open(plt) as f:
                arrays["plt_dat"] = np.array(f.read())
        np.savez_compressed(os.path.join(HERE, name + ".npz"), generator=gen, kwargs=json.dumps(kw),
                            n_escaped=out["n_escaped"], **arrays)
        print(name, "packets", int(out["n_packets"]), "escaped", int(out["n_escaped"]))
    for name, (gen, kw, steps) in TD_CASES.items():
        if only and name not in only:
            continue
        w = make_workload(gen, kw)
        out = run_ref.run(w, "replay", threads=1, seed=kw.get("seed", 0), steps=steps, dt=w.notes["dt"])
        arrays = {}
        for k in ("init_ind", "init_type", "init_state"):
            if k in out:
                arrays[k] = out[k]
        for st in range(steps):
            for k in TD_KEYS + (TD_RADIO_KEYS if kw.get("n_radioactive") else []):
                arrays["%s_s%d" % (k, st)] = out["%s_s%d" % (k, st)]
            arrays["n_escaped_s%d" % st] = out["n_escaped_s%d" % st]
        np.savez_compressed(os.path.join(HERE, name + ".npz"), generator=gen, kwargs=json.dumps(kw), steps=steps,
                            **arrays)
        print(name, "steps", steps, "census", [int(arrays["census_ind_s%d" % i].size) for i in range(steps)])
    # free-running reference steps (its own transport::step, OpenMP, streams
    # independent of the per-packet replay streams) for the chi-squared tests
    for name, (gen, kw) in FREE_CASES.items():
        if only and name not in only:
            continue
        w = make_workload(gen, kw)
        out = run_ref.run(w, "free", threads=os.cpu_count() or 1, seed=kw.get("seed", 0))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), generator=gen, kwargs=json.dumps(kw),
                            spec_flux=out["spec_flux"], spec_click=out["spec_click"], e_rad=out["e_rad"],
                            e_abs=out["e_abs"])
        print(name, "clicks", int(out["spec_click"].sum()))
    # locate_array_test: stderr holds "value index" lines, one block of 8
    # values per grid; the first block (20 zero walls, uninitialised minimum)
    # is skipped
    if only and "locate_kat" not in only:
        return
    exe = os.path.join(ROOT, "oracle", "_ref", "locate_array_test")
    r = subprocess.run([exe], capture_output=True, text=True, check=True)
    pairs = [ln.split() for ln in r.stderr.strip().splitlines()]
    with open(os.path.join(HERE, "locate_kat.json"), "w") as f:
        json.dump({"source": "src/utils/locate_array_test.cpp", "pairs": pairs}, f, indent=0)
    print("locate pairs", len(pairs))


if __name__ == "__main__":
    main()

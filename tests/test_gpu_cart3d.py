"""3D Cartesian grid (grid_3D_cart) on the GPU: parity with the reference's
own replayed step, with the oracle on a non-cubic grid with uneven walls,
the line-expansion opacity in both precisions, and the chunked opacity build.

Criteria as for the 1D paths: integer packet histories identical, final
states by oracle_lib.check_states, tallies within oracle_lib.TALLY_RTOL /
ZONE_TALLY_RTOL, FP64 tables 1e-12 and FP32 tables 1e-5 relative.
"""
import json
import os

import numpy as np
import pytest

from pubsed_b200 import abi, workloads
from pubsed_b200.grids import LocGrid, log_delta_for_bins
import oracle_lib

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rel(a, b, floor=1e-300):
    fin = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), fin)
    s = np.maximum(np.abs(b[fin]), floor)
    return float(np.max(np.abs(a[fin] - b[fin]) / s)) if s.size else 0.0


def _rel_ext(a, b, ext):
    """Error relative to the bin's total extinction (abs + scat).  A Sobolev
    line adds 1 - exp(-tau); for tau << 1 a last-bit difference between
    libm's and CUDA's exp is amplified by 1/tau, so bins whose absorption
    comes only from very weak lines (1e-28 cm^-1 next to 1e-12 cm^-1 of
    electron scattering) differ in relative terms while the extinction a
    packet sees agrees to rounding."""
    return float(np.max(np.abs(a - b) / np.maximum(ext, 1e-300)))


def test_cart3d_replay_matches_reference(sed_lib):
    ref = np.load(os.path.join(GOLDEN, "replay_cart3d.npz"))
    w = workloads.cart3d(**json.loads(str(ref["kwargs"])))
    g = oracle_lib.Engine(sed_lib, "sed_", w)
    g.set_opacity(1.0)
    O = g.opacity()
    assert _rel(O["n_elec"], ref["n_elec"]) <= 1e-12
    ext = ref["abs"] + ref["scat"]
    for k in ("abs", "scat"):
        assert _rel_ext(O[k], ref[k], ext) <= 1e-12, k
    assert _rel(O["emis_cdf"], ref["emis_cdf"]) <= 1e-12
    g.record(True)
    n = int(ref["pkt_fate"].size)
    st = g.transport(1.0)
    r = g.records(n)
    assert np.array_equal(r["fate"], ref["pkt_fate"])
    assert np.array_equal(r["ind"], ref["pkt_ind"])
    assert np.array_equal(r["draws"], ref["pkt_draws"])
    oracle_lib.check_states(r["state"], ref["pkt_state"].reshape(-1, 9))
    assert st["n_escaped"] == int(ref["n_escaped"])
    f, c = g.spectrum()
    assert np.array_equal(c, ref["spec_click"])
    assert _rel(f, ref["spec_flux"]) <= oracle_lib.TALLY_RTOL
    T = g.tallies()
    oracle_lib.zone_tally_close(T["J_nu"], ref["J_nu"])
    oracle_lib.zone_tally_close(T["e_abs"], ref["e_abs"])
    oracle_lib.zone_tally_close(T["e_rad"], ref["e_rad"])
    g.close()


def _uneven_axis(n, half, rng):
    w = rng.uniform(0.5, 1.5, n)
    edges = np.concatenate([[0.0], np.cumsum(w)])
    edges = (edges / edges[-1] * 2 - 1) * half
    return LocGrid(edges[1:].copy(), float(edges[0]), 0.0, abi.LOC_FLEX)


def grey_box(n_packets, shape=(5, 7, 4), seed=0, radiative_eq=1):
    """Grey 3D model on a non-cubic grid with uneven walls: lognormal density,
    kappa = 0.3 cm^2/g, epsilon = 0.5, central lightbulb of radius 0.1 W."""
    rng = np.random.default_rng(1234)
    t = 10 * 86400.0
    half = 1e9 * t
    axes = [_uneven_axis(n, half, rng) for n in shape]
    dx = [a.right - a.left() for a in axes]
    vol = (dx[0][:, None, None] * dx[1][None, :, None] * dx[2][None, None, :]).reshape(-1)
    nzn = int(np.prod(shape))
    rho = 3e-14 * np.exp(rng.normal(0, 0.5, nzn))
    zones = workloads.ZoneModel(type=abi.GRID_3D_CART, t_now=t, rho=rho, T=np.full(nzn, 1e4),
                                X=np.ones((nzn, 1)), elem_Z=np.array([1], np.int32),
                                elem_A=np.array([1], np.int32), vol=vol, axes=axes, shape=tuple(shape))
    d = log_delta_for_bins(1e14, 1e16, 256)
    params = {
        "grid_type": "grid_3D_cart", "hydro_module": "homologous",
        "transport_nu_grid": [1e14, 1e16, d, 1], "spectrum_nu_grid": [1e14, 1e16, d, 1],
        "spectrum_n_mu": 8, "spectrum_n_phi": 4,
        "transport_steady_iterate": 1, "transport_radiative_equilibrium": radiative_eq,
        "opacity_grey_opacity": 0.3, "opacity_epsilon": 0.5,
        "core_n_emit": int(n_packets), "core_radius": 0.1 * half, "core_temperature": 1e4,
        "core_luminosity": 1e43, "transport_fix_rng_seed": 1, "transport_rng_seed": int(seed),
        "particles_max_total": max(int(1e7), int(n_packets)),
    }
    return workloads.Workload("grey_box_3d", params, zones)


@pytest.mark.parametrize("radiative_eq", [0, 1])
def test_noncubic_grey_box_replay_matches_oracle(sed_lib, radiative_eq):
    n = 3000
    w = grey_box(n, seed=21 + radiative_eq, radiative_eq=radiative_eq)
    o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    g = oracle_lib.Engine(sed_lib, "sed_", w)
    for e in (o, g):
        e.set_opacity(1.0)
        e.record(True)
    so, sg = o.transport(1.0), g.transport(1.0)
    ro, rg = o.records(n), g.records(n)
    assert np.array_equal(ro["fate"], rg["fate"])
    assert np.array_equal(ro["ind"], rg["ind"])
    assert np.array_equal(ro["draws"], rg["draws"])
    oracle_lib.check_states(rg["state"], ro["state"])
    for k in ("n_escaped", "n_absorbed", "n_segments", "n_scatters"):
        assert so[k] == sg[k], k
    fo, co = o.spectrum()
    fg, cg = g.spectrum()
    assert np.array_equal(co, cg)
    assert _rel(fg, fo) <= oracle_lib.TALLY_RTOL
    To, Tg = o.tallies(), g.tallies()
    for k in ("J_nu", "e_abs", "e_rad", "fx", "fy", "fz"):
        oracle_lib.zone_tally_close(Tg[k], To[k])
    g.close()


def test_cart3d_line_expansion_replay_matches_oracle(sed_lib):
    n = 1500
    w = workloads.cart3d(n_packets=n, n_cells=10, n_lines=6000, n_bins=512, spectrum_bins=128, n_mu=16, seed=5)
    o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    g = oracle_lib.Engine(sed_lib, "sed_", w)
    for e in (o, g):
        e.set_opacity(1.0)
        e.record(True)
    Oo, Og = o.opacity(), g.opacity()
    ext = Oo["abs"] + Oo["scat"]
    for k in ("abs", "scat"):
        assert _rel_ext(Og[k], Oo[k], ext) <= 1e-12, k
    for k in ("n_elec", "emis_cdf", "planck_mean", "rosseland_mean", "L_thermal"):
        assert _rel(Og[k], Oo[k]) <= 1e-12, k
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
    oracle_lib.zone_tally_close(g.tallies()["J_nu"], o.tallies()["J_nu"])
    g.close()


def test_cart3d_mixed_tables_within_tolerance(sed_lib):
    w = workloads.cart3d(n_packets=10, n_cells=8, n_lines=20000, n_bins=1024, seed=6)
    o = oracle_lib.Engine(oracle_lib.oracle_lib(), "oracle_", w)
    g = oracle_lib.Engine(sed_lib, "sed_", w, precision=abi.PREC_MIXED)
    o.set_opacity(1.0)
    g.set_opacity(1.0)
    Oo, Og = o.opacity(), g.opacity()
    assert _rel(Og["n_elec"], Oo["n_elec"]) <= 1e-12
    # FP32 tables cannot hold the 1e-40 cm^-1 absorption floor of bins
    # without lines (1e-20 epsilon times electron scattering): absorption
    # is compared against the bin's total extinction, scattering per entry
    assert _rel_ext(Og["abs"], Oo["abs"], Oo["abs"] + Oo["scat"]) <= 1e-5
    assert _rel(Og["scat"], Oo["scat"]) <= 1e-5
    g.close()


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_MIXED])
def test_chunked_opacity_build_is_identical(sed_lib, precision, monkeypatch):
    """The opacity build in passes over chunks of zones (here 9^3 zones in
    chunks of ~70, the last one ragged) gives bit-identical tables to the
    single-pass build."""
    w = workloads.cart3d(n_packets=10, n_cells=9, n_lines=3000, n_bins=256, seed=8)
    monkeypatch.delenv("SEDONA_GPU_OPACITY_SCRATCH_BYTES", raising=False)
    one = oracle_lib.Engine(sed_lib, "sed_", w, precision=precision)
    one.set_opacity(1.0)
    A = one.opacity()
    one.close()
    nl = sum(a.lev_ion.size for a in w.atoms.atoms)
    ni = sum(a.n_ions for a in w.atoms.atoms)
    per_zone = (3 * 256 + 2 * 6 + 2 * ni + 2 * nl) * 8
    monkeypatch.setenv("SEDONA_GPU_OPACITY_SCRATCH_BYTES", str(70 * per_zone))
    many = oracle_lib.Engine(sed_lib, "sed_", w, precision=precision)
    many.set_opacity(1.0)
    B = many.opacity()
    st = many.transport(1.0)
    many.close()
    for k in A:
        assert np.array_equal(A[k], B[k]), k
    assert st["n_escaped"] == 10

"""Synthetic ejecta workloads (seeded) with the shapes of the benchmark
configurations, plus their translation into the C ABI structs.

A Workload holds Sedona parameters under their reference names (`params`),
a zone model (`zones`) and, for microphysical opacities, an atomic model.
Everything derived from them (bin walls, zone volumes, mass fractions) is
computed with the reference's own formulas so the CUDA library, the oracle
and the reference harness all see identical inputs.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Any, Optional

import numpy as np

from . import abi
from .atomic import AtomicModel, add_fuzz_lines, synthetic_atoms
from .grids import LocGrid, PI, grid_from_spec, lin_grid, lin_grid_n, log_delta_for_bins, shell_volumes
from .params import Params

M_SUN = 1.98892e33  # physical_constants::m_sun


@dataclass
class ZoneModel:
    """Zone geometry + gas state (grid_1D_sphere / grid_3D_cart + zone)."""
    type: int
    t_now: float
    rho: np.ndarray
    T: np.ndarray
    X: np.ndarray            # [n_zones, n_elems], normalised like the model readers
    elem_Z: np.ndarray
    elem_A: np.ndarray
    vol: np.ndarray
    homologous: int = 1
    # 1D sphere
    r_min: float = 0.0
    r_out: Optional[np.ndarray] = None
    v: Optional[np.ndarray] = None
    # 3D Cartesian
    axes: Optional[list] = None  # [LocGrid x, y, z]
    shape: Optional[tuple] = None

    @property
    def n_zones(self) -> int:
        return int(self.rho.size)

    @property
    def n_elems(self) -> int:
        return int(self.elem_Z.size)


@dataclass
class Workload:
    name: str
    params: dict[str, Any]
    zones: ZoneModel
    atoms: Optional[AtomicModel] = None
    notes: dict[str, Any] = field(default_factory=dict)

    # ------------------------------------------------------------ derived
    @property
    def P(self) -> Params:
        return Params(self.params)

    def nu_grid(self) -> LocGrid:
        return grid_from_spec(self.P.vector("transport_nu_grid"))

    def spectrum_grids(self):
        P = self.P
        t = P.vector("spectrum_time_grid")
        tg = lin_grid(float(t[0]), float(t[1]), float(t[2]))          # spectrum_array.cpp:40-43
        ng = grid_from_spec(P.vector("spectrum_nu_grid"))
        mg = lin_grid_n(-1.0, 1.0, P.scalar("spectrum_n_mu", int))      # :66
        pg = lin_grid_n(0.0, 2 * PI, P.scalar("spectrum_n_phi", int))   # :69
        return tg, ng, mg, pg

    @property
    def n_packets(self) -> int:
        return int(self.P.scalar("core_n_emit", int))

    def total_grey(self) -> np.ndarray:
        return np.full(self.zones.n_zones, float(self.P.scalar("opacity_grey_opacity")))

    # ------------------------------------------------------------ C structs
    def transport_params(self, keep: abi.Keep, precision: int = abi.PREC_FP64,
                         n_packets: Optional[int] = None) -> abi.TransportParams:
        P = self.P
        tg, ng, mg, pg = self.spectrum_grids()
        tp = abi.TransportParams()
        tp.steady_state = int(P.scalar("transport_steady_iterate", int) > 0)
        tp.radiative_eq = P.scalar("transport_radiative_equilibrium", int)
        tp.boundary_in_reflect = P.scalar("transport_boundary_in_reflect", int)
        tp.boundary_out_reflect = P.scalar("transport_boundary_out_reflect", int)
        tp.store_Jnu = P.scalar("transport_store_Jnu", int)
        tp.omit_scattering = P.scalar("opacity_no_scattering", int)
        tp.core_fix_luminosity = P.scalar("core_fix_luminosity", int)
        tp.tally_forces = 1
        tp.precision = precision
        tp.rng_seed = P.scalar("transport_rng_seed", int) & 0xFFFFFFFF
        tp.max_particles = P.scalar("particles_max_total", int)
        tp.core_n_emit = self.n_packets if n_packets is None else int(n_packets)
        tp.core_radius = P.scalar("core_radius")
        T_core, L_core, _ = self.core_source()
        tp.core_luminosity = L_core
        tp.core_temperature = T_core
        tp.core_photon_frequency = P.scalar("core_photon_frequency")
        tp.fleck_alpha = P.scalar("transport_fleck_alpha")
        tp.max_segments = P.scalar("gpu_max_segments", int)
        tp.nu_grid = abi.locate_grid(keep, self.nu_grid())
        tp.spec_time = abi.locate_grid(keep, tg)
        tp.spec_nu = abi.locate_grid(keep, ng)
        tp.spec_mu = abi.locate_grid(keep, mg)
        tp.spec_phi = abi.locate_grid(keep, pg)
        # radioactive source (emit_radioactive).  The reference reads
        # gamma_nu_grid but builds the gamma-ray spectrum on spectrum_nu_grid
        # (transport_init.cpp:170-173), so MeV energies land in the first bin
        # (spectrum_array::count keeps off-grid energies there); the same grid
        # is passed here
        tp.n_emit_radioactive = int(P.scalar("particles_n_emit_radioactive", int))
        tp.force_rprocess_heating = int(P.scalar("force_rprocess_heating", int))
        tp.gamma_nu = abi.locate_grid(keep, ng)
        # discrete diffusion (transport_init.cpp:336-341)
        tp.use_ddmc = int(P.scalar("transport_use_ddmc", int))
        tp.ddmc_tau = float(P.scalar("transport_ddmc_tau_threshold")) if tp.use_ddmc else 0.0
        return tp

    def core_source(self):
        """transport::setup_core_emission (src/transport/transport_init.cpp:
        465-547) and the luminosity emit_inner_source takes (emission.cpp:
        386-388): T_core from L and r_core when it is 0; the per-bin emission
        weights (a blackbody at T_core, or L_nu read from core_spectrum_file),
        and L = core_luminosity at the grid time, or, when that is 0, the
        spectrum's luminosity (sum over bins of 4 pi r_core^2 pi B_nu dnu, or
        of L_nu dnu).  Returns (T_core, L, weights) with weights None for the
        blackbody, which the library forms itself."""
        P = self.P
        r_core = P.scalar("core_radius")
        T_core = P.scalar("core_temperature")
        L0 = P.function("core_luminosity", 0.0)
        if L0 != 0 and r_core != 0 and T_core == 0:
            T_core = (L0 / (4.0 * PI * r_core * r_core * SB_CGS)) ** 0.25
        L = P.function("core_luminosity", self.zones.t_now)
        if P.scalar("core_n_emit", int) <= 0:  # no emission spectrum is set up then (:481)
            return T_core, (L if L != 0 else L0), None
        g = self.nu_grid()
        path = P.get("core_spectrum_file")
        weights, L_sum = None, 0.0
        cspec = read_core_spectrum(path) if path else None
        if cspec is not None:
            weights = np.zeros(g.n)
            for j in range(g.n):
                nu, dnu = g.center_at(j), g.delta_at(j)
                ind = _lower_bound(cspec[0], nu) - 1
                Lnu = 0.0 if (ind < 0 or ind >= len(cspec[0]) - 1) else cspec[1][ind]
                weights[j] = Lnu * dnu * 1.0
                L_sum += Lnu * dnu
        else:
            for j in range(g.n):
                nu, dnu = g.center_at(j), g.delta_at(j)
                if T_core <= 0:
                    bb = 1.0
                else:
                    bb = 2.0 * nu * nu * nu * H_CGS / C_CGS / C_CGS / (math.exp(H_CGS * nu / K_CGS / T_core) - 1)
                L_sum += 4.0 * PI * r_core * r_core * PI * bb * dnu
        if L == 0:
            L = L0 if L0 != 0 else L_sum
        return T_core, L, weights

    def grid_struct(self, keep: abi.Keep) -> abi.Grid:
        z = self.zones
        g = abi.Grid()
        g.type = z.type
        g.n_zones = z.n_zones
        g.homologous = z.homologous
        g.n_elems = z.n_elems
        g.t_now = z.t_now
        if z.type == abi.GRID_1D_SPHERE:
            g.r_min = z.r_min
            g.r_out = keep.d(z.r_out)
            g.v_r = keep.d(z.v if z.v is not None else np.zeros(z.n_zones))
        else:
            g.nx, g.ny, g.nz = z.shape
            g.x_axis = abi.locate_grid(keep, z.axes[0])
            g.y_axis = abi.locate_grid(keep, z.axes[1])
            g.z_axis = abi.locate_grid(keep, z.axes[2])
        g.vol = keep.d(z.vol)
        g.rho = keep.d(z.rho)
        g.T_gas = keep.d(z.T)
        g.e_gas = keep.d(np.zeros(z.n_zones))
        g.total_grey_opacity = keep.d(self.total_grey())
        g.X = keep.d(z.X.reshape(-1))
        g.elem_Z = keep.i(z.elem_Z)
        g.elem_A = keep.i(z.elem_A)
        return g

    def opacity_params(self, keep: abi.Keep) -> abi.OpacityParams:
        P = self.P
        op = abi.OpacityParams()
        op.use_electron_scattering = P.scalar("opacity_electron_scattering", int)
        op.use_free_free = P.scalar("opacity_free_free", int)
        op.use_bound_free = P.scalar("opacity_bound_free", int)
        op.use_line_expansion = P.scalar("opacity_line_expansion", int)
        op.use_fuzz_expansion = P.scalar("opacity_fuzz_expansion", int)
        ze = [int(v) for v in P.vector("opacity_atom_zero_epsilon")]
        op.n_atom_zero_epsilon = len(ze)
        op.atom_zero_epsilon = keep.i(np.array(ze, dtype=np.int32)) if ze else None
        op.epsilon = P.scalar("opacity_epsilon")
        op.maximum_opacity = P.scalar("opacity_maximum_opacity")
        op.temp_min = P.scalar("limits_temp_min")
        op.temp_max = P.scalar("limits_temp_max")
        op.line_velocity_width = P.scalar("line_velocity_width")
        return op

    def atomic_struct(self, keep: abi.Keep) -> Optional[abi.AtomicData]:
        if self.atoms is None:
            return None
        return self.atoms.to_struct(keep, self.nu_grid())


# ---------------------------------------------------------------- 1D models
def sphere_model(v_edges: np.ndarray, t_now: float, rho: np.ndarray, T: np.ndarray,
                 X: np.ndarray, elem_Z, elem_A, r_min: float = 0.0) -> ZoneModel:
    """A 1D_sphere "SNR" model: r_out = v t (grid_1D_sphere.cpp:318-324);
    mass fractions normalised per zone as the reader does (:335-351)."""
    v = np.asarray(v_edges, dtype=np.float64)
    r_out = np.array([vi * t_now for vi in v], dtype=np.float64)
    X = np.asarray(X, dtype=np.float64).reshape(v.size, -1)
    Xn = np.empty_like(X)
    for i in range(X.shape[0]):
        norm = 0.0
        for k in range(X.shape[1]):
            norm += X[i, k]
        for k in range(X.shape[1]):
            Xn[i, k] = X[i, k] / norm
    return ZoneModel(type=abi.GRID_1D_SPHERE, t_now=float(t_now), rho=np.asarray(rho, np.float64),
                     T=np.asarray(T, np.float64), X=Xn,
                     elem_Z=np.asarray(elem_Z, np.int32), elem_A=np.asarray(elem_A, np.int32),
                     vol=shell_volumes(r_min, r_out), r_min=float(r_min), r_out=r_out, v=v)


def lightbulb_grey(n_packets: int = 1_000_000, n_zones: int = 128, n_bins: int = 1024,
                   radiative_eq: int = 0, seed: int = 0) -> Workload:
    """Plain method, small: 1D homologous sphere at t = 10 d, 128 zones to
    v_max = 1e9 cm/s, rho = 1e-13 g/cm^3, grey kappa = 0.1 cm^2/g with
    epsilon = 0.1, central 1e4 K blackbody lightbulb, 1024 log bins
    1e14..1e16 Hz, FP64 throughout."""
    t = 10 * 86400.0
    v = np.array([(i + 1) * 1e9 / n_zones for i in range(n_zones)])
    z = sphere_model(v, t, np.full(n_zones, 1e-13), np.full(n_zones, 1e4),
                     np.ones((n_zones, 1)), [1], [1])
    d = log_delta_for_bins(1e14, 1e16, n_bins)
    grid = [1e14, 1e16, d, 1]
    params = {
        "grid_type": "grid_1D_sphere", "hydro_module": "homologous",
        "transport_nu_grid": grid, "spectrum_nu_grid": grid,
        "transport_steady_iterate": 1, "transport_radiative_equilibrium": radiative_eq,
        "opacity_grey_opacity": 0.1, "opacity_epsilon": 0.1,
        "core_n_emit": int(n_packets), "core_radius": 0.0, "core_temperature": 1e4,
        "core_luminosity": 1e43,
        "transport_fix_rng_seed": 1, "transport_rng_seed": int(seed),
        "particles_max_total": max(int(1e7), int(n_packets)),
    }
    return Workload("lightbulb_grey_1d", params, z,
                    notes={"log_del": d, "v_max": 1e9, "t_days": 10.0})


H_CGS, K_CGS, C_CGS, SB_CGS = 6.6260755e-27, 1.380658e-16, 2.99792458e10, 5.6704e-5  # physical_constants.h


def _lower_bound(a, v) -> int:
    """std::lower_bound's binary search, step for step (the result on an
    unsorted list is the reference's too)."""
    first, n = 0, len(a)
    while n > 0:
        half = n >> 1
        if a[first + half] < v:
            first += half + 1
            n -= half + 1
        else:
            n = half
    return first


def read_core_spectrum(path: str):
    """The (nu, L_nu) pairs setup_core_emission reads from core_spectrum_file
    (transport_init.cpp:488-501), as its stream loop reads them: pairs while
    the stream is not at its end, where a read that finds the end leaves its
    variable as it was.  So a file that ends in whitespace yields the last
    pair twice, and an odd token count repeats the previous L_nu.  An
    unreadable file reads as no file (None)."""
    try:
        with open(path) as f:
            data = f.read()
    except OSError:
        return None
    toks = data.split()
    n = len(toks)
    trailing = n > 0 and data[-1].isspace()
    nus, Ls = [], []
    i, eof = 0, False
    x1 = x2 = None
    while not eof:
        failed = False
        if i < n:
            x1 = float(toks[i]); i += 1
            if i == n and not trailing:
                eof = True
        else:
            eof = failed = True
        if not (failed or eof):
            if i < n:
                x2 = float(toks[i]); i += 1
                if i == n and not trailing:
                    eof = True
            else:
                eof = True
        if x1 is None or x2 is None:
            raise ValueError("core_spectrum_file %s holds no (nu, L_nu) pair" % path)
        nus.append(x1)
        Ls.append(x2)
    return nus, Ls


def with_params(base: str, params: dict, **kw) -> Workload:
    """The workload `base(**kw)` with `params` set over its parameters; a
    relative core_spectrum_file is taken from the repository root."""
    w = globals()[base](**kw)
    p = dict(params)
    f = p.get("core_spectrum_file")
    if f and not os.path.isabs(f):
        p["core_spectrum_file"] = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), f)
    w.params.update(p)
    return w


def time_dependent(base: str, n_initialize: int = 0, dt_days: float = 0.1, params: Optional[dict] = None,
                   **kw) -> Workload:
    """The workload `base(**kw)` run time-dependently
    (transport_steady_iterate = 0): packets that reach the end of a step are
    carried to the next, the grid expands homologously between steps
    (`homologous_step`), and particles_n_initialize packets of the initial
    radiation field (e_rad = a T^4) start in the census; `params` are set
    last, over the base's parameters and these.  notes["dt"] is the step (dt_days)."""
    w = globals()[base](**kw)
    w.params["transport_steady_iterate"] = 0
    w.params["particles_n_initialize"] = int(n_initialize)
    w.params["particles_max_total"] = max(int(w.params.get("particles_max_total", 1e7)), 4 * int(n_initialize) + 1)
    w.params.update(params or {})
    w.name = w.name + "_td"
    w.notes["dt"] = dt_days * 86400.0
    return w


def diffusing_pulse(n_initialize: int = 100_000, seed: int = 0, method: int = 2) -> Workload:
    """The reference's diffusing-pulse test (tests/diffusing_pulse/1D_ddmc;
    model from tests/diffusing_pulse/models/make_mod.py): a static 1D sphere
    ("standard" model, v = 0, hydro "none"), 200 zones of 0.5 cm out to
    100 cm, rho = 1 g/cm^3, T = 1e4 K inside r < 5 cm and 0 outside, one
    species 1.1, grey opacity 1 cm^2/g with epsilon = 0 (pure scattering),
    one frequency bin, 1e5 packets of the initial radiation field and no
    other source; discrete diffusion (method 2) above zone optical depth
    0.1; steps of at most 5e-10 s growing by at most 10% of the time (the
    default tstep_max_delta: the test's own "tstel_max_delta" is a typo the
    defaults shadow) to 1e-8 s, plot files every 5e-10 s.  Its check: at the
    6th, 12th and 18th plot file T_rad within 10% (mean) of the diffusion
    solution of a pulse at r0 = 2.5 cm with D = c / (3 rho kappa)."""
    n, dr = 200, 1.0e2 / 200
    r_out = np.array([(i + 1) * dr for i in range(n)])
    T = np.array([1e4 if (i + 1) * dr < 5.0 else 0.0 for i in range(n)])
    z = ZoneModel(type=abi.GRID_1D_SPHERE, t_now=0.0, rho=np.ones(n), T=T, X=np.ones((n, 1)),
                  elem_Z=np.array([1], np.int32), elem_A=np.array([1], np.int32), vol=shell_volumes(0.0, r_out),
                  homologous=0, r_min=0.0, r_out=r_out, v=np.zeros(n))
    params = {
        "grid_type": "grid_1D_sphere", "hydro_module": "none",
        "tstep_max_steps": 1000, "tstep_time_stop": 1e-8, "tstep_max_dt": 5e-10, "tstep_min_dt": 0.0,
        "particles_n_initialize": int(n_initialize), "transport_use_ddmc": int(method),
        "transport_ddmc_tau_threshold": 0.1, "transport_steady_iterate": 0,
        "opacity_grey_opacity": 1.0, "opacity_epsilon": 0.0,
        "output_write_plt_file_time": 5e-10, "spectrum_time_grid": [0, 1e-9, 1e-7],
        "transport_fix_rng_seed": 1, "transport_rng_seed": int(seed),
        "particles_max_total": 4 * int(n_initialize),
    }
    return Workload("diffusing_pulse_1d", params, z, notes={"r0": 2.5, "rho": 1.0, "kappa": 1.0})


def initial_e_rad(zones: ZoneModel) -> np.ndarray:
    """Zone radiation energy density of a model without an erad column:
    a T_gas^4 (grid_1D_sphere.cpp:354, :130)."""
    return A_RAD_CGS * np.power(zones.T, 4.0)


def homologous_step(zones: ZoneModel, dt: float) -> None:
    """hydro_homologous::step (src/hydro/hydro_homologous.cpp:27-45) on a 1D
    sphere: e = (t + dt) / t, rho /= e^3, walls and r_min scaled by e
    (locate_array::scale), shell volumes recomputed (grid_1D_sphere::expand,
    :413-426), t += dt; the reference's operations in its order."""
    if zones.type != abi.GRID_1D_SPHERE:
        raise ValueError("homologous_step: 1D spheres only")
    e = (zones.t_now + dt) / zones.t_now
    zones.rho = zones.rho / e / e / e
    zones.r_out = zones.r_out * e
    zones.r_min = zones.r_min * e
    zones.vol = shell_volumes(zones.r_min, zones.r_out)
    zones.t_now = zones.t_now + dt


A_RAD_CGS = 7.5657e-15  # physical_constants::a


# Type Ia-like layered composition: (Z, A) and mass fractions per layer
IA_ELEMENTS = [(6, 12), (8, 16), (14, 28), (16, 32), (20, 40), (28, 56)]
IA_LAYERS = [  # (v_upper cm/s, mass fractions in IA_ELEMENTS order)
    (4e8, [0.0, 0.0, 0.0, 0.0, 0.0, 1.0]),          # 56Ni
    (1.2e9, [0.0, 0.0, 0.6, 0.3, 0.1, 0.0]),        # Si/S/Ca
    (math.inf, [0.5, 0.5, 0.0, 0.0, 0.0, 0.0]),     # C/O
]


def type_ia(n_packets: int = 10_000_000, n_zones: int = 256, n_lines: int = 500_000, n_bins: int = 4096,
            n_levels_per_ion: int = 20, v_max: float = 3e9, epsilon: float = 1.0, seed: int = 0, data_seed: int = 0,
            bound_free: int = 0, free_free: int = 1, spectrum_bins: int = 1024,
            v_core: float = 1e9, radiative_eq: int = 1, n_radioactive: int = 0,
            t_days: float = 20.0) -> Workload:
    """Precision configuration: 1D Type Ia-like ejecta, 256 zones, 1.4 Msun,
    rho ~ exp(-v / 2.7e8 cm/s), t = 20 d, layered 56Ni / Si-S-Ca / C-O
    composition, T falling linearly from 1.2e4 K (inner) to 5e3 K (outer),
    LTE Saha-Boltzmann populations, 5e5 synthetic fuzz lines (lambda
    log-uniform 1000-30000 A, gf log-uniform 1e-4..1, El uniform 0-10 eV)
    binned into 4096 log frequency bins, electron scattering and free-free,
    a central 1.2e4 K lightbulb, radiative equilibrium (absorbed packets are
    re-emitted from the zone emissivity), steady-state iteration.
    n_radioactive > 0 adds that many 56Ni/56Co decay packets
    (particles_n_emit_radioactive) with gamma-ray transport; t_days moves
    the epoch (the ejecta thin out as t^-3, so gamma-rays escape late).

    Choices the configuration leaves open, fixed here: v_max = 3e9 cm/s;
    Si/S/Ca = 0.6/0.3/0.1 and C/O = 0.5/0.5 by mass; five ion stages per
    element with approximate real ionisation energies plus the bare stage,
    `n_levels_per_ion` levels per stage (E uniform in [0, 0.8 chi), odd g);
    each line's (element, stage) uniform over the 30 real stages; the
    lightbulb is an inner boundary (core_radius = v_core * t, v_core = 1e9
    cm/s, absorbing) radiating a 1.2e4 K blackbody with L = 1e43 erg/s;
    opacity_epsilon = 1 (absorptive lines, Sedona's default).  With this line
    list the ejecta are optically thick at every frequency; a central point
    source costs ~5e4 segments per packet, the inner boundary ~2e3.
    radiative_eq = 0 makes absorption final (the form the differentiable
    transport needs)."""
    rng = np.random.default_rng(data_seed)  # synthetic atoms and lines; `seed` keys the packets
    t = t_days * 86400.0
    v = np.array([(i + 1) * v_max / n_zones for i in range(n_zones)])
    vc = np.concatenate([[0.0], v[:-1]]) * 0.5 + v * 0.5
    Z = [e[0] for e in IA_ELEMENTS]
    A = [e[1] for e in IA_ELEMENTS]
    X = np.zeros((n_zones, len(Z)))
    for i in range(n_zones):
        for vu, frac in IA_LAYERS:
            if vc[i] < vu:
                X[i] = frac
                break
    T = np.array([1.2e4 + (5e3 - 1.2e4) * i / (n_zones - 1) for i in range(n_zones)])
    shape = np.exp(-vc / 2.7e8)
    z0 = sphere_model(v, t, shape, T, X, Z, A)
    rho0 = 1.4 * M_SUN / float(np.sum(shape * z0.vol))
    z = sphere_model(v, t, rho0 * shape, T, X, Z, A)
    atoms = synthetic_atoms(Z, n_levels_per_ion, 0, rng)
    add_fuzz_lines(atoms, n_lines, 1000.0, 30000.0, 1e-4, 1.0, 10.0, rng)
    d = log_delta_for_bins(1e14, 3e15, n_bins)
    ds = log_delta_for_bins(1e14, 3e15, spectrum_bins)
    params = {
        "grid_type": "grid_1D_sphere", "hydro_module": "homologous",
        "transport_nu_grid": [1e14, 3e15, d, 1], "spectrum_nu_grid": [1e14, 3e15, ds, 1],
        "transport_steady_iterate": 1, "transport_radiative_equilibrium": int(radiative_eq),
        "opacity_grey_opacity": 0, "opacity_epsilon": epsilon,
        "opacity_electron_scattering": 1, "opacity_fuzz_expansion": 1,
        "opacity_free_free": int(free_free), "opacity_bound_free": int(bound_free),
        "dont_decay_composition": 1,
        "core_n_emit": int(n_packets), "core_radius": float(v_core * t), "core_temperature": 1.2e4,
        "core_luminosity": 1e43,
        "transport_fix_rng_seed": 1, "transport_rng_seed": int(seed),
        "particles_max_total": max(int(1e7), int(n_packets) + int(n_radioactive)),
    }
    if n_radioactive > 0:
        params["particles_n_emit_radioactive"] = int(n_radioactive)
    return Workload("type_ia_1d", params, z, atoms,
                    notes={"v_max": v_max, "t_days": t_days, "rho0": rho0, "log_del": d,
                           "n_lines": n_lines, "n_levels_per_ion": n_levels_per_ion})


# ---------------------------------------------------------------- 3D models
def gaussian_random_field(n: int, corr_cells: float, rng: np.random.Generator) -> np.ndarray:
    """Unit-variance Gaussian random field on an n^3 periodic lattice: white
    noise filtered in Fourier space by exp(-k^2 l^2 / 2) (a Gaussian
    two-point correlation of length l = corr_cells), rescaled to zero mean
    and unit variance.  Indexed [i, j, k] = [x, y, z]."""
    w = rng.standard_normal((n, n, n))
    k = 2 * np.pi * np.fft.fftfreq(n)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    g = np.fft.ifftn(np.fft.fftn(w) * np.exp(-0.5 * k2 * corr_cells ** 2)).real
    g -= g.mean()
    return g / g.std()


def cart_axis(half_width: float, n: int) -> LocGrid:
    """Explicit cell walls -W + (i+1) 2W/n with minimum -W, as a model file's
    x_out/y_out/z_out + rmin give them (grid_3D_cart.cpp:88-131: a `flex`
    locate_array)."""
    from .abi import LOC_FLEX
    d = 2.0 * half_width / n
    right = np.array([-half_width + (i + 1) * d for i in range(n - 1)] + [half_width], dtype=np.float64)
    return LocGrid(right, -half_width, 0.0, LOC_FLEX)


def cart3d(n_packets: int = 100_000_000, n_cells: int = 128, n_lines: int = 100_000, n_bins: int = 2048,
           n_mu: int = 16, spectrum_bins: int = 1024, sigma: float = 0.5, corr_cells: float = 8.0,
           mass_msun: float = 1.4, v_max: float = 2e9, v_e: float = 2.7e8, t_days: float = 30.0,
           n_levels_per_ion: int = 30, epsilon: float = 1.0, v_core: float = 3e8, line_A_min: float = 1e-2,
           line_A_max: float = 1e2, seed: int = 0, data_seed: int = 0) -> Workload:
    """3D configuration: homologous ejecta on an n_cells^3 Cartesian grid
    spanning +-v_max t on each axis.  rho = rho0 exp(-|v|/v_e) times a
    lognormal clumping field exp(sigma G - sigma^2/2), G a unit-variance
    Gaussian random field with correlation length corr_cells cells (seeded);
    rho0 sets the mass on the grid to mass_msun.  Composition layered in |v|
    as in the 1D Type Ia-like model; T falls linearly in |v| from 1.2e4 K at
    the centre to 5e3 K at v_max (5e3 K beyond).  Opacity: electron
    scattering (the grey scattering term) plus the Sobolev line-expansion
    opacity of n_lines synthetic level-to-level lines (LTE populations),
    opacity_epsilon = epsilon, radiative equilibrium.  n_bins log frequency
    bins over 1e14-3e15 Hz; spectra in spectrum_bins log bins and n_mu
    viewing-angle bins (mu = D_z).  Source: a 1.2e4 K blackbody lightbulb of
    radius v_core t, L = 1e43 erg/s.

    Choices the configuration leaves open, fixed here: the ejecta
    parameters above; level energies below min(0.8 chi, 12 eV) so that
    transitions fall inside the frequency grid; each line's (element, stage)
    uniform over the real stages, its level pair uniform with the transition
    frequency inside the grid, A log-uniform in 1e-2..1e2 s^-1 (weak lines:
    with t = 30 d the median optical depth from the centre is ~5, so a packet
    takes a few hundred segments rather than the ~1e4 of saturated lines)."""
    from .atomic import add_level_lines
    rng = np.random.default_rng(data_seed)
    t = t_days * 86400.0
    W = v_max * t
    ax = cart_axis(W, n_cells)
    n = n_cells
    left = ax.left()
    dx = np.array([ax.right[i] - left[i] for i in range(n)])   # locate_array::delta
    c = 0.5 * (left + ax.right)
    x, y, zz = np.meshgrid(c, c, c, indexing="ij")
    vr = np.sqrt(x * x + y * y + zz * zz).reshape(-1) / t
    vol = (dx[:, None, None] * dx[None, :, None] * dx[None, None, :]).reshape(-1)
    G = gaussian_random_field(n, corr_cells, rng).reshape(-1)
    shape = np.exp(-vr / v_e) * np.exp(sigma * G - 0.5 * sigma * sigma)
    rho = mass_msun * M_SUN / float(np.sum(shape * vol)) * shape
    T = 1.2e4 + (5e3 - 1.2e4) * np.minimum(vr / v_max, 1.0)
    Z = [e[0] for e in IA_ELEMENTS]
    A = [e[1] for e in IA_ELEMENTS]
    X = np.zeros((rho.size, len(Z)))
    for vu, frac in reversed(IA_LAYERS):
        X[vr < vu] = frac
    zones = ZoneModel(type=abi.GRID_3D_CART, t_now=float(t), rho=rho, T=T, X=X,
                      elem_Z=np.asarray(Z, np.int32), elem_A=np.asarray(A, np.int32), vol=vol,
                      axes=[ax, ax, ax], shape=(n, n, n))
    atoms = synthetic_atoms(Z, n_levels_per_ion, 0, rng, E_max_eV=12.0)
    add_level_lines(atoms, n_lines, 1e14, 3e15, rng, line_A_min, line_A_max)
    d = log_delta_for_bins(1e14, 3e15, n_bins)
    ds = log_delta_for_bins(1e14, 3e15, spectrum_bins)
    params = {
        "grid_type": "grid_3D_cart", "hydro_module": "homologous",
        "transport_nu_grid": [1e14, 3e15, d, 1], "spectrum_nu_grid": [1e14, 3e15, ds, 1],
        "spectrum_n_mu": int(n_mu),
        "transport_steady_iterate": 1, "transport_radiative_equilibrium": 1,
        "opacity_grey_opacity": 0, "opacity_epsilon": epsilon,
        "opacity_electron_scattering": 1, "opacity_line_expansion": 1,
        "dont_decay_composition": 1,
        "core_n_emit": int(n_packets), "core_radius": float(v_core * t), "core_temperature": 1.2e4,
        "core_luminosity": 1e43,
        "transport_fix_rng_seed": 1, "transport_rng_seed": int(seed),
        "particles_max_total": max(int(1e7), int(n_packets)),
    }
    return Workload("cart3d", params, zones, atoms,
                    notes={"v_max": v_max, "t_days": t_days, "n_cells": n, "n_lines": n_lines,
                           "sigma": sigma, "corr_cells": corr_cells, "mass_msun": mass_msun, "v_e": v_e})


# ---------------------------------------------------------------- batches
@dataclass
class BatchWorkload:
    """Independent 1D models stepped as one batch.  Every model is a complete
    Workload (so it can also run on its own context); the models share the
    frequency and spectrum grids, transport and opacity switches, atomic data,
    element list and grid time, and differ in zones, core source, packet
    count and Philox key."""
    name: str
    models: list
    notes: dict[str, Any] = field(default_factory=dict)

    @property
    def n_packets(self) -> int:
        return int(sum(m.n_packets for m in self.models))

    @property
    def n_zones(self) -> int:
        return int(sum(m.zones.n_zones for m in self.models))


def batch_model(n_zones: int, n_packets: int, v_max: float, mass_msun: float, atoms: AtomicModel,
                seed: int, t_days: float = 20.0, v_e_frac: float = 0.125, v_core_frac: float = 0.25,
                T_core: float = 1.2e4, L_core: float = 1e43, n_bins: int = 2048, spectrum_bins: int = 1024,
                epsilon: float = 1.0) -> Workload:
    """One ejecta model of a batch: homologous 1D sphere of `n_zones` zones to
    v_max at t_days, rho = rho0 exp(-v / v_e) with v_e = v_e_frac v_max and
    rho0 set by mass_msun, Type Ia-like layers at fixed fractions of v_max
    (56Ni below 0.15, Si/S/Ca below 0.45, C/O beyond), T linear from 1.2e4 K
    to 5e3 K, electron scattering + free-free + fuzz line expansion from the
    shared `atoms`, radiative equilibrium, an absorbing inner boundary at
    v_core_frac v_max radiating a T_core blackbody of luminosity L_core."""
    t = t_days * 86400.0
    v = np.array([(i + 1) * v_max / n_zones for i in range(n_zones)])
    vc = np.concatenate([[0.0], v[:-1]]) * 0.5 + v * 0.5
    Z = [e[0] for e in IA_ELEMENTS]
    A = [e[1] for e in IA_ELEMENTS]
    X = np.zeros((n_zones, len(Z)))
    layers = [(0.15 * v_max, IA_LAYERS[0][1]), (0.45 * v_max, IA_LAYERS[1][1]), (math.inf, IA_LAYERS[2][1])]
    for i in range(n_zones):
        for vu, frac in layers:
            if vc[i] < vu:
                X[i] = frac
                break
    T = np.array([1.2e4 + (5e3 - 1.2e4) * i / max(n_zones - 1, 1) for i in range(n_zones)])
    shape = np.exp(-vc / (v_e_frac * v_max))
    z0 = sphere_model(v, t, shape, T, X, Z, A)
    rho0 = mass_msun * M_SUN / float(np.sum(shape * z0.vol))
    z = sphere_model(v, t, rho0 * shape, T, X, Z, A)
    d = log_delta_for_bins(1e14, 3e15, n_bins)
    ds = log_delta_for_bins(1e14, 3e15, spectrum_bins)
    params = {
        "grid_type": "grid_1D_sphere", "hydro_module": "homologous",
        "transport_nu_grid": [1e14, 3e15, d, 1], "spectrum_nu_grid": [1e14, 3e15, ds, 1],
        "transport_steady_iterate": 1, "transport_radiative_equilibrium": 1,
        "opacity_grey_opacity": 0, "opacity_epsilon": epsilon,
        "opacity_electron_scattering": 1, "opacity_fuzz_expansion": 1, "opacity_free_free": 1,
        "dont_decay_composition": 1,
        "core_n_emit": int(n_packets), "core_radius": float(v_core_frac * v_max * t),
        "core_temperature": float(T_core), "core_luminosity": float(L_core),
        "transport_fix_rng_seed": 1, "transport_rng_seed": int(seed),
        "particles_max_total": max(int(1e7), int(n_packets)),
    }
    return Workload("batch_model", params, z, atoms,
                    notes={"v_max": v_max, "t_days": t_days, "mass_msun": mass_msun, "n_lines": atoms.n_fuzz()})


def batch64(n_models: int = 64, zones: tuple = (64, 512), packets: tuple = (1e5, 1e7), v_max: tuple = (5e8, 2e9),
            mass_msun: tuple = (0.2, 1.0), n_lines: int = 30_000, n_bins: int = 2048, packet_scale: float = 1.0,
            n_levels_per_ion: int = 20, seed: int = 0, data_seed: int = 0) -> BatchWorkload:
    """Batching configuration: `n_models` independent 1D ejecta models, zone
    counts uniform in zones[0]..zones[1], packet counts log-uniform in
    packets[0]..packets[1] (times packet_scale), v_max uniform in
    v_max[0]..v_max[1] cm/s, each with a seeded exponential density (mass
    uniform in mass_msun) and electron-scattering + line opacity from one
    shared synthetic fuzz list of n_lines lines.  Model m uses Philox key
    seed + m.  Open choices fixed here: t = 20 d for every model (one grid
    time per batch), v_e = v_max / 8, layers and temperatures as in
    batch_model, core T uniform 1.0e4-1.5e4 K and L log-uniform 0.5e43-2e43
    erg/s, 3e4 lines (a model then costs ~300 segments per packet, most of
    them zone and frequency-bin crossings)."""
    rng = np.random.default_rng(data_seed)
    Z = [e[0] for e in IA_ELEMENTS]
    atoms = synthetic_atoms(Z, n_levels_per_ion, 0, rng)
    add_fuzz_lines(atoms, n_lines, 1000.0, 30000.0, 1e-4, 1.0, 10.0, rng)
    models = []
    for m in range(n_models):
        nz = int(rng.integers(zones[0], zones[1] + 1))
        npk = int(10 ** rng.uniform(math.log10(packets[0]), math.log10(packets[1])))
        npk = max(1, int(npk * packet_scale))
        vm = float(rng.uniform(v_max[0], v_max[1]))
        ms = float(rng.uniform(mass_msun[0], mass_msun[1]))
        Tc = float(rng.uniform(1.0e4, 1.5e4))
        Lc = float(10 ** rng.uniform(math.log10(0.5e43), math.log10(2e43)))
        models.append(batch_model(nz, npk, vm, ms, atoms, seed + m, T_core=Tc, L_core=Lc, n_bins=n_bins))
    return BatchWorkload("batch64_1d", models,
                         notes={"n_models": n_models, "n_lines": n_lines, "n_bins": n_bins,
                                "packet_scale": packet_scale})


# ---------------------------------------------------------------- model files
def read_mod_1d(path: str, grey_opacity: float = 0.0) -> ZoneModel:
    """A 1D_sphere ASCII model file (".mod"), as grid_1D_sphere::read_ascii_file
    reads it (src/grid/grid_1D_sphere.cpp:241-332): "1D_sphere <standard|SNR>",
    n_zones, r_min, t_exp, n_elems, the Z.A species, then per zone r_out (not
    in SNR files, where r_out = v t), v, rho, T_gas and the mass fractions,
    normalised per zone.  The zone velocities are kept for non-homologous
    runs (hydro_module "none")."""
    with open(path) as f:
        tok = f.read().split()
    if tok[0] != "1D_sphere":
        raise ValueError("grid type given in model file is not 1D_sphere")
    system = tok[1]
    if system not in ("standard", "SNR"):
        raise ValueError("don't recognize model type " + system)
    snr = system == "SNR"
    n = int(tok[2])
    r_min = float(tok[3])
    t = float(tok[4])
    ne = int(tok[5])
    species = tok[6:6 + ne]
    Z = [int(s.split(".")[0]) for s in species]
    A = [int(s.split(".")[1]) for s in species]
    p = 6 + ne
    cols = (3 if snr else 4) + ne
    vals = [float(x) for x in tok[p:p + n * cols]]
    if len(vals) != n * cols:
        raise ValueError("model file ends early")
    r_out, v, rho, T, X = [], [], [], [], []
    for i in range(n):
        row = vals[i * cols:(i + 1) * cols]
        if snr:
            v_i, rho_i, T_i = row[0], row[1], row[2]
            r_i = v_i * t
            xs = row[3:]
        else:
            r_i, v_i, rho_i, T_i = row[0], row[1], row[2], row[3]
            xs = row[4:]
        norm = 0.0
        for x in xs:
            norm += x
        r_out.append(r_i); v.append(v_i); rho.append(rho_i); T.append(T_i)
        X.append([x / norm for x in xs])
    r_out = np.array(r_out)
    return ZoneModel(type=abi.GRID_1D_SPHERE, t_now=t, rho=np.array(rho), T=np.array(T), X=np.array(X),
                     elem_Z=np.asarray(Z, np.int32), elem_A=np.asarray(A, np.int32),
                     vol=shell_volumes(r_min, r_out), homologous=1, r_min=r_min, r_out=r_out, v=np.array(v))


def lightbulb_vacuum(n_packets: int = 200_000, seed: int = 0) -> Workload:
    """The reference's spherical-lightbulb test (tests/spherical_lightbulb/1D):
    a static vacuum 1D sphere (100 zones, r_out = (i+1) 1.728e13 cm to five
    significant digits, v = 0,
    rho = 1e-20 g/cm^3, T = 2e5 K, one species 1.1, t = 20 d, hydro "none"),
    grey opacity 1e-10 cm^2/g, a 1e4 K lightbulb of radius 5e14 cm and
    L = 1e43 erg/s, log nu grid {0.2e14, 5e15, 0.01}, radiative equilibrium,
    one steady-state iteration.  Its analytic checks: T_gas and T_rad within
    1% of the dilution-factor temperature beyond 5e14 cm, the spectrum within
    10% (mean) of the core blackbody."""
    n = 100
    # the model file holds the radii to five significant digits
    r_out = np.array([float("%.4e" % ((i + 1) * 1.728e13)) for i in range(n)])
    z = ZoneModel(type=abi.GRID_1D_SPHERE, t_now=1728000.0, rho=np.full(n, 1e-20), T=np.full(n, 2e5),
                  X=np.ones((n, 1)), elem_Z=np.array([1], np.int32), elem_A=np.array([1], np.int32),
                  vol=shell_volumes(0.0, r_out), homologous=0, r_min=0.0, r_out=r_out, v=np.zeros(n))
    grid = [0.2e14, 5.0e15, 0.01, 1]
    params = {
        "grid_type": "grid_1D_sphere", "hydro_module": "none",
        "transport_nu_grid": grid, "spectrum_nu_grid": grid,
        "transport_radiative_equilibrium": 1, "transport_steady_iterate": 1,
        "core_n_emit": int(n_packets), "core_radius": 5.0e14, "core_luminosity": 1.0e43,
        "core_temperature": 1.0e4, "opacity_grey_opacity": 1e-10,
        "transport_fix_rng_seed": 1, "transport_rng_seed": int(seed),
    }
    return Workload("lightbulb_vacuum_1d", params, z, notes={"r0": 5.0e14, "T": 1e4, "L": 1e43})

"""Sedona's Lua parameter interface for the transport step.

`DEFAULTS` lists every parameter the transport, grid and opacity code read,
under the reference's names and with its default values (the reference
keeps them in defaults/sedona_defaults.lua and reads them through
ParameterReader, src/utils/ParameterReader.h:59-144).  Names and meanings
are an interface and are kept identical.

`read_param_file` evaluates the subset of Lua used by parameter files
(assignments of numbers, strings, tables, arithmetic, `..` concatenation,
os.getenv and one-argument functions such as core_luminosity(t)).
`to_lua` renders a parameter dict back to Lua.
"""
from __future__ import annotations

import math
import os
import re
from typing import Any, Callable

DEFAULTS: dict[str, Any] = {
    "data_atomic_file": "", "data_fuzzline_file": "",
    "grid_type": "grid_1D_sphere", "model_file": "",
    "run_do_restart": 0, "run_do_checkpoint": 0, "run_do_checkpoint_test": 0,
    "run_restart_file": "chk.h5", "run_checkpoint_name_base": "chk",
    "run_chk_timestep_interval": 0, "run_chk_walltime_interval": 0.0,
    "run_chk_simtime_interval": 0.0, "run_chk_walltime_max_buffer": 0.0,
    "run_chk_walltime_max": 0.0, "run_chk_number_start": 0,
    "hydro_module": "none",
    "transport_module": "monte_carlo", "transport_nu_grid": [1, 1, 1],
    "transport_radiative_equilibrium": 0, "transport_steady_iterate": 0,
    "transport_boundary_in_reflect": 0, "transport_boundary_out_reflect": 0,
    "transport_store_Jnu": 1, "transport_use_ddmc": 0,
    "transport_ddmc_tau_threshold": 100, "transport_fleck_alpha": 0,
    "transport_fix_rng_seed": 0, "transport_rng_seed": 0,
    "transport_solve_Tgas_with_updated_opacities": 0,
    "transport_fix_Tgas_during_transport": 0, "transport_set_Tgas_to_Trad": 0,
    "core_n_emit": 0, "core_radius": 0, "core_luminosity": 0, "core_temperature": 0,
    "core_photon_frequency": 0, "core_timescale": 0, "core_spectrum_file": "",
    "core_fix_luminosity": 0,
    "particles_max_total": 1e7, "particles_n_emit_radioactive": 0,
    "particles_n_emit_thermal": 0, "particles_n_initialize": 0,
    "particles_n_emit_pointsources": 0, "particles_pointsource_file": "",
    "particles_last_iter_pump": 1, "multiply_particles_n_emit_by_dt_over_dtmax": 0,
    "force_rprocess_heating": 0,
    "tstep_max_steps": 1000, "tstep_time_start": 0.0, "tstep_time_stop": 100.0,
    "tstep_max_dt": 1000.0, "tstep_min_dt": 0.0, "tstep_max_delta": 0.1,
    "output_write_atomic_levels": 0, "output_write_radiation": 0,
    "output_write_plt_file_time": 1, "output_write_plt_log_space": 0,
    "output_write_mass_fractions": 0,
    "limits_temp_max": 1e8, "limits_temp_min": 1000,
    "opacity_grey_opacity": 0, "opacity_zone_specific_grey_opacity": 0,
    "opacity_user_defined": 0, "opacity_epsilon": 1.0, "opacity_atom_zero_epsilon": [],
    "opacity_electron_scattering": 0, "opacity_line_expansion": 0,
    "opacity_fuzz_expansion": 0, "opacity_bound_free": 0, "opacity_bound_bound": 0,
    "opacity_free_free": 0, "opacity_use_nlte": 0, "opacity_atoms_in_nlte": [],
    "opacity_use_collisions_nlte": 1, "opacity_no_ground_recomb": 0,
    "opacity_minimum_extinction": 0, "opacity_maximum_opacity": 1e40,
    "opacity_no_scattering": 0, "dont_decay_composition": 0,
    "opacity_compton_scatter_photons": 0,
    "line_velocity_width": 0, "line_profile": "voigt", "line_x_extent": 100,
    "spectrum_name": "spectrum", "spectrum_time_grid": [0, 1, 1],
    "spectrum_nu_grid": [1, 1, 1], "spectrum_n_mu": 1, "spectrum_n_phi": 1,
    "spectrum_suppress_txt": 0, "gamma_name": "", "gamma_nu_grid": [1, 1, 1],
    "spectrum_particle_list_name": "", "spectrum_particle_list_maxn": 1e9,
    # knobs of this implementation (no reference counterpart): the per-packet
    # segment limit (0: 10^7), after which a packet stops and the step
    # returns SED_ERR_LIMIT
    "gpu_max_segments": 0,
}


class Params:
    """Parameter lookup with the reference's fallback order: the parameter
    file first, then the defaults (ParameterReader::getScalar)."""

    def __init__(self, values: dict[str, Any] | None = None, defaults: dict[str, Any] | None = None):
        self.values = dict(values or {})
        self.defaults = dict(DEFAULTS if defaults is None else defaults)

    def get(self, name: str) -> Any:
        if name in self.values:
            return self.values[name]
        if name in self.defaults:
            return self.defaults[name]
        raise KeyError('Can\'t find parameter "%s" in either param file or defaults' % name)

    def scalar(self, name: str, kind=float):
        v = self.get(name)
        if callable(v):
            raise TypeError("parameter %s is a function" % name)
        if kind is int:
            return int(v)  # Lua numbers read as int truncate (lua_tointeger)
        return kind(v)

    def vector(self, name: str) -> list:
        v = self.get(name)
        return list(v) if isinstance(v, (list, tuple)) else [v]

    def function(self, name: str, x: float) -> float:
        """ParameterReader::getFunction: a Lua function of one argument, or a number"""
        v = self.get(name)
        return float(v(x)) if callable(v) else float(v)

    def __getitem__(self, name):
        return self.get(name)


# ------------------------------------------------------------------ Lua writer
def _lua_value(v) -> str:
    if isinstance(v, bool):
        return "1" if v else "0"
    if isinstance(v, (int,)):
        return str(v)
    if isinstance(v, float):
        if math.isinf(v):
            return "math.huge" if v > 0 else "-math.huge"
        return repr(v)
    if isinstance(v, str):
        return '"' + v.replace("\\", "\\\\").replace('"', '\\"') + '"'
    if isinstance(v, (list, tuple)):
        return "{" + ", ".join(_lua_value(x) for x in v) + "}"
    raise TypeError("cannot render %r as Lua" % (v,))


def to_lua(values: dict[str, Any]) -> str:
    lines = []
    for k, v in values.items():
        if callable(v):
            src = getattr(v, "lua_source", None)
            if src is None:
                raise TypeError("function parameter %s has no Lua source" % k)
            lines.append(src)
        else:
            lines.append("%s = %s" % (k, _lua_value(v)))
    return "\n".join(lines) + "\n"


# ------------------------------------------------------------------ Lua reader
_TOKEN = re.compile(r"""
    (?P<ws>\s+|--[^\n]*) |
    (?P<num>(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?) |
    (?P<str>"(?:[^"\\]|\\.)*"|'(?:[^'\\]|\\.)*') |
    (?P<name>[A-Za-z_][A-Za-z_0-9]*(?:\.[A-Za-z_][A-Za-z_0-9]*)*) |
    (?P<op>\.\.|==|~=|<=|>=|[-+*/^%(){},=;<>])
""", re.X)


def _tokens(src: str):
    pos = 0
    out = []
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m:
            raise SyntaxError("unsupported Lua near %r" % src[pos:pos + 30])
        pos = m.end()
        if m.lastgroup == "ws":
            continue
        out.append((m.lastgroup, m.group()))
    return out


class _LuaSubset:
    def __init__(self, src: str, env: dict[str, Any]):
        self.t = _tokens(src)
        self.i = 0
        self.env = env

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and tok[1] != val:
            raise SyntaxError("expected %r, got %r" % (val, tok[1]))
        self.i += 1
        return tok

    def run(self):
        while self.i < len(self.t):
            kind, val = self.peek()
            if val == ";":
                self.take()
            elif val == "function":
                self.function_def()
            elif kind == "name" and val == "local":
                self.take()
            elif kind == "name":
                name = self.take()[1]
                self.take("=")
                self.env[name] = self.expr()
            else:
                raise SyntaxError("unexpected %r" % val)
        return self.env

    def function_def(self):
        self.take("function")
        name = self.take()[1]
        self.take("(")
        arg = self.take()[1]
        self.take(")")
        self.take("return")
        start = self.i
        # body is a single return expression followed by `end`
        depth = 0
        while not (self.peek()[1] == "end" and depth == 0):
            v = self.take()[1]
            depth += v == "("
            depth -= v == ")"
        body = self.t[start:self.i]
        self.take("end")
        env = self.env

        def f(x, body=body, arg=arg):
            sub = _LuaSubset("", dict(env))
            sub.t = list(body)
            sub.env[arg] = x
            return sub.expr()

        f.lua_source = None
        self.env[name] = f

    # precedence: .. < + - < * / % < unary < ^
    def expr(self):
        left = self.additive()
        if self.peek()[1] == "..":
            self.take()
            right = self.expr()
            return _lstr(left) + _lstr(right)
        return left

    def additive(self):
        v = self.term()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            r = self.term()
            v = v + r if op == "+" else v - r
        return v

    def term(self):
        v = self.unary()
        while self.peek()[1] in ("*", "/", "%"):
            op = self.take()[1]
            r = self.unary()
            v = v * r if op == "*" else (v / r if op == "/" else math.fmod(v, r))
        return v

    def unary(self):
        if self.peek()[1] == "-":
            self.take()
            return -self.unary()
        return self.power()

    def power(self):
        b = self.atom()
        if self.peek()[1] == "^":
            self.take()
            return b ** self.unary()
        return b

    def atom(self):
        kind, val = self.take()
        if kind == "num":
            f = float(val)
            return int(f) if re.fullmatch(r"\d+", val) else f
        if kind == "str":
            return bytes(val[1:-1], "utf-8").decode("unicode_escape")
        if val == "(":
            v = self.expr()
            self.take(")")
            return v
        if val == "{":
            items = []
            while self.peek()[1] != "}":
                items.append(self.expr())
                if self.peek()[1] in (",", ";"):
                    self.take()
            self.take("}")
            return items
        if kind == "name":
            if val == "os.getenv":
                self.take("(")
                key = self.expr()
                self.take(")")
                return os.environ.get(key)
            if val == "math.huge":
                return math.inf
            if val.startswith("math."):
                fn = getattr(math, val[5:])
                self.take("(")
                a = self.expr()
                self.take(")")
                return fn(a)
            v = self.env.get(val)
            if callable(v) and self.peek()[1] == "(":
                self.take("(")
                a = self.expr()
                self.take(")")
                return v(a)
            return v
        raise SyntaxError("unexpected token %r" % val)


def _lstr(v) -> str:
    if isinstance(v, float) and v.is_integer():
        return str(int(v))
    return str(v)


def read_param_file(path: str) -> Params:
    """Reads a Sedona parameter file (the Lua subset above).  A
    `defaults_file` it names is read the same way for the fallback values."""
    with open(path) as f:
        env = _LuaSubset(f.read(), {}).run()
    defaults = dict(DEFAULTS)
    dfile = env.get("defaults_file")
    if isinstance(dfile, str) and os.path.exists(dfile):
        with open(dfile) as f:
            defaults.update(_LuaSubset(f.read(), {}).run())
    env.pop("defaults_file", None)
    return Params(env, defaults)

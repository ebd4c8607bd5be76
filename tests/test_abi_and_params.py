"""CPU checks of the boundary: the CUDA library loads and exports every
entry point include/*.h declares (no compute calls), the oracle mirrors the
same calls, and the Lua parameter reader handles Sedona parameter files."""
import ctypes as C
import glob
import math
import os
import re

import pytest

from pubsed_b200 import _lib, params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(sed_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_abi():
    names = declared_functions()
    for n in _lib.EXPORTED:
        assert n in names, n


def test_library_loads_and_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    lib = C.CDLL(_lib.LIB_PATH)  # loading makes no CUDA calls
    for n in declared_functions():
        assert hasattr(lib, n), n
    lib.sed_version.restype = C.c_char_p
    assert b"sm_100a" in lib.sed_version()


def test_oracle_mirrors_the_abi():
    import oracle_lib
    lib = oracle_lib.oracle_lib()
    for n in declared_functions():
        if n in ("sed_step", "sed_version", "sed_lte_electron_density_noalloc"):
            continue
        # device-pointer forms have no CPU counterpart (their host forms are checked)
        if n.endswith("_dev"):
            continue
        # a batch is checked model by model against separate oracle contexts
        if n.startswith("sed_batch_"):
            continue
        assert hasattr(lib, n.replace("sed_", "oracle_", 1)), n


PARAM_FILE = """
-- a Sedona parameter file
sedona_home   = os.getenv('SEDONA_TEST_HOME')
defaults_file = sedona_home.."/defaults.lua"
model_file    = "../models/vacuum_1D.mod"
transport_nu_grid  = {0.2e14,5.0e15,0.01,1}  -- frequency grid
transport_radiative_equilibrium  = 1
core_n_emit      = 2e5
core_radius      = 5.0e14
core_temperature = 1.0e4
tstep_time_start = 20*3600.0*24.0
spectrum_nu_grid   = transport_nu_grid
function core_luminosity(t) return 1e43*(1 + t/86400)^-2 end
"""


def test_lua_parameter_file(tmp_path, monkeypatch):
    monkeypatch.setenv("SEDONA_TEST_HOME", str(tmp_path))
    (tmp_path / "defaults.lua").write_text(params.to_lua({"opacity_epsilon": 0.5, "core_n_emit": 0}))
    p = tmp_path / "param.lua"
    p.write_text(PARAM_FILE)
    P = params.read_param_file(str(p))
    assert P.vector("transport_nu_grid") == [0.2e14, 5.0e15, 0.01, 1]
    assert P.vector("spectrum_nu_grid") == [0.2e14, 5.0e15, 0.01, 1]
    assert P.scalar("transport_radiative_equilibrium", int) == 1
    assert P.scalar("core_n_emit", int) == 200000
    assert P.scalar("tstep_time_start") == 20 * 3600.0 * 24.0
    assert P.scalar("opacity_epsilon") == 0.5          # from the defaults file
    assert P.scalar("transport_store_Jnu", int) == 1  # built-in default
    assert math.isclose(P.function("core_luminosity", 86400.0), 1e43 / 4)
    assert P.get("model_file") == "../models/vacuum_1D.mod"
    with pytest.raises(KeyError):
        P.get("not_a_parameter")


def test_lua_roundtrip():
    vals = {"a": 1, "b": 2.5e-3, "c": "x.h5", "d": [1e14, 1e16, 0.0045, 1]}
    import tempfile
    with tempfile.NamedTemporaryFile("w", suffix=".lua", delete=False) as f:
        f.write(params.to_lua(vals))
    P = params.read_param_file(f.name)
    for k, v in vals.items():
        assert P.get(k) == v

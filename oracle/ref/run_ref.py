"""oracle/ref/run_ref.py -- TEST INFRASTRUCTURE.

Runs the reference harness (oracle/_ref/sedona_ref, built from the
reference's own sources by oracle/ref/build_ref.sh) on a Workload:
renders the Lua parameter file and its defaults file, the model file and the
in-memory-HDF5 store (atomic data, fuzz lines, 3-D models), runs one mode
and loads the arrays it writes.  Used by the tests, the golden-fixture
script and bench.py's reference arm only.
"""
from __future__ import annotations

import json
import os
import struct
import subprocess
import tempfile
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(os.path.dirname(HERE), "_ref", "sedona_ref")
# the same harness with its "gpu" mode: the compiled C++ binding of the B200
# library stepping the reference's transport
REF_GPU_BIN = os.path.join(os.path.dirname(HERE), "_ref", "sedona_ref_gpu")


def available() -> bool:
    return os.path.exists(REF_BIN) and os.access(REF_BIN, os.X_OK)


# ------------------------------------------------------------------ store file
class Store:
    """Records served by the HDF5 stand-in (format read by ref_harness.cpp)."""

    def __init__(self):
        self.buf = bytearray()

    @staticmethod
    def _s(s: str) -> bytes:
        b = s.encode()
        return struct.pack("<I", len(b)) + b

    def attr(self, file: str, obj: str, name: str, v: int):
        self.buf += struct.pack("<B", 2) + self._s(file) + self._s(obj) + self._s(name) + struct.pack("<i", int(v))

    def dset(self, file: str, path: str, a, dims=None):
        a = np.asarray(a)
        is_int = np.issubdtype(a.dtype, np.integer)
        dims = list(a.shape) if dims is None else list(dims)
        if not dims:
            dims = [1]
        rec = struct.pack("<B", 1 if is_int else 0) + self._s(file) + self._s(path)
        rec += struct.pack("<I", len(dims)) + b"".join(struct.pack("<Q", int(d)) for d in dims)
        flat = a.reshape(-1)
        rec += struct.pack("<Q", flat.size)
        rec += flat.astype("<i4" if is_int else "<f8").tobytes()
        self.buf += rec

    def write(self, path: str):
        with open(path, "wb") as f:
            f.write(bytes(self.buf))


def atoms_to_store(store: Store, atom_file: str, fuzz_file: str, model):
    """Old-style atomic data layout (AtomicData.cpp:459-651) and the fuzz
    file layout (AtomicData.cpp:783-820)."""
    for a in model.atoms:
        g = "%d/" % a.Z
        store.attr(atom_file, g, "n_ions", a.n_ions)
        store.attr(atom_file, g, "n_levels", a.lev_ion.size)
        store.attr(atom_file, g, "n_lines", a.line_l.size)
        store.dset(atom_file, g + "ion_chi", np.asarray(a.ion_chi, np.float64))
        store.dset(atom_file, g + "ion_ground", np.asarray(a.ion_ground, np.int32))
        store.dset(atom_file, g + "level_i", np.asarray(a.lev_ion, np.int32))
        store.dset(atom_file, g + "level_g", np.asarray(a.lev_g, np.int32))
        store.dset(atom_file, g + "level_E", np.asarray(a.lev_E, np.float64))
        if a.line_l.size:
            store.dset(atom_file, g + "line_l", np.asarray(a.line_l, np.int32))
            store.dset(atom_file, g + "line_u", np.asarray(a.line_u, np.int32))
            store.dset(atom_file, g + "line_A", np.asarray(a.line_A, np.float64))
        store.attr(fuzz_file, g, "n_lines", a.fuzz_nu.size)
        store.dset(fuzz_file, g + "nu", np.asarray(a.fuzz_nu, np.float64))
        store.dset(fuzz_file, g + "ion", np.asarray(a.fuzz_ion, np.int32))
        store.dset(fuzz_file, g + "gf", np.asarray(a.fuzz_gf, np.float64))
        store.dset(fuzz_file, g + "El", np.asarray(a.fuzz_El, np.float64))


def write_mod_file(path: str, zones):
    """1D_sphere ASCII model (grid_1D_sphere.cpp:241-332): "SNR" (r_out = v t)
    for homologous models, "standard" (explicit r_out column) otherwise;
    numbers are written with 17 significant digits so they parse back
    exactly."""
    snr = bool(zones.homologous)
    with open(path, "w") as f:
        f.write("1D_sphere %s\n" % ("SNR" if snr else "standard"))
        f.write("%d %r %r %d\n" % (zones.n_zones, float(zones.r_min), float(zones.t_now), zones.n_elems))
        f.write(" ".join("%d.%d" % (z, a) for z, a in zip(zones.elem_Z, zones.elem_A)) + "\n")
        for i in range(zones.n_zones):
            row = [] if snr else [repr(float(zones.r_out[i]))]
            row += [repr(float(zones.v[i])), repr(float(zones.rho[i])), repr(float(zones.T[i]))]
            row += [repr(float(x)) for x in zones.X[i]]
            f.write(" ".join(row) + "\n")


def model3d_to_store(store: Store, model_file: str, zones):
    """3-D Cartesian model layout read by grid_3D_cart::read_model_file
    (src/grid/grid_3D_cart.cpp:27-200): explicit walls x_out/y_out/z_out + rmin."""
    nx, ny, nz = zones.shape
    store.dset(model_file, "time", np.array([zones.t_now]))
    store.dset(model_file, "comp", zones.X.reshape(nx, ny, nz, -1))
    store.dset(model_file, "Z", np.asarray(zones.elem_Z, np.int32))
    store.dset(model_file, "A", np.asarray(zones.elem_A, np.int32))
    store.dset(model_file, "x_out", zones.axes[0].right)
    store.dset(model_file, "y_out", zones.axes[1].right)
    store.dset(model_file, "z_out", zones.axes[2].right)
    store.dset(model_file, "rmin", np.array([zones.axes[0].min, zones.axes[1].min, zones.axes[2].min]))
    store.dset(model_file, "rho", zones.rho)
    store.dset(model_file, "temp", zones.T)
    for name in ("vx", "vy", "vz", "erad"):
        store.dset(model_file, name, np.zeros(zones.n_zones))


def render(workload, outdir: str, n_packets: Optional[int] = None) -> tuple[str, str]:
    """Writes param.lua, defaults.lua, the model and the store into outdir."""
    from pubsed_b200.params import DEFAULTS, to_lua
    params = dict(workload.params)
    if n_packets is not None:
        params["core_n_emit"] = int(n_packets)
    store = Store()
    atom_file = os.path.join(outdir, "atoms.h5")
    fuzz_file = os.path.join(outdir, "fuzz.h5")
    with open(atom_file, "w") as f:  # transport::init only checks that the file opens
        f.write("served by the oracle HDF5 stand-in\n")
    params["data_atomic_file"] = atom_file
    if workload.atoms is not None:
        atoms_to_store(store, atom_file, fuzz_file, workload.atoms)
        with open(fuzz_file, "w") as f:
            f.write("served by the oracle HDF5 stand-in\n")
        params["data_fuzzline_file"] = fuzz_file
    z = workload.zones
    if z.type == 0:
        mf = os.path.join(outdir, "model.mod")
        write_mod_file(mf, z)
    else:
        mf = os.path.join(outdir, "model.h5")
        model3d_to_store(store, mf, z)
        params["grid_type"] = "grid_3D_cart"
    params["model_file"] = mf
    dpath = os.path.join(outdir, "defaults.lua")
    with open(dpath, "w") as f:
        f.write(to_lua(DEFAULTS))
    params["defaults_file"] = dpath
    ppath = os.path.join(outdir, "param.lua")
    with open(ppath, "w") as f:
        f.write(to_lua(params))
    spath = os.path.join(outdir, "store.bin")
    store.write(spath)
    return ppath, spath


def load_outputs(prefix: str) -> dict:
    with open(prefix + ".meta.json") as f:
        meta = json.load(f)
    out = dict(meta["scalars"])
    for name, m in meta["arrays"].items():
        dt = {"f64": np.float64, "i32": np.int32, "i64": np.int64}[m["type"]]
        out[name] = np.fromfile(m["file"], dtype=dt, count=m["count"])
    return out


def run(workload, mode: str, n_packets: Optional[int] = None, threads: Optional[int] = None,
        seed: Optional[int] = None, steps: int = 1, timeout: float = 3600, keep_dir: Optional[str] = None,
        dt: Optional[float] = None, precision: Optional[int] = None) -> dict:
    """mode: replay | free | opacity, or gpu (sedona_ref_gpu: the binding's
    steps; precision: enum sed_precision).  dt: the step of a time-dependent
    run.  Returns the harness outputs."""
    binary = REF_GPU_BIN if mode == "gpu" else REF_BIN
    if not (os.path.exists(binary) and os.access(binary, os.X_OK)):
        raise FileNotFoundError("reference harness not built: " + binary)
    d = keep_dir or tempfile.mkdtemp(prefix="sedref_")
    ppath, spath = render(workload, d, n_packets)
    prefix = os.path.join(d, "out")
    cmd = [binary, mode, ppath, prefix, "--store", spath, "--steps", str(steps)]
    if precision is not None:
        cmd += ["--precision", str(int(precision))]
    if dt is not None:
        cmd += ["--dt", repr(float(dt))]
    if seed is not None:
        cmd += ["--seed", str(seed)]
    else:
        cmd += ["--seed", str(int(workload.params.get("transport_rng_seed", 0)))]
    if threads is not None:
        cmd += ["--threads", str(threads)]
    env = dict(os.environ)
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env, cwd=d)
    if r.returncode != 0:
        raise RuntimeError("sedona_ref failed (%d): %s\n%s" % (r.returncode, r.stderr[-2000:], r.stdout[-2000:]))
    out = load_outputs(prefix)
    out["_stdout"] = r.stdout
    out["_dir"] = d
    return out

"""The allocation-free LTE entry point against the regular path.

sed_lte_electron_density_noalloc serves callers that cannot allocate device
memory when they need the result (their device memory is owned by their own
pool allocator, or the call sits in a per-step loop that cannot take the
synchronisation of cudaMalloc/cudaFree).  Its scratch is a fixed array in
the library.  This test (the test allocates its buffers; the entry point
does not) checks two consecutive calls, with different zone counts and
temperatures, against the electron densities the regular sed_set_opacity
path produces for the same zones.  The file is named to run last.
"""
import ctypes as C

import numpy as np
import pytest

from pubsed_b200 import abi, workloads
import oracle_lib

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # same kernel arithmetic; the FP64 parity tolerance of the GPU tests


def _regular_n_elec(sed_lib, w):
    g = oracle_lib.Engine(sed_lib, "sed_", w)
    g.set_opacity(1.0)
    ne = g.opacity()["n_elec"]
    g.close()
    return ne


def _noalloc_n_elec(sed_lib, w):
    import torch

    dev = torch.device("cuda:0")
    keep = abi.Keep()
    a = w.atomic_struct(keep)  # host arrays in the ABI layout
    na = a.n_atoms
    n_ions = int(np.ctypeslib.as_array(a.ion_off, shape=(na + 1,))[na])
    n_levs = int(np.ctypeslib.as_array(a.lev_off, shape=(na + 1,))[na])

    def d(ptr, n, dt):
        host = np.ctypeslib.as_array(ptr, shape=(n,)).copy()
        return torch.from_numpy(host).to(dev)

    t_ion_off = d(a.ion_off, na + 1, np.int32)
    t_ion_chi = d(a.ion_chi, n_ions, np.float64)
    t_lev_off = d(a.lev_off, na + 1, np.int32)
    t_lev_ion = d(a.lev_ion, n_levs, np.int32)
    t_lev_g = d(a.lev_g, n_levs, np.int32)
    t_lev_E = d(a.lev_E, n_levs, np.float64)
    z = w.zones
    t_rho = torch.from_numpy(z.rho.copy()).to(dev)
    t_T = torch.from_numpy(z.T.copy()).to(dev)
    t_X = torch.from_numpy(np.ascontiguousarray(z.X.reshape(-1))).to(dev)
    t_A = torch.from_numpy(z.elem_A.astype(np.int32)).to(dev)
    t_ne = torch.zeros(z.n_zones, dtype=torch.float64, device=dev)
    t_err = torch.full((z.n_zones,), -1, dtype=torch.int32, device=dev)

    ad = abi.AtomicData()
    ad.n_atoms = na
    ad.ion_off = C.cast(t_ion_off.data_ptr(), abi._ip)
    ad.ion_chi = C.cast(t_ion_chi.data_ptr(), abi._dp)
    ad.lev_off = C.cast(t_lev_off.data_ptr(), abi._ip)
    ad.lev_ion = C.cast(t_lev_ion.data_ptr(), abi._ip)
    ad.lev_g = C.cast(t_lev_g.data_ptr(), abi._ip)
    ad.lev_E = C.cast(t_lev_E.data_ptr(), abi._dp)
    P = w.P
    f = sed_lib.sed_lte_electron_density_noalloc
    f.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(abi.AtomicData),
                  C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    stream = torch.cuda.current_stream(dev)
    rc = f(z.n_zones, t_rho.data_ptr(), t_T.data_ptr(), t_X.data_ptr(), z.n_elems, t_A.data_ptr(), C.byref(ad),
           n_ions, n_levs, P.scalar("limits_temp_min"), P.scalar("limits_temp_max"), t_ne.data_ptr(),
           t_err.data_ptr(), C.c_void_p(stream.cuda_stream))
    assert rc == 0, rc
    torch.cuda.synchronize(dev)
    return t_ne.cpu().numpy(), t_err.cpu().numpy()


def test_noalloc_lte_matches_regular_path_twice(sed_lib):
    import torch

    # two calls in a row on the shared scratch array: a larger model first,
    # then a smaller and hotter one, so leftovers of the first call would show
    w1 = workloads.type_ia(n_packets=10, n_zones=48, n_lines=1000, n_bins=256, n_levels_per_ion=8, seed=21)
    w2 = workloads.type_ia(n_packets=10, n_zones=20, n_lines=1000, n_bins=256, n_levels_per_ion=8, seed=21)
    w2.zones.T = w2.zones.T * 1.3
    for w in (w1, w2):
        ne, err = _noalloc_n_elec(sed_lib, w)
        ref = _regular_n_elec(sed_lib, w)
        assert np.all(err == 0)
        assert np.all(ne > 0)
        assert np.max(np.abs(ne - ref) / np.abs(ref)) <= RTOL


def test_noalloc_rejects_oversized_request(sed_lib):
    f = sed_lib.sed_lte_electron_density_noalloc
    f.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(abi.AtomicData),
                  C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    ad = abi.AtomicData()
    ad.n_atoms = 1
    fake = C.cast(1, abi._ip)
    fake_d = C.cast(1, abi._dp)
    ad.ion_off = ad.lev_off = ad.lev_ion = ad.lev_g = fake
    ad.ion_chi = ad.lev_E = fake_d
    # 100000 zones x (2 + 2 + 2*2 + 2*2) doubles is far above the 4 MiB array;
    # the size check runs before any device access
    rc = f(100000, 1, 1, 1, 1, 1, C.byref(ad), 2, 2, 1e3, 1e8, 1, 1, None)
    assert rc == abi.SED_ERR_CAPACITY
    # counts whose 64-bit product zones x doubles-per-zone wraps around to
    # 458740, below the array size: still refused
    nz, na, ni, nl = 2147450882, 1431677610, 1431677609, 1431677609
    assert (nz * (2 * na + 2 + 2 * ni + 2 * nl)) % 2**64 < 524288
    ad.n_atoms = na
    rc = f(nz, 1, 1, 1, na, 1, C.byref(ad), ni, nl, 1e3, 1e8, 1, 1, None)
    assert rc == abi.SED_ERR_CAPACITY
